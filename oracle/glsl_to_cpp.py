"""Mechanical GLSL -> C++ translation of the reference's fragment shaders, for
the shading pin (test infrastructure only; oracle/Makefile target ``shade``).

    python oracle/glsl_to_cpp.py SRC.glsl OUT.inc

The output is the shader's own source with only the edits C++ needs to
compile it against oracle/glsl_shim.hpp:

* float literals get an ``f`` suffix (GLSL literals are single precision);
* ``in`` / ``out`` / ``uniform`` qualifiers and ``layout(...)`` on globals are
  dropped (the harness sets the globals), ``out T x`` parameters become
  ``T& x``;
* swizzles ``e.rgb`` / ``e.xyz`` / ``e.xy`` / ``e.xz`` become calls
  ``rgb(e)`` ..., and ``v.rgb += e;`` becomes ``v = set_rgb(v, rgb(v) + (e));``.

Nothing else is touched: the statements, their order and their arithmetic are
the reference's.  The output goes under oracle/_ref/ (never committed).
"""
from __future__ import annotations

import re
import sys

_FLOAT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][-+]?\d+)?|\d+[eE][-+]?\d+)(?![\w.])")
_OPERAND = r"(texture\s*\([^()]*\)|[A-Za-z_]\w*(?:\[[^\]]*\])?)"


def translate(src: str) -> str:
    out = []
    for line in src.splitlines():
        code, sep, comment = line.partition("//")
        if code.lstrip().startswith("#"):
            if code.lstrip().startswith("#define"):
                code = _FLOAT.sub(r"\1f", code)
            out.append(code + (sep + comment if sep else ""))
            continue
        code = re.sub(r"^\s*layout\s*\([^)]*\)\s*", "", code)
        code = re.sub(r"^\s*(in|out|uniform)\s+", "", code)
        code = re.sub(r"\bout\s+([A-Za-z_]\w*)\s+([A-Za-z_]\w*)", r"\1& \2", code)
        code = _FLOAT.sub(r"\1f", code)
        m = re.match(r"^(\s*)([A-Za-z_]\w*)\.rgb\s*\+=\s*(.*);\s*$", code)
        if m:
            code = f"{m.group(1)}{m.group(2)} = set_rgb({m.group(2)}, rgb({m.group(2)}) + ({m.group(3)}));"
        for sw in ("rgb", "xyz", "xy", "xz"):
            code = re.sub(_OPERAND + r"\." + sw + r"\b", sw + r"(\1)", code)
        out.append(code + (sep + comment if sep else ""))
    return "\n".join(out) + "\n"


if __name__ == "__main__":
    with open(sys.argv[1]) as f:
        text = f.read()
    with open(sys.argv[2], "w") as f:
        f.write(f"// translated from {sys.argv[1].rsplit('/', 1)[-1]} by glsl_to_cpp.py\n")
        f.write(translate(text))

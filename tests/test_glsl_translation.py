"""The mechanical GLSL -> C++ translation behind the shading pin
(oracle/glsl_to_cpp.py): only the edits C++ needs, nothing else."""
import importlib.util
import pathlib

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _tr():
    spec = importlib.util.spec_from_file_location("glsl_to_cpp", ROOT / "oracle" / "glsl_to_cpp.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.translate


def test_literals_qualifiers_and_swizzles():
    t = _tr()
    src = "\n".join([
        "#define EPSILON 1e-3",
        "layout (location = 0) out vec4 color;",
        "uniform vec4 phaseColors[4];",
        "in vec3 fragPos;",
        "void f(vec3 a, out Hit hit) {",
        "  float x = 0.5 * a.x + 1.0 / 2 + .25 + 3e2;",
        "  vec2 p = pos.xy - boxMin.xy; vec2 q = hitPos.xz;",
        "  vec3 c = texture(skybox, direction).rgb + phaseColors[i].rgb;",
        "  tintColor.rgb += colorFractions[i] * phaseColors[i].rgb;",
        "  float a2 = phaseColors[0].a; // 0.5 stays in comments",
        "}",
    ])
    out = t(src).splitlines()
    assert out[0] == "#define EPSILON 1e-3f"
    assert out[1] == "vec4 color;"
    assert out[2] == "vec4 phaseColors[4];"
    assert out[3] == "vec3 fragPos;"
    assert out[4] == "void f(vec3 a, Hit& hit) {"
    assert out[5] == "  float x = 0.5f * a.x + 1.0f / 2 + .25f + 3e2f;"
    assert out[6] == "  vec2 p = xy(pos) - xy(boxMin); vec2 q = xz(hitPos);"
    assert out[7] == "  vec3 c = rgb(texture(skybox, direction)) + rgb(phaseColors[i]);"
    assert out[8] == "  tintColor = set_rgb(tintColor, rgb(tintColor) + (colorFractions[i] * rgb(phaseColors[i])));"
    assert out[9] == "  float a2 = phaseColors[0].a; // 0.5 stays in comments"


def test_integers_and_names_untouched():
    t = _tr()
    src = "int xi = int(xz.x + 100);\nif ((xi + zi) % 2 == 0) return vec3(1, 0, 0);\nfloat v2 = x2.y;"
    out = t(src).splitlines()
    assert out[0] == "int xi = int(xz.x + 100);"
    assert out[1] == "if ((xi + zi) % 2 == 0) return vec3(1, 0, 0);"
    assert out[2] == "float v2 = x2.y;"

"""The header-only C++ wrapper compiles and links against the library as a
reference user would build it (g++ -std=c++14, no CUDA headers needed)."""
import pathlib
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _build(tmp_path, built_library):
    exe = tmp_path / "wrapper_demo"
    cmd = ["g++", "-std=c++14", "-O1", f"-I{ROOT / 'include'}", str(ROOT / "tests" / "cpp" / "wrapper_demo.cpp"),
           str(built_library), f"-Wl,-rpath,{built_library.parent}", "-o", str(exe)]
    subprocess.run(cmd, check=True)
    return exe


def test_wrapper_builds_and_runs(tmp_path, built_library):
    exe = _build(tmp_path, built_library)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_wrapper_steps_on_gpu(tmp_path, built_library):
    exe = _build(tmp_path, built_library)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "particles" in r.stdout, r.stdout + r.stderr

"""The C++ facade (include/glscam.hpp): a caller written against the
reference's class names (tests/cpp/facade_demo.cpp) compiles and links
against libglscam.so on the CPU, and runs end to end on the GPU."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIBDIR = ROOT / "glasscamerapublic_b200"


def _build(tmp_path) -> Path:
    exe = tmp_path / "facade_demo"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}",
           str(ROOT / "tests" / "cpp" / "facade_demo.cpp"), f"-L{LIBDIR}", "-lglscam", f"-Wl,-rpath,{LIBDIR}",
           "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_facade_compiles_and_links(tmp_path):
    assert _build(tmp_path).exists()


@pytest.mark.gpu
def test_facade_runs_end_to_end(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "facade ok" in r.stdout, r.stdout + r.stderr

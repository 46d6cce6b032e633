"""The C++ drop-in headers: the program tests/dropin/test_dropin.cpp compiles
against include/b2s/math/*.hpp and libb2s.so (CPU), and passes its
known-answer checks on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "dropin", "test_dropin.cpp")
EXE = os.path.join(ROOT, "tests", "dropin", "test_dropin")


def build():
    lib_dir = os.path.join(ROOT, "cpp-fem-solver_b200")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++17", "-O2", f"-I{os.path.join(ROOT, 'include', 'b2s')}", SRC, "-o", EXE,
                    f"-L{lib_dir}", "-lb2s", f"-Wl,-rpath,{lib_dir}"], check=True)


def test_dropin_compiles(b2s):
    b2s.load_extension()
    build()
    assert os.path.exists(EXE)


@pytest.mark.gpu
def test_dropin_runs(b2s):
    build()
    out = subprocess.run([EXE], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "ALL PASSED" in out.stdout

"""The planners on the CPU (host code compiled by nvcc, no GPU needed):
tests/band_plan/band_plan.cu checks that the band plan of a lower
triangle's strict transpose made from the lower pattern equals the plan made
from the transposed pattern (csrc/trsv_band.cuh), and that the chunk plan
(csrc/trsv_plan.hpp) does not depend on the number of host threads."""
import os
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "band_plan", "band_plan.cu")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not found")
def test_band_plan_transposed():
    inc = [f"-I{os.path.join(ROOT, 'include')}", f"-I{os.path.join(ROOT, 'cpp-fem-solver_b200', 'csrc')}"]
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "band_plan")
        subprocess.run([NVCC, "-std=c++17", "-O2", *inc, SRC, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("OK")

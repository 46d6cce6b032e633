"""The chunked triangular-solve planner (csrc/trsv_plan.hpp), checked on the
CPU: tests/chunk_sim/chunk_sim.cpp plans 2-D / 3-D stencil, 27-point block
and random triangles (scalar rows and 2x2 / 3x3 / 4x4 blocks) at several
shared-memory budgets, packs the value blobs the way k_chunk_pack does and
replays the index arithmetic of k_trsv_chunk / k_btrsv_chunk with every
shared-memory access bounds-checked; the solution must equal a serial
triangular solve bit for bit in FP64 and in both FP32 variants."""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "chunk_sim", "chunk_sim.cpp")


def test_chunk_plan_replay():
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "chunk_sim")
        subprocess.run([cxx, "-std=c++17", "-O2", SRC, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("OK")
    # the 512^2 IC(0) factor: levels of at most 64 rows, so one compute warp per chunk
    line = [l for l in out.stdout.splitlines() if l.startswith("512^2 lower (C5 IC0 L) [f64]")][0]
    assert int(line.split("level_rows=")[1].split()[0]) <= 64

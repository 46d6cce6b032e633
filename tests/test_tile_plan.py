"""The tiled persistent PCG kernel's planner (csrc/tile_plan.hpp), checked on
the CPU: tests/tile_sim/tile_sim.cpp plans 5-point grids (square, flat, tall,
odd sizes, fewer SMs, up to 16 sweeps) and replays the kernel's index
arithmetic -- each tile's k + 1 passes over its extended sets with the
pass-s prefix of layers, the dependencies as local indices, the SpMV over
local columns -- with every shared-memory index bounds-checked.  The owned
rows must equal the global Jacobi-sweep definition bit for bit (FP32) and
the SpMV the CSR product in column order (FP64); every row is owned once; a
pattern outside the kernel's reach (three upper entries in a row) gets no
plan."""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "tile_sim", "tile_sim.cpp")


def test_tile_plan_replay():
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "tile_sim")
        subprocess.run([cxx, "-std=c++17", "-O2", "-ffp-contract=off", "-pthread", SRC, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("ALL PASSED")
    # the benchmark's 512^2 grid with 6 sweeps: 2-D blocks, one CTA per SM at most
    line = [l for l in out.stdout.splitlines() if l.startswith("5-point 512^2, k=6")][0]
    assert "ok=1" in line and int(line.split("tiles=")[1].split()[0]) <= 148

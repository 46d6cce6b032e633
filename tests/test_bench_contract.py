"""bench.py's reference arm on the CPU: one solve of the benchmark system by
the reference compiled from its sources (oracle/_ref), printed as one JSON
line with the keys the benchmark contract asks of that arm.  The GPU arm's
line is produced on a B200 only."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref.so")),
                    reason="the compiled reference is not built")
def test_reference_arm_line():
    # run the arm in-process in a child interpreter, then report whether the
    # product library was ever mapped into that process
    code = ("import runpy, sys\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0']\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\n"
            "except SystemExit as e:\n    assert not e.code, e.code\n"
            "print('PRODUCT_MAPPED', 'libb2s.so' in open('/proc/self/maps').read())\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    assert lines[-1] == "PRODUCT_MAPPED False", lines[-1]
    line = json.loads(lines[-2])
    assert line["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "config",
              "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["higher_is_better"] is False and line["value"] > 0
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    # the same config object as the GPU arm prints for the same flags
    assert line["config"] == bench.arm_config(argparse.Namespace(method="learned_ic0_j6"), 1)
    assert line["config"]["workload"] == "grf_diffusion_512 pcg rtol1e-8"
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}

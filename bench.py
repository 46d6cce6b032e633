"""Benchmark: time-to-tolerance of preconditioned CG on one B200.

Workload (the configuration the headline metric is quoted on): -div(k grad u)
= f on a 512 x 512 grid, 5-point finite volume, harmonic-mean face
coefficients, log k a Gaussian random field (squared-exponential covariance,
correlation length 0.05, variance uniform in [1, 4] drawn per seed), f
uniform[-1, 1].  Systems are generated from held-out seeds (2000 + step on
rank 0; ranks > 0 use their own seed range).  A step is one complete solve:
preconditioner setup + PCG from x0 = 0 to relative residual 1e-8, verified by
an FP64 true residual b - Ax.  Matrix generation and upload are outside the
timed region; the right-hand side is already in HBM (`value`), or comes from
pinned host memory together with the matrix (`e2e`).

Arms
  default            this library (C ABI, sm_100a kernels)
  --impl reference   the reference library's own SMatrix::pcg(A, b, "ic")
                     compiled from its sources (oracle/_ref/libref.so), on
                     the host cores, same systems.

Multi-GPU: the systems are independent, so N GPUs run N replicas on disjoint
seeds ("scaling": "weak"); there is no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRID = 512
CORR = 0.05
TOL = 1e-8
MAXIT = 20000
L2_FLUSH_BYTES = 512 << 20
METRIC = "time-to-rtol 1e-8 & iters: learned/mixed-prec PCG vs plain FP64 PCG, 1 B200"


def replica_seeds(rank: int, count: int) -> list:
    """Seeds of the systems one replica solves: held-out seeds 2000+ on rank
    0, a disjoint range per further rank."""
    return [2000 + rank * 100000 + k for k in range(count)]


def max_over_ranks(value: float, device) -> float:
    """The largest value over all ranks (the whole job's time per step)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def load_b2s():
    import __graft_entry__ as ge
    return ge._load()


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        out_dir = os.environ.get("B2S_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out_dir, f"clocks_bench_{device}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            p = [s.strip() for s in line.split(",")]
            if len(p) >= 9:
                try:
                    rows.append(p)
                except Exception:
                    pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_system(b2s, seed):
    n, rp, ci, v = b2s.gen_grf_diffusion(N_GRID, seed, corr=CORR)
    b = b2s.uniform(seed, n)
    return n, rp, ci, v, b


# DRAM bytes (read + write) of one persistent PCG launch on the 512^2
# learned solve: dram__bytes.sum.per_second x gpu__time_duration.sum of an ncu
# capture of `bench.py --kernel solve_c5` (SpeedOfLight and
# MemoryWorkloadAnalysis sections, one launch): 3.40 GB/s x 11.02 ms for the
# fused tile kernel with 6 sweeps, 33.7 MB for the strip kernel with 8.
PCG_DRAM_BYTES = {"k_pcg_band": 33.7e6, "k_pcg_tile": 37.4e6}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "of measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "of fallback"


# ---------------------------------------------------------------- single-kernel mode

KERNELS = {
    "spmv_c2": "k_spmv_warp: CSR SpMV on the 128^3 7-point Poisson matrix (C2)",
    "baij_c4": "k_baij_warp<3>: BAIJ 3x3 matvec on the Q1 elasticity matrix (C4, 64^3 elements)",
    "trsv_c5": "k_trsv_grid5: FP32 IC(0) exact apply (L then L^T, 5-point grid schedule) on a 512^2 GRF system (C5)",
    "trsv_c5_fp64": "k_trsv_grid5: FP64 IC(0) exact apply (5-point grid schedule) on a 512^2 GRF system (C5)",
    "trsv_c5_j8": "k_trsv_band: FP32 IC(0) apply with 8 Jacobi sweeps per triangle on a 512^2 GRF system (C5)",
    "trsv_c2": "k_trsv_grid7: FP64 ILU(0) exact apply (7-point grid schedule) on the 128^3 Poisson matrix (C2)",
    "btrsv_c4": "k_btrsv_chunk: FP64 block ILU(0) apply on the Q1 elasticity matrix (C4, 64^3 elements)",
    "vcycle_c2": "SA-AMG V-cycle (k_jacobi, BAIJ matvecs, k_dense_solve) on C2",
    "vcycle_c4": "block SA-AMG V-cycle on the Q1 elasticity matrix (C4, 64^3 elements, 3x3 blocks)",
    "dense_c5": "k_linear_tc<64,128>: the learned network's tcgen05 dense layer on the 512^2 grid's node states "
                "(n=262144 rows, 64 -> 128)",
    "solve_c5": "one learned IC(0) PCG solve (6 Jacobi sweeps per triangle, the whole loop in the persistent "
                "kernel) on a 512^2 GRF system; a step is setup + solve",
    "pcg_c2_diag": "one PCG + diagonal solve on the 128^3 Poisson matrix (C2) to rtol 1e-10, no graphs: the "
                   "fused k_vec updates and the CSR SpMV",
    "gmres_c3_cgs2": "one GMRES(30) + ILU(0) solve with CGS2 orthogonalisation on the 96^3 convection-diffusion "
                     "matrix (C3): the batched Arnoldi dots and updates",
    "bilu0_setup_c4": "block ILU(0) factorisation of the Q1 elasticity matrix (C4, 64^3 elements)",
}


def run_kernel(args):
    """Launch one hot kernel `--warmup` + `--steps` times on its workload and
    report the mean CUDA-event time per launch.  For profilers (ncu -k ...):
    the inputs are built first, then only that kernel runs."""
    import ctypes as C

    import torch
    b2s = load_b2s()
    ctx = b2s.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    dev = torch.device("cuda", 0)
    k = args.kernel
    if k == "spmv_c2":
        n, rp, ci, v = b2s.gen_poisson3d(128)
        A = b2s.CSR(ctx, n, n, rp, ci, v)
        x = torch.rand(n, dtype=torch.float64, device=dev)
        y = torch.empty_like(x)
        step = lambda: A.spmv_device(x.data_ptr(), y.data_ptr())
    elif k == "baij_c4":
        nbr, rp, ci, v = b2s.gen_elasticity_q1(64)
        A = b2s.BAIJ(ctx, 3, nbr, nbr, rp, ci, v)
        x = torch.rand(3 * nbr, dtype=torch.float64, device=dev)
        y = torch.empty_like(x)
        step = lambda: ctx.check(b2s.lib().b2s_baij_matvec_device(ctx.h, A.h, C.c_void_p(x.data_ptr()),
                                                                  C.c_void_p(y.data_ptr())), "baij_matvec")
    elif k == "solve_c5":
        n, rp, ci, v = b2s.gen_grf_diffusion(N_GRID, 2003, corr=CORR)
        A = b2s.CSR(ctx, n, n, rp, ci, v)
        bt = torch.from_numpy(b2s.uniform(2003, n)).to(dev)
        xt = torch.zeros(n, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()

        def step():
            M = b2s.Precond(ctx, A, b2s.PC_LEARNED_IC0, precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=6,
                            factor_sweeps=5)
            b2s.solve_device(ctx, A, bt.data_ptr(), xt.data_ptr(), b2s.PCG, M, tol=TOL, maxit=MAXIT)
    elif k in ("pcg_c2_diag", "gmres_c3_cgs2"):
        if k == "pcg_c2_diag":
            n, rp, ci, v = b2s.gen_poisson3d(128)
            A = b2s.CSR(ctx, n, n, rp, ci, v)
            M = b2s.Precond(ctx, A, b2s.PC_DIAG)
            method, so = b2s.PCG, {"tol": 1e-10, "maxit": 2000, "use_graphs": 0}
        else:
            n, rp, ci, v = b2s.gen_convdiff3d(96)
            A = b2s.CSR(ctx, n, n, rp, ci, v)
            M = b2s.Precond(ctx, A, b2s.PC_ILU0)
            method, so = b2s.GMRES, {"tol": 1e-8, "maxit": 2000, "restart": 30, "orth": b2s.ORTH_CGS2,
                                     "use_graphs": 0}
        bt = torch.from_numpy(b2s.uniform(7, n)).to(dev)
        xt = torch.zeros(n, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        step = lambda: b2s.solve_device(ctx, A, bt.data_ptr(), xt.data_ptr(), method, M, **so)
    elif k == "bilu0_setup_c4":
        nbr, rp, ci, v = b2s.gen_elasticity_q1(64)
        A = b2s.BAIJ(ctx, 3, nbr, nbr, rp, ci, v)
        torch.cuda.synchronize()
        step = lambda: b2s.Precond(ctx, A, b2s.PC_BILU0)
    elif k == "dense_c5":
        n = N_GRID * N_GRID
        g = torch.Generator(device=dev).manual_seed(5)
        x = torch.randn(n, 64, generator=g, device=dev, dtype=torch.float32)
        w = (0.1 * torch.randn(128, 64, generator=g, device=dev)).to(torch.bfloat16)
        y = torch.empty(n, 128, dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        step = lambda: ctx.check(b2s.lib().b2s_dense_bf16_device(ctx.h, n, 64, 128, C.c_void_p(x.data_ptr()),
                                                                C.c_void_p(w.data_ptr()), None,
                                                                C.c_void_p(y.data_ptr())), "dense_bf16")
    else:
        if k in ("trsv_c5", "trsv_c5_fp64", "trsv_c5_j8"):
            n, rp, ci, v = b2s.gen_grf_diffusion(N_GRID, 2000, corr=CORR)
            A = b2s.CSR(ctx, n, n, rp, ci, v)
            if k == "trsv_c5_j8":
                M = b2s.Precond(ctx, A, b2s.PC_IC0, precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=8)
            else:
                M = b2s.Precond(ctx, A, b2s.PC_IC0, precision=b2s.FP32 if k == "trsv_c5" else b2s.FP64)
        elif k == "trsv_c2":
            n, rp, ci, v = b2s.gen_poisson3d(128)
            A = b2s.CSR(ctx, n, n, rp, ci, v)
            M = b2s.Precond(ctx, A, b2s.PC_ILU0)
        elif k == "btrsv_c4":
            nbr, rp, ci, v = b2s.gen_elasticity_q1(64)
            A = b2s.BAIJ(ctx, 3, nbr, nbr, rp, ci, v)
            n = 3 * nbr
            M = b2s.Precond(ctx, A, b2s.PC_BILU0)
        elif k == "vcycle_c2":
            n, rp, ci, v = b2s.gen_poisson3d(128)
            A = b2s.CSR(ctx, n, n, rp, ci, v)
            M = b2s.Precond(ctx, A, b2s.PC_SA_AMG)
        elif k == "vcycle_c4":
            nbr, rp, ci, v = b2s.gen_elasticity_q1(64)
            A = b2s.BAIJ(ctx, 3, nbr, nbr, rp, ci, v)
            n = 3 * nbr
            M = b2s.Precond(ctx, A, b2s.PC_BSA_AMG)
        else:
            raise SystemExit(f"unknown kernel {k}; one of {sorted(KERNELS)}")
        r = torch.rand(n, dtype=torch.float64, device=dev)
        z = torch.empty_like(r)
        step = lambda: ctx.check(b2s.lib().b2s_pc_apply_device(ctx.h, M.h, C.c_void_p(r.data_ptr()),
                                                              C.c_void_p(z.data_ptr())), "pc_apply")
    for _ in range(args.warmup):
        step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    out = {"kernel": k, "what": KERNELS[k], "launches": args.steps, "ms_per_step": ms}
    if k == "dense_c5":
        # X read once (n x 64 FP32), Y written once (n x 128 FP32), W (128 x 64 BF16)
        nbytes = n * (64 + 128) * 4 + 128 * 64 * 2
        pk, which = peaks()
        out.update({"algorithmic_bytes": nbytes, "achieved_gbs": nbytes / (ms * 1e-3) / 1e9,
                    "frac_hbm": nbytes / (ms * 1e-3) / 1e9 / pk["hbm_gbs"], "peak": which,
                    "tflops": 2.0 * n * 64 * 128 / (ms * 1e-3) / 1e12})
    print(json.dumps(out))
    ctx.close()
    return 0


# ---------------------------------------------------------------- config suite

def run_suite(args):
    """The other configurations of the benchmark definition (C1-C4), one JSON
    line per solver: GPU setup and solve time (CUDA events on the library's
    stream, inputs resident, best of `reps` after one warm-up), iterations and
    the FP64 true residual; beside it the reference's solver on the host cores
    (`oracle/_ref`, one run) where it has the same solver.  Documentation of
    the other configurations, not the benchmark line."""
    import torch
    b2s = load_b2s()
    ctx = b2s.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    dev = torch.device("cuda", 0)
    ref = None
    if not args.no_ref:
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle
            ref = oracle.Ref()
            ref.set_threads(os.cpu_count() or 1)
        except Exception as e:  # the compiled reference did not travel
            print(json.dumps({"suite": "reference unavailable", "why": str(e)[:200]}), flush=True)

    def gpu(A, n, kind, method, tol, maxit, reps=3, pco=None, so=None, x64=None):
        """Best of `reps` timed solves; error_vs_fp64 = ||x - x64|| / ||x64||."""
        bt = torch.from_numpy(b2s.uniform(7, n)).to(dev)
        best = None
        for r in range(reps + 1):
            xt = torch.zeros(n, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            e0, em, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            M = b2s.Precond(ctx, A, kind, **(pco or {})) if kind is not None else None
            em.record(stream)
            st = b2s.solve_device(ctx, A, bt.data_ptr(), xt.data_ptr(), method, M, tol=tol, maxit=maxit,
                                  **(so or {}))
            e1.record(stream)
            e1.synchronize()
            del M
            if r == 0:
                continue
            cur = {"setup_ms": round(e0.elapsed_time(em), 3), "solve_ms": round(em.elapsed_time(e1), 3),
                   "iterations": st["iterations"], "relres_true": st["relres_true"], "status": st["status"]}
            cur["total_ms"] = round(cur["setup_ms"] + cur["solve_ms"], 3)
            if x64 is not None:
                x = xt.cpu().numpy()
                cur["error_vs_fp64"] = float(np.linalg.norm(x - x64) / np.linalg.norm(x64))
            if best is None or cur["total_ms"] < best["total_ms"]:
                best = cur
        return best

    def fp64_solution(A, n, kind, method, so=None):
        """FP64 solution to rtol 1e-12 (the yardstick of each line's error)."""
        M = b2s.Precond(ctx, A, kind)
        x, st = b2s.solve(ctx, A, b2s.uniform(7, n), method, M, tol=1e-12, maxit=5000, **(so or {}))
        assert st["relres_true"] < 1e-11, st
        return x

    def cpu(rp, ci, v, n, method, pc, tol, maxit):
        if ref is None:
            return None
        Ar = ref.csr(n, n, rp, ci, v)
        t0 = time.perf_counter()
        _, it = ref.solve(Ar, method, pc, b2s.uniform(7, n), tol, maxit)
        return {"ms": round((time.perf_counter() - t0) * 1e3, 1), "it": it, "cores": os.cpu_count()}

    def emit(config, solver, g, r):
        line = {"config": config, "solver": solver, "gpu": g, "reference_cpu": r}
        if isinstance(r, dict) and g:
            line["speedup"] = round(r["ms"] / g["total_ms"], 1)
        print(json.dumps(line), flush=True)

    # the B200-native apply for comparison: FP32 factor, 8 Jacobi sweeps per triangle (not the exact solve)
    sweeps8 = {"precision": b2s.FP32, "trsv": b2s.TRSV_JACOBI, "trsv_sweeps": 8}

    # every line's error is against the FP64 solution of the same system to
    # rtol 1e-12 (SA-AMG PCG for the SPD systems, GMRES(30) + ILU(0) for C3)
    c = "C1 poisson2d 256^2, rtol 1e-8"
    n, rp, ci, v = b2s.gen_poisson2d(256)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    x64 = fp64_solution(A, n, b2s.PC_SA_AMG, b2s.PCG)
    emit(c, "pcg+diag", gpu(A, n, b2s.PC_DIAG, b2s.PCG, 1e-8, 20000, x64=x64),
         cpu(rp, ci, v, n, 0, "diag", 1e-8, 20000))
    emit(c, "pcg+ic0", gpu(A, n, b2s.PC_IC0, b2s.PCG, 1e-8, 20000, x64=x64), cpu(rp, ci, v, n, 0, "ic", 1e-8, 20000))
    emit(c, "pcg+ic0_fp32_j8 (inexact apply)", gpu(A, n, b2s.PC_IC0, b2s.PCG, 1e-8, 20000, pco=sweeps8, x64=x64),
         None)
    del A

    c = "C2 poisson3d 128^3, rtol 1e-10"
    n, rp, ci, v = b2s.gen_poisson3d(128)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    x64 = fp64_solution(A, n, b2s.PC_SA_AMG, b2s.PCG)
    for prec, pname in ((b2s.FP64, "fp64"), (b2s.FP32, "fp32")):
        emit(c, f"pcg+sa_amg_{pname}", gpu(A, n, b2s.PC_SA_AMG, b2s.PCG, 1e-10, 2000, pco={"precision": prec},
                                           x64=x64),
             "not run: the reference's aggregation does not coarsen this operator")
    emit(c, "pcg+ilu0", gpu(A, n, b2s.PC_ILU0, b2s.PCG, 1e-10, 2000, reps=1, x64=x64),
         cpu(rp, ci, v, n, 0, "ilu", 1e-10, 2000))
    emit(c, "pcg+ilu0_fp32_j8 (inexact apply)", gpu(A, n, b2s.PC_ILU0, b2s.PCG, 1e-10, 2000, reps=1, pco=sweeps8,
                                                    x64=x64), None)
    del A

    c = "C3 convdiff3d 96^3, rtol 1e-8"
    n, rp, ci, v = b2s.gen_convdiff3d(96)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    x64 = fp64_solution(A, n, b2s.PC_ILU0, b2s.GMRES, so={"restart": 30})
    emit(c, "bicgstab+ilu0", gpu(A, n, b2s.PC_ILU0, b2s.BICGSTAB, 1e-8, 2000, x64=x64),
         cpu(rp, ci, v, n, 1, "ilu", 1e-8, 2000))
    emit(c, "bicgstab+ilu0_fp32_j8 (inexact apply)", gpu(A, n, b2s.PC_ILU0, b2s.BICGSTAB, 1e-8, 2000, pco=sweeps8,
                                                         x64=x64), None)
    emit(c, "gmres30+ilu0", gpu(A, n, b2s.PC_ILU0, b2s.GMRES, 1e-8, 2000, so={"restart": 30}, x64=x64),
         cpu(rp, ci, v, n, 2, "ilu", 1e-8, 2000))
    emit(c, "fgmres30+ilu0_fp32+ir", gpu(A, n, b2s.PC_ILU0, b2s.FGMRES, 1e-8, 2000, pco={"precision": b2s.FP32},
                                        so={"restart": 30, "ir_steps": 5, "ir_inner_tol": 1e-4}, x64=x64), None)
    emit(c, "gmres30+ilu0_fp32 (FP32 factors and solves inside FP64 GMRES)",
         gpu(A, n, b2s.PC_ILU0, b2s.GMRES, 1e-8, 2000, pco={"precision": b2s.FP32}, so={"restart": 30}, x64=x64),
         None)
    del A

    c = "C4 elasticity Q1 64^3 elements (3x3 BAIJ), rtol 1e-8"
    nbr, rp, ci, v = b2s.gen_elasticity_q1(64)
    B = b2s.BAIJ(ctx, 3, nbr, nbr, rp, ci, v)
    x64 = fp64_solution(B, 3 * nbr, b2s.PC_BSA_AMG, b2s.PCG)
    for name, kind, prec in (("bilu0_fp64", b2s.PC_BILU0, b2s.FP64), ("bilu0_fp32", b2s.PC_BILU0, b2s.FP32),
                             ("bsa_amg_fp64", b2s.PC_BSA_AMG, b2s.FP64), ("bsa_amg_fp32", b2s.PC_BSA_AMG, b2s.FP32)):
        emit(c, f"cg+{name}", gpu(B, 3 * nbr, kind, b2s.PCG, 1e-8, 5000, reps=1, pco={"precision": prec}, x64=x64),
             "not run: the reference's block matrix has GMRES only")
    # the reference's block solver: GMRES(30) with block ILU(0)
    r = None
    if ref is not None:
        Br = ref.blk(3, nbr, nbr, rp, ci, v)
        t0 = time.perf_counter()
        _, it = ref.blk_gmres(Br, b2s.uniform(7, 3 * nbr), "blockilu", 1e-8, 1000, 30)
        r = {"ms": round((time.perf_counter() - t0) * 1e3, 1), "it": it, "cores": os.cpu_count()}
    emit(c, "gmres30+bilu0_fp64", gpu(B, 3 * nbr, b2s.PC_BILU0, b2s.GMRES, 1e-8, 1000, reps=1, so={"restart": 30},
                                      x64=x64), r)
    del B
    ctx.close()
    return 0


# ---------------------------------------------------------------- reference arm

def arm_config(args, world):
    """The workload's `config` object, the same for both arms."""
    return {"workload": "grf_diffusion_512 pcg rtol1e-8", "method": args.method, "grid": N_GRID, "corr": CORR,
            "parallelism": f"replicas x{world}", "l2": "flushed (512 MB write) before every step"}


def run_reference(args):
    """The reference's own SMatrix::pcg(A, b, "ic") (oracle/_ref/libref.so,
    compiled from its sources) on all host cores, on the systems the GPU arm
    solves.  The systems come from oracle/_ref/libgen.so (the library's
    generators built on their own), so this process maps only the reference
    and the generators, never the product library."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    try:
        ref = oracle.Ref()
        gen = oracle.Gen()
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference library not built: {e}"}))
        return 0
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    times, its = [], []
    for k in range(args.warmup + args.steps):
        seed = 2000 + k
        n, rp, ci, v = gen.grf_diffusion(N_GRID, seed, corr=CORR)
        b = gen.uniform(seed, n)
        A = ref.csr(n, n, rp, ci, v)
        t0 = time.perf_counter()
        x, it = ref.solve(A, 0, "ic", b, TOL, MAXIT)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt * 1e3)
            its.append(it)
    ms = float(np.mean(times))
    line = {"metric": METRIC, "value": ms, "unit": "ms",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded GRF diffusion, held-out seeds 2000+)", "impl": "reference",
            "config": arm_config(args, world),
            "reference_solver": {"call": "SMatrix::pcg(A, b, \"ic\", 1e-8, 20000)",
                                 "seeds": [2000 + args.warmup, 2000 + args.warmup + args.steps - 1]},
            "iterations_mean": float(np.mean(its)),
            "cpu_baseline": {"value": ms, "unit": "ms", "cores": cores, "kind": "reference",
                             "sample": f"{args.steps} full solves (one system each)"},
            "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- GPU arm

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b2s", choices=["b2s", "reference"])
    ap.add_argument("--method", default="learned_ic0_j6",
                    choices=["learned_ic0_j6", "learned_ic0_j8", "learned_ic0", "fp32_ic0_j6", "fp32_ic0_j8",
                             "fp32_ic0", "fp64_ic0", "learned_ic0_j6_strips", "sa_amg"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kernel", default=None, choices=sorted(KERNELS),
                    help="run one hot kernel only (for profilers), not the benchmark")
    ap.add_argument("--suite", action="store_true",
                    help="time the other configurations (C1-C4), one JSON line each; not the benchmark")
    ap.add_argument("--no-ref", action="store_true", help="--suite without the reference's CPU timings")
    args = ap.parse_args()
    if args.suite:
        return run_suite(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.kernel:
        return run_kernel(args)

    import torch
    rank, world, local = env_rank()
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    b2s = load_b2s()
    ctx = b2s.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    dev = torch.device("cuda", local)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    seeds = replica_seeds(rank, args.warmup + args.steps)
    systems = [make_system(b2s, s) for s in seeds]

    # method -> (preconditioner, precision, triangular-solve schedule, sweeps, factorisation sweeps)
    kinds = {"learned_ic0_j6": (b2s.PC_LEARNED_IC0, b2s.FP32, b2s.TRSV_JACOBI, 6, 5),
             "learned_ic0_j8": (b2s.PC_LEARNED_IC0, b2s.FP32, b2s.TRSV_JACOBI, 8, 5),
             "learned_ic0": (b2s.PC_LEARNED_IC0, b2s.FP32, b2s.TRSV_AUTO, 0, 0),
             "fp32_ic0_j6": (b2s.PC_IC0, b2s.FP32, b2s.TRSV_JACOBI, 6, 5),
             "fp32_ic0_j8": (b2s.PC_IC0, b2s.FP32, b2s.TRSV_JACOBI, 8, 5),
             "fp32_ic0": (b2s.PC_IC0, b2s.FP32, b2s.TRSV_AUTO, 0, 0),
             "fp64_ic0": (b2s.PC_IC0, b2s.FP64, b2s.TRSV_AUTO, 0, 0),
             "learned_ic0_j6_strips": (b2s.PC_LEARNED_IC0, b2s.FP32, b2s.TRSV_JACOBI, 6, 5),
             "sa_amg": (b2s.PC_SA_AMG, b2s.FP64, b2s.TRSV_AUTO, 0, 0)}
    # the persistent PCG kernel: 2-D tiles when they can be planned (default), or row strips
    persist = {"learned_ic0_j6_strips": b2s.PERSIST_STRIPS}

    def make_pc(A, method):
        kind, prec, trsv, sweeps, fsweeps = kinds[method]
        return b2s.Precond(ctx, A, kind, precision=prec, trsv=trsv, trsv_sweeps=sweeps, factor_sweeps=fsweeps)

    x64_cache = {}

    def fp64_solution(k):
        """The FP64 solution of system k to rtol 1e-12 (FP64 SA-AMG PCG), the
        yardstick of every method's error."""
        if k not in x64_cache:
            n, rp, ci, v, b = systems[k]
            A = b2s.CSR(ctx, n, n, rp, ci, v)
            M = b2s.Precond(ctx, A, b2s.PC_SA_AMG)
            x, st = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-12, maxit=MAXIT)
            assert st["relres_true"] < 1e-11, st
            x64_cache[k] = x
        return x64_cache[k]

    def timed_solve(n, rp, ci, v, b, method):
        """Device-resident inputs; returns (ms, stats, launches, x on the host)."""
        A = b2s.CSR(ctx, n, n, rp, ci, v)
        bt = torch.from_numpy(b).to(dev)
        xt = torch.zeros(n, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0, em, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        l0 = ctx.kernel_launches
        e0.record(stream)
        M = make_pc(A, method)
        em.record(stream)
        st = b2s.solve_device(ctx, A, bt.data_ptr(), xt.data_ptr(), b2s.PCG, M, tol=TOL, maxit=MAXIT,
                              persistent=persist.get(method, b2s.PERSIST_AUTO))
        e1.record(stream)
        e1.synchronize()
        launches = ctx.kernel_launches - l0
        st["setup_ms_event"] = e0.elapsed_time(em)
        st["iter_ms_event"] = em.elapsed_time(e1)
        return e0.elapsed_time(e1), st, launches, xt.cpu().numpy()

    timed_idx = list(range(args.warmup, args.warmup + args.steps))

    def run(method, warm_idx):
        """Warm-up solves on warm_idx, then one timed solve per timed system."""
        for k in warm_idx:
            timed_solve(*systems[k], method)
        ms, its, rel, launches, split, fb, errs = [], [], [], 0, [], 0, []
        for k in timed_idx:
            t, st, nl, x = timed_solve(*systems[k], method)
            ms.append(t)
            its.append(st["iterations"])
            rel.append(st["relres_true"])
            split.append((st["setup_ms_event"], st["iter_ms_event"]))
            launches += nl
            fb += st["fallbacks"]
            errs.append((k, x))
        run.split = split
        run.fallbacks = fb
        run.errors = errs
        return ms, its, rel, launches

    def error_summary(errs):
        """||x - x_FP64|| / ||x_FP64|| over the timed systems (computed after timing)."""
        e = [float(np.linalg.norm(x - fp64_solution(k)) / np.linalg.norm(fp64_solution(k))) for k, x in errs]
        return {"max": max(e), "mean": float(np.mean(e)),
                "against": "FP64 SA-AMG PCG to rtol 1e-12 on the same system"}

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        head_ms, head_its, head_rel, launches = run(args.method, range(args.warmup))
    head_split = run.split
    head_fallbacks = run.fallbacks
    head_err = error_summary(run.errors)
    torch.cuda.synchronize()
    clocks = clk.summary()
    base_ms, base_its, base_rel, _ = run("fp64_ic0", range(min(1, args.warmup))) if args.method != "fp64_ic0" else (
        head_ms, head_its, head_rel, 0)
    base_split = run.split
    base_err = error_summary(run.errors) if args.method != "fp64_ic0" else head_err
    # the other methods on the same systems (context for the headline: what
    # the learned values and the sweep solves each contribute)
    variants = {}
    for m in kinds:
        if m in (args.method, "fp64_ic0"):
            continue
        v_ms, v_its, v_rel, _ = run(m, range(min(1, args.warmup)))
        variants[m] = {"ms": float(np.mean(v_ms)), "iterations_mean": float(np.mean(v_its)),
                       "relres_true_max": float(np.max(v_rel)), "fallbacks": int(run.fallbacks),
                       "setup_ms_mean": float(np.mean([a for a, _ in run.split])),
                       "error_vs_fp64": error_summary(run.errors),
                       "speedup_vs_fp64_ic0": float(np.mean(base_ms)) / float(np.mean(v_ms))}

    # e2e: host CSR + host b -> device, preconditioner, solve, x -> host (public C ABI, host pointers).
    # The inputs sit in pinned host memory, filled before the timed region.
    def pinned(a):
        t = torch.empty(a.shape, dtype={np.uint32: torch.int32, np.float64: torch.float64}[a.dtype.type],
                        pin_memory=True)
        h = t.numpy().view(a.dtype)
        h[...] = a
        return h, t

    e2e_ms, h2d, d2h = [], 0, 0
    kind, prec, trsv, sweeps, _ = kinds[args.method]
    for k in range(args.steps):
        n, rp, ci, v, b = systems[args.warmup + k]
        held = [pinned(a) for a in (rp, ci, v, b)]
        rp, ci, v, b = (h for h, _ in held)
        torch.cuda.synchronize()
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        A = b2s.CSR(ctx, n, n, rp, ci, v)
        M = make_pc(A, args.method)
        x, st = b2s.solve(ctx, A, b, b2s.PCG, M, tol=TOL, maxit=MAXIT)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        h2d = rp.nbytes + ci.nbytes + v.nbytes + b.nbytes
        d2h = x.nbytes
        del A, M, held

    # roofline of the dominant kernel: one triangle of the preconditioner
    # apply (forward L, backward L^T).  Sweep schedule (k_trsv_band): per row
    # W packed strict entries (u16 offset + FP32 value), the FP32 reciprocal,
    # the rhs (FP64 forward / FP32 backward) and the FP32 result, each read or
    # written once (the FP64 copy of the backward result is not counted).
    # Exact schedule (k_trsv_chunk): factor values + column indices + row
    # pointers + rhs + solution + diagonal.
    n, rp, ci, v, b = systems[args.warmup]
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    M = make_pc(A, args.method)
    r = torch.from_numpy(b).to(dev)
    z = torch.empty_like(r)
    nnz_l = (len(v) + n) // 2
    vb = 4 if prec == b2s.FP32 else 8
    if trsv == b2s.TRSV_JACOBI:
        tri_bytes = n * (2 * 6 + 4 + 6 + 4)
        tri_kernel = f"k_trsv_band (Jacobi-sweep triangle, {sweeps} sweeps in one launch)"
        tri_note = ("one launch per triangle; the halo rows (k*B = 4096 per 1,792-row tile) are re-read and "
                    "recomputed by each tile, so the kernel moves about 3.3x the algorithmic bytes, from L2")
    else:
        tri_bytes = nnz_l * (vb + 4) + 4 * (n + 1) + 3 * vb * n
        tri_kernel = "k_trsv_chunk (IC(0) triangular solve, one triangle per launch)"
        tri_note = "latency-bound: a 1023-level dependency chain per triangle on the 512^2 grid"
    for _ in range(3):
        b2s.lib().b2s_pc_apply_device(ctx.h, M.h, b2s.C.c_void_p(r.data_ptr()), b2s.C.c_void_p(z.data_ptr()))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 50
    e0.record(stream)
    for _ in range(reps):
        b2s.lib().b2s_pc_apply_device(ctx.h, M.h, b2s.C.c_void_p(r.data_ptr()), b2s.C.c_void_p(z.data_ptr()))
    e1.record(stream)
    e1.synchronize()
    tri_ms = e0.elapsed_time(e1) / reps / 2
    pk, pk_kind = peaks()
    achieved = tri_bytes / (tri_ms * 1e-3) / 1e9
    trsv_apply = {"kernel": tri_kernel, "bound": "hbm",
                  "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                  "peak_kind": pk_kind, "traffic": None, "bytes_per_launch": tri_bytes, "ms_per_launch": tri_ms,
                  "note": tri_note}
    roofline = trsv_apply
    if trsv == b2s.TRSV_JACOBI and prec == b2s.FP32:
        # The timed solves run as one persistent cooperative launch each
        # (k_pcg_band).  Algorithmic bytes per PCG iteration, canonical fused
        # schedule: SpMV (12 nnz + 4(n+1) + 8n x + 8n y) + 16n (p, Ap)
        # + 64n (reads x, p, r, Ap, M-data; writes x, r, z) + 24n (p update)
        # + both sweep-applied triangles; times the mean iteration count.
        spmv_bytes = 12 * len(v) + 4 * (n + 1) + 16 * n
        it_bytes = spmv_bytes + 16 * n + 64 * n + 24 * n + 2 * tri_bytes
        launch_bytes = it_bytes * float(np.mean(head_its))
        solve_ms = float(np.mean([b for _, b in head_split]))
        achieved = launch_bytes / (solve_ms * 1e-3) / 1e9
        tiles = M.sizes("pcg.tiles")[0] if persist.get(args.method, b2s.PERSIST_AUTO) == b2s.PERSIST_AUTO else 0
        kname = "k_pcg_tile" if tiles else "k_pcg_band"
        kdesc = (f"k_pcg_tile (persistent cooperative PCG over {tiles} 2-D tiles, the whole solve in one launch)"
                 if tiles else "k_pcg_band (persistent cooperative PCG over row strips, the whole solve in one launch)")
        roofline = {"kernel": kdesc,
                    "bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                    "frac": achieved / pk["hbm_gbs"], "peak_kind": pk_kind, "traffic": PCG_DRAM_BYTES[kname],
                    "bytes_per_launch": launch_bytes, "bytes_per_iteration": it_bytes, "ms_per_launch": solve_ms,
                    "note": "duration = the event-timed solve phase of the timed steps (the launch plus the final "
                            "FP64 residual check); the operator, factors and vectors stay in L2, so DRAM traffic "
                            "(ncu, one launch) is a small fraction of the algorithmic bytes and the kernel is bound "
                            "by its per-iteration synchronisation, not by HBM"}

    # the learned network's tcgen05 dense layer (64 -> 128) on this grid's node
    # states: X read once, Y written once
    nd = N_GRID * N_GRID
    gx = torch.Generator(device=dev).manual_seed(5)
    xd = torch.randn(nd, 64, generator=gx, device=dev, dtype=torch.float32)
    wd = (0.1 * torch.randn(128, 64, generator=gx, device=dev)).to(torch.bfloat16)
    yd = torch.empty(nd, 128, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    dense = lambda: ctx.check(b2s.lib().b2s_dense_bf16_device(ctx.h, nd, 64, 128, b2s.C.c_void_p(xd.data_ptr()),
                                                             b2s.C.c_void_p(wd.data_ptr()), None,
                                                             b2s.C.c_void_p(yd.data_ptr())), "dense_bf16")
    for _ in range(3):
        dense()
    e0.record(stream)
    for _ in range(20):
        dense()
    e1.record(stream)
    e1.synchronize()
    dense_ms = e0.elapsed_time(e1) / 20
    dense_bytes = nd * (64 + 128) * 4 + 128 * 64 * 2
    dense_gbs = dense_bytes / (dense_ms * 1e-3) / 1e9
    dense_layer = {"kernel": "k_linear_tc<64,128> (tcgen05.mma kind::f16, BF16 x BF16 -> FP32 in TMEM)",
                   "workload": f"{nd} node states x 64 -> 128", "ms": dense_ms, "achieved": dense_gbs,
                   "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": dense_gbs / pk["hbm_gbs"],
                   "bytes_per_launch": dense_bytes, "tflops": 2.0 * nd * 64 * 128 / (dense_ms * 1e-3) / 1e12}
    del xd, yd

    # C2 (3-D Poisson 128^3) CSR SpMV against the HBM roofline (inputs > L2)
    n3, rp3, ci3, v3 = b2s.gen_poisson3d(128)
    A3 = b2s.CSR(ctx, n3, n3, rp3, ci3, v3)
    x3 = torch.rand(n3, dtype=torch.float64, device=dev)
    y3 = torch.empty_like(x3)
    for _ in range(3):
        A3.spmv_device(x3.data_ptr(), y3.data_ptr())
    e0.record(stream)
    for _ in range(20):
        A3.spmv_device(x3.data_ptr(), y3.data_ptr())
    e1.record(stream)
    e1.synchronize()
    spmv_ms = e0.elapsed_time(e1) / 20
    spmv_bytes = 12 * len(v3) + 4 * (n3 + 1) + 16 * n3
    spmv_gbs = spmv_bytes / (spmv_ms * 1e-3) / 1e9
    spmv = {"kernel": "k_spmv_warp", "workload": "poisson3d_128 (n=2097152, nnz=14581760)",
            "ms": spmv_ms, "achieved": spmv_gbs, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": spmv_gbs / pk["hbm_gbs"], "bytes_per_launch": spmv_bytes}

    value = max_over_ranks(float(np.mean(head_ms)), dev)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle
            ref = oracle.Ref()
            cores = os.cpu_count() or 1
            ref.set_threads(cores)
            n, rp, ci, v, b = systems[args.warmup]
            Ar = ref.csr(n, n, rp, ci, v)
            t0 = time.perf_counter()
            xr, itr = ref.solve(Ar, 0, "ic", b, TOL, MAXIT)
            cms = (time.perf_counter() - t0) * 1e3
            cpu = {"value": cms, "unit": "ms", "cores": cores, "kind": "reference", "iterations": itr,
                   "sample": f"one full SMatrix::pcg(A,b,\"ic\") solve of seed {seeds[args.warmup]}"}
        except Exception as e:
            cpu = {"value": None, "unit": "ms", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": value, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 outer / f32 preconditioner" if prec == b2s.FP32 else "f64",
            "method": {"learned_ic0_j6": "learned IC(0) values (tcgen05 network) on a 5-sweep fixed-point IC(0) "
                                         "factor, FP32, 6 Jacobi sweeps per triangle, the whole PCG loop in one "
                                         "persistent launch, FP64 PCG and true residual",
                       "learned_ic0_j8": "the same with 8 Jacobi sweeps per triangle",
                       "learned_ic0": "learned IC(0) values on the exact factor, FP32, exact chunk-scheduled "
                                      "triangular solves",
                       "fp32_ic0_j6": "plain IC(0) (5-sweep fixed-point factor), FP32, 6 Jacobi sweeps per triangle",
                       "fp32_ic0_j8": "plain IC(0) (5-sweep fixed-point factor), FP32, 8 Jacobi sweeps per triangle",
                       "fp32_ic0": "plain IC(0), FP32 factor, exact triangular solves",
                       "fp64_ic0": "plain IC(0), FP64, exact triangular solves",
                       "learned_ic0_j6_strips": "learned_ic0_j6 with the whole PCG loop in the row-strip "
                                                "persistent kernel (k_pcg_band) instead of the 2-D tile one",
                       "sa_amg": "smoothed-aggregation AMG V-cycle (FP64)"}[args.method],
            "data": "synthetic (seeded GRF diffusion, held-out seeds 2000+)",
            "config": arm_config(args, world),
            "iterations_mean": float(np.mean(head_its)), "relres_true_max": float(np.max(head_rel)),
            "fallbacks": int(head_fallbacks),
            "error_vs_fp64": head_err,
            "setup_ms_mean": float(np.mean([a for a, _ in head_split])),
            "iter_ms_mean": float(np.mean([b for _, b in head_split])),
            "fp64_ic0_pcg": {"ms": float(np.mean(base_ms)), "iterations_mean": float(np.mean(base_its)),
                             "relres_true_max": float(np.max(base_rel)),
                             "error_vs_fp64": base_err,
                             "setup_ms_mean": float(np.mean([a for a, _ in base_split])),
                             "iter_ms_mean": float(np.mean([b for _, b in base_split]))},
            "speedup_vs_fp64_ic0": float(np.mean(base_ms)) / value,
            "variants": variants,
            "e2e": {"value": float(np.mean(e2e_ms)), "unit": "ms", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "trsv_apply": trsv_apply,
            "spmv_c2": spmv,
            "dense_layer": dense_layer,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

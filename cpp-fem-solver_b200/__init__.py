"""b2s -- B200-native sparse iterative solvers (Python host mirror).

This package drives ``libb2s.so`` (built in this directory from ``csrc/`` by
``make -C cpp-fem-solver_b200``) through its C ABI (``include/b2s.h``).  It
mirrors the solver surface of xuyinshen/cpp-FEM-solver's ``sparse::SMatrix``
(ode-solver/include/math/array.hpp:266-373) and ``block::BlockMatrix``
(ode-solver/include/math/blockMatrix.hpp:139-452): same names, same argument
meaning, same returned ``(x, it)`` pairs with the reference's iteration-count
conventions, and the same exception split -- ``ValueError`` where the
reference throws ``std::invalid_argument``, ``RuntimeError`` where it throws
``std::runtime_error``.

There is no CPU path: every compute call runs on the GPU, and importing works
without one, but creating a :class:`Context` fails loudly (``B2SError`` with
``B2S_NO_DEVICE``) when no B200 is present or the library is not built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libb2s.so")
REPO = os.path.dirname(HERE)

# ------------------------------------------------------------------ status

STATUS = {
    0: "B2S_OK", 1: "B2S_INVALID_ARG", 2: "B2S_SHAPE", 3: "B2S_NOT_SPD", 4: "B2S_BREAKDOWN",
    5: "B2S_ZERO_PIVOT", 6: "B2S_MISSING_DIAG", 7: "B2S_SINGULAR_BLOCK", 8: "B2S_DIVERGED",
    9: "B2S_TIMEOUT", 10: "B2S_CUDA_ERROR", 11: "B2S_NO_DEVICE", 12: "B2S_OUT_OF_MEMORY", 13: "B2S_UNSUPPORTED",
}
OK, INVALID_ARG, SHAPE, NOT_SPD, BREAKDOWN, ZERO_PIVOT, MISSING_DIAG, SINGULAR_BLOCK, DIVERGED, TIMEOUT = range(10)
CUDA_ERROR, NO_DEVICE, OUT_OF_MEMORY, UNSUPPORTED = 10, 11, 12, 13

# preconditioner kinds / methods / options (b2s.h)
PC_NONE, PC_DIAG, PC_IC0, PC_ILU0, PC_SSOR, PC_SA_AMG, PC_LEARNED_IC0, PC_BJACOBI, PC_BILU0, PC_BSA_AMG = range(10)
PC_SCHUR, PC_SCALED = 10, 11
PCG, BICGSTAB, GMRES, FGMRES, BLOCK_GMRES, STATIONARY = range(6)
FP64, FP32, BF16 = range(3)
TRSV_AUTO, TRSV_LEVEL, TRSV_SYNCFREE, TRSV_CHUNK, TRSV_JACOBI = range(5)
ORTH_MGS, ORTH_CGS2 = range(2)

PC_NAMES = {"none": PC_NONE, "diag": PC_DIAG, "ic0": PC_IC0, "ilu0": PC_ILU0, "ssor": PC_SSOR,
            "sa_amg": PC_SA_AMG, "amg": PC_SA_AMG, "learned_ic0": PC_LEARNED_IC0, "bjacobi": PC_BJACOBI,
            "bilu0": PC_BILU0, "bsa_amg": PC_BSA_AMG}


class B2SError(Exception):
    """A failed b2s call; ``status`` is the b2s_status code."""

    def __init__(self, status: int, msg: str):
        self.status = status
        self.name = STATUS.get(status, str(status))
        super().__init__(f"{self.name}: {msg}")


class B2SInvalidArgument(B2SError, ValueError):
    """std::invalid_argument in the reference."""


class B2SRuntimeError(B2SError, RuntimeError):
    """std::runtime_error in the reference (numerical breakdown)."""


def _raise(status: int, msg: str):
    if status in (INVALID_ARG, SHAPE):
        raise B2SInvalidArgument(status, msg)
    if status in (NOT_SPD, BREAKDOWN, ZERO_PIVOT, MISSING_DIAG, SINGULAR_BLOCK, DIVERGED, TIMEOUT):
        raise B2SRuntimeError(status, msg)
    raise B2SError(status, msg)


# ------------------------------------------------------------------ library

class PcOpts(C.Structure):
    _fields_ = [("omega", C.c_double), ("precision", C.c_int), ("trsv", C.c_int), ("amg_ref_coarse", C.c_int),
                ("amg_max_levels", C.c_int), ("amg_coarse_max", C.c_int), ("amg_aggregation", C.c_int),
                ("learned_weights", C.c_char_p), ("trsv_sweeps", C.c_int), ("trsv_segment", C.c_int),
                ("factor_sweeps", C.c_int)]


class SolveOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("maxit", C.c_int), ("restart", C.c_int), ("orth", C.c_int),
                ("ir_steps", C.c_int), ("ir_inner_tol", C.c_double), ("check_every", C.c_int),
                ("use_graphs", C.c_int), ("stall_window", C.c_int), ("persistent", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("it", C.c_int), ("iterations", C.c_int), ("spmvs", C.c_int), ("pc_applies", C.c_int),
                ("restarts", C.c_int), ("status", C.c_int), ("relres", C.c_double), ("relres_true", C.c_double),
                ("setup_ms", C.c_double), ("solve_ms", C.c_double), ("fallbacks", C.c_int),
                ("stalled_at", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_lib = None

# every symbol declared in include/b2s.h
EXPORTS = [
    "b2s_ctx_create", "b2s_ctx_destroy", "b2s_last_error", "b2s_status_name", "b2s_ctx_stream",
    "b2s_ctx_synchronize", "b2s_ctx_kernel_launches", "b2s_csr_create", "b2s_csr_destroy", "b2s_csr_info",
    "b2s_baij_create", "b2s_baij_destroy", "b2s_baij_info", "b2s_spmv", "b2s_spmv_device", "b2s_dot",
    "b2s_dot_device", "b2s_baij_matvec", "b2s_baij_matvec_device", "b2s_pc_opts_default", "b2s_pc_create",
    "b2s_pc_create_baij", "b2s_pc_create_host", "b2s_pc_destroy", "b2s_pc_apply", "b2s_pc_apply_device",
    "b2s_pc_export", "b2s_pc_kind_from_name", "b2s_solve_opts_default", "b2s_solve", "b2s_solve_device",
    "b2s_solve_baij", "b2s_solve_baij_device", "b2s_gen_poisson2d", "b2s_gen_poisson3d", "b2s_gen_convdiff3d",
    "b2s_gen_elasticity_q1", "b2s_gen_grf_diffusion", "b2s_gen_uniform", "b2s_learner_create",
    "b2s_learner_destroy", "b2s_learner_load", "b2s_learner_save", "b2s_learner_params", "b2s_learner_step",
    "b2s_pc_create_learned", "b2s_dot_noalloc", "b2s_dense_bf16_device",
    "b2s_learner_set_loss", "b2s_sor", "b2s_sor_device", "b2s_csr_matmul", "b2s_csr_transpose", "b2s_csr_export",
    "b2s_ctx_set_wait_limits", "b2s_baij_set_halo", "b2s_baij_halo_info", "b2s_baij_halo_pack_device",
    "b2s_baij_dist_matvec_owned_device", "b2s_baij_dist_matvec_ghost_device", "b2s_pc_create_schur",
    "b2s_pc_create_scaled", "b2s_learner_set_sweeps",
]


def build(quiet: bool = True) -> None:
    """Compile libb2s.so for sm_100a in place (nvcc cross-compiles without a GPU)."""
    subprocess.run(["make", "-C", HERE, "-j8"], check=True, stdout=subprocess.DEVNULL if quiet else None)


def lib():
    """The loaded libb2s.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise B2SError(UNSUPPORTED, f"{LIB_PATH} is not built; run `make -C {HERE}`")
    L = C.CDLL(LIB_PATH)
    vp, u32, u64, f64, i32, cp = C.c_void_p, C.c_uint32, C.c_uint64, C.c_double, C.c_int, C.c_char_p
    pp = C.POINTER(C.c_void_p)
    u32ptr = C.POINTER(C.c_uint32)

    def f(name, res, *args):
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = list(args)

    f("b2s_ctx_create", i32, i32, pp)
    f("b2s_ctx_destroy", i32, vp)
    f("b2s_last_error", cp, vp)
    f("b2s_status_name", cp, i32)
    f("b2s_ctx_stream", vp, vp)
    f("b2s_ctx_synchronize", i32, vp)
    f("b2s_ctx_kernel_launches", u64, vp)
    f("b2s_csr_create", i32, vp, u32, u32, _u32p, _u32p, _f64p, pp)
    f("b2s_csr_destroy", i32, vp)
    f("b2s_csr_info", i32, vp, u32ptr, u32ptr, u32ptr)
    f("b2s_baij_create", i32, vp, i32, u32, u32, _u32p, _u32p, _f64p, pp)
    f("b2s_baij_destroy", i32, vp)
    f("b2s_baij_info", i32, vp, C.POINTER(C.c_int), u32ptr, u32ptr, u32ptr)
    f("b2s_spmv", i32, vp, vp, _f64p, _f64p)
    f("b2s_spmv_device", i32, vp, vp, vp, vp)
    f("b2s_dot", i32, vp, u64, _f64p, _f64p, C.POINTER(C.c_double))
    f("b2s_dot_device", i32, vp, u64, vp, vp, C.POINTER(C.c_double))
    f("b2s_baij_matvec", i32, vp, vp, _f64p, _f64p)
    f("b2s_baij_matvec_device", i32, vp, vp, vp, vp)
    f("b2s_pc_opts_default", None, C.POINTER(PcOpts))
    f("b2s_pc_create", i32, vp, vp, i32, C.POINTER(PcOpts), pp)
    f("b2s_pc_create_baij", i32, vp, vp, i32, C.POINTER(PcOpts), pp)
    f("b2s_pc_create_host", i32, vp, u64, vp, vp, pp)
    f("b2s_pc_destroy", i32, vp)
    f("b2s_pc_apply", i32, vp, vp, _f64p, _f64p)
    f("b2s_pc_apply_device", i32, vp, vp, vp, vp)
    f("b2s_pc_export", i32, vp, vp, cp, C.POINTER(C.c_uint64), vp, vp, vp)
    f("b2s_pc_kind_from_name", i32, i32, cp, C.POINTER(C.c_int))
    f("b2s_solve_opts_default", None, C.POINTER(SolveOpts))
    f("b2s_solve", i32, vp, vp, vp, i32, C.POINTER(SolveOpts), _f64p, _f64p, C.POINTER(Stats))
    f("b2s_solve_device", i32, vp, vp, vp, i32, C.POINTER(SolveOpts), vp, vp, C.POINTER(Stats))
    f("b2s_solve_baij", i32, vp, vp, vp, i32, C.POINTER(SolveOpts), _f64p, _f64p, C.POINTER(Stats))
    f("b2s_solve_baij_device", i32, vp, vp, vp, i32, C.POINTER(SolveOpts), vp, vp, C.POINTER(Stats))
    f("b2s_gen_poisson2d", i32, u32, u32ptr, u32ptr, vp, vp, vp)
    f("b2s_gen_poisson3d", i32, u32, u32ptr, u32ptr, vp, vp, vp)
    f("b2s_gen_convdiff3d", i32, u32, f64, f64, f64, u32ptr, u32ptr, vp, vp, vp)
    f("b2s_gen_elasticity_q1", i32, u32, f64, f64, u32ptr, u32ptr, vp, vp, vp)
    f("b2s_gen_grf_diffusion", i32, u32, f64, f64, u64, u32ptr, u32ptr, vp, vp, vp, vp)
    f("b2s_gen_uniform", i32, u64, u64, _f64p)
    f("b2s_learner_create", i32, vp, u64, pp)
    f("b2s_learner_destroy", i32, vp)
    f("b2s_learner_load", i32, vp, cp)
    f("b2s_learner_save", i32, vp, cp)
    f("b2s_learner_params", i32, vp, vp, C.POINTER(C.c_uint64), i32)
    f("b2s_learner_step", i32, vp, vp, vp, i32, u64, vp, f64, i32, C.POINTER(C.c_double), vp)
    f("b2s_pc_create_learned", i32, vp, vp, vp, C.POINTER(PcOpts), pp)
    f("b2s_dot_noalloc", i32, vp, vp, u64, vp, vp)
    f("b2s_dense_bf16_device", i32, vp, u64, i32, i32, vp, vp, vp, vp)
    f("b2s_learner_set_loss", i32, vp, i32)
    f("b2s_sor", i32, vp, vp, i32, f64, f64, i32, _f64p, _f64p, C.POINTER(Stats))
    f("b2s_sor_device", i32, vp, vp, i32, f64, f64, i32, vp, vp, C.POINTER(Stats))
    f("b2s_csr_matmul", i32, vp, vp, vp, pp)
    f("b2s_csr_transpose", i32, vp, vp, pp)
    f("b2s_csr_export", i32, vp, vp, vp, vp, vp)
    f("b2s_ctx_set_wait_limits", i32, vp, u32, u32)
    i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    f("b2s_baij_set_halo", i32, vp, vp, i32, i32p, i32p, _u32p, i32, i32p, i32p, _u32p, u32)
    f("b2s_baij_halo_info", i32, vp, u32ptr, u32ptr, u32ptr)
    f("b2s_baij_halo_pack_device", i32, vp, vp, vp, vp)
    f("b2s_baij_dist_matvec_owned_device", i32, vp, vp, vp, vp)
    f("b2s_baij_dist_matvec_ghost_device", i32, vp, vp, vp, vp)
    f("b2s_pc_create_schur", i32, vp, u64, u64, vp, vp, vp, vp, pp)
    f("b2s_pc_create_scaled", i32, vp, vp, f64, pp)
    f("b2s_learner_set_sweeps", i32, vp, i32, i32)
    _lib = L
    return L


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ------------------------------------------------------------------ context

class Context:
    """One GPU, one CUDA stream (b2s_ctx)."""

    def __init__(self, device: int = 0):
        L = lib()
        h = C.c_void_p()
        st = L.b2s_ctx_create(device, C.byref(h))
        if st != OK:
            _raise(st, f"cannot create a b2s context on device {device}")
        self.h = h
        self.device = device

    def check(self, st: int, what: str = ""):
        if st != OK:
            msg = lib().b2s_last_error(self.h).decode(errors="replace")
            _raise(st, f"{what}: {msg}" if what else msg)

    @property
    def stream(self) -> int:
        return lib().b2s_ctx_stream(self.h)

    @property
    def kernel_launches(self) -> int:
        return lib().b2s_ctx_kernel_launches(self.h)

    def synchronize(self):
        self.check(lib().b2s_ctx_synchronize(self.h), "synchronize")

    def set_wait_limits(self, spin_polls: int = 0, sleep_polls: int = 0):
        """Bounds of the chunked triangular solves' device waits ((0, 0): defaults)."""
        self.check(lib().b2s_ctx_set_wait_limits(self.h, int(spin_polls), int(sleep_polls)), "set_wait_limits")

    def close(self):
        if getattr(self, "h", None):
            lib().b2s_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class CSR:
    """Device-resident CSR matrix (b2s_csr)."""

    def __init__(self, ctx: Context, n, m, rp, ci, v):
        self.ctx, self.n, self.m = ctx, int(n), int(m)
        self.rp, self.ci, self.v = _u32(rp), _u32(ci), _f64(v)
        h = C.c_void_p()
        ctx.check(lib().b2s_csr_create(ctx.h, self.n, self.m, self.rp, self.ci, self.v, C.byref(h)), "csr_create")
        self.h = h

    @property
    def nnz(self):
        return int(self.rp[-1])

    def spmv(self, x):
        y = np.zeros(self.n)
        self.ctx.check(lib().b2s_spmv(self.ctx.h, self.h, _f64(x), y), "spmv")
        return y

    def spmv_device(self, x_ptr: int, y_ptr: int):
        self.ctx.check(lib().b2s_spmv_device(self.ctx.h, self.h, C.c_void_p(x_ptr), C.c_void_p(y_ptr)), "spmv")

    @classmethod
    def _adopt(cls, ctx: Context, h) -> "CSR":
        """A handle made on the device (product, transpose), with its host arrays."""
        n, m, nnz = C.c_uint32(), C.c_uint32(), C.c_uint32()
        lib().b2s_csr_info(h, C.byref(n), C.byref(m), C.byref(nnz))
        out = cls.__new__(cls)
        out.ctx, out.n, out.m, out.h = ctx, n.value, m.value, h
        out.rp = np.zeros(n.value + 1, np.uint32)
        out.ci = np.zeros(nnz.value, np.uint32)
        out.v = np.zeros(nnz.value, np.float64)
        ctx.check(lib().b2s_csr_export(ctx.h, h, _ptr(out.rp), _ptr(out.ci), _ptr(out.v)), "csr_export")
        return out

    def transpose(self) -> "CSR":
        """A^T on the device (SMatrix::transpose)."""
        h = C.c_void_p()
        self.ctx.check(lib().b2s_csr_transpose(self.ctx.h, self.h, C.byref(h)), "csr_transpose")
        return CSR._adopt(self.ctx, h)

    def matmul(self, B: "CSR") -> "CSR":
        """A B on the device (SMatrix::operator*)."""
        h = C.c_void_p()
        self.ctx.check(lib().b2s_csr_matmul(self.ctx.h, self.h, B.h, C.byref(h)), "csr_matmul")
        return CSR._adopt(self.ctx, h)

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.ctx.h:
                lib().b2s_csr_destroy(self.h)
        except Exception:
            pass


class BAIJ:
    """Device-resident block-CSR matrix (b2s_baij)."""

    def __init__(self, ctx: Context, bs, nbr, nbc, rp, ci, v):
        self.ctx, self.bs, self.nbr, self.nbc = ctx, int(bs), int(nbr), int(nbc)
        self.rp, self.ci, self.v = _u32(rp), _u32(ci), _f64(v)
        h = C.c_void_p()
        ctx.check(lib().b2s_baij_create(ctx.h, self.bs, self.nbr, self.nbc, self.rp, self.ci, self.v, C.byref(h)),
                  "baij_create")
        self.h = h

    @property
    def n(self):
        return self.nbr * self.bs

    def matvec(self, x):
        y = np.zeros(self.nbr * self.bs)
        self.ctx.check(lib().b2s_baij_matvec(self.ctx.h, self.h, _f64(x), y), "baij_matvec")
        return y

    def set_halo(self, recv_procs, recv_cnts, recv_global, send_procs, send_cnts, send_local, owned_global_start):
        """BlockMatrix::set_halo: this handle holds one rank's block rows (global columns)."""
        i32 = lambda a: np.ascontiguousarray(a, np.int32)
        rp_, rc_, sp_, sc_ = i32(recv_procs), i32(recv_cnts), i32(send_procs), i32(send_cnts)
        self.ctx.check(lib().b2s_baij_set_halo(self.ctx.h, self.h, len(rp_), rp_, rc_, _u32(recv_global), len(sp_),
                                               sp_, sc_, _u32(send_local), int(owned_global_start)), "set_halo")

    def halo_info(self):
        """(n_owned, n_ghost, n_send) block rows of the halo set by set_halo."""
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self.ctx.check(lib().b2s_baij_halo_info(self.h, C.byref(a), C.byref(b), C.byref(c)), "halo_info")
        return a.value, b.value, c.value

    def halo_pack_device(self, x_ptr: int, buf_ptr: int):
        self.ctx.check(lib().b2s_baij_halo_pack_device(self.ctx.h, self.h, C.c_void_p(x_ptr), C.c_void_p(buf_ptr)),
                       "halo_pack")

    def dist_matvec_owned_device(self, xfull_ptr: int, y_ptr: int):
        self.ctx.check(lib().b2s_baij_dist_matvec_owned_device(self.ctx.h, self.h, C.c_void_p(xfull_ptr),
                                                                C.c_void_p(y_ptr)), "dist_matvec_owned")

    def dist_matvec_ghost_device(self, xfull_ptr: int, y_ptr: int):
        self.ctx.check(lib().b2s_baij_dist_matvec_ghost_device(self.ctx.h, self.h, C.c_void_p(xfull_ptr),
                                                                C.c_void_p(y_ptr)), "dist_matvec_ghost")

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.ctx.h:
                lib().b2s_baij_destroy(self.h)
        except Exception:
            pass


def pc_opts(omega=1.2, precision=FP64, trsv=TRSV_AUTO, amg_ref_coarse=0, amg_max_levels=0, amg_coarse_max=0,
            amg_aggregation=0, learned_weights=None, trsv_sweeps=0, trsv_segment=0, factor_sweeps=0) -> PcOpts:
    o = PcOpts()
    lib().b2s_pc_opts_default(C.byref(o))
    o.omega, o.precision, o.trsv, o.trsv_sweeps = omega, precision, trsv, trsv_sweeps
    o.trsv_segment, o.factor_sweeps = trsv_segment, factor_sweeps
    o.amg_ref_coarse, o.amg_max_levels, o.amg_coarse_max = amg_ref_coarse, amg_max_levels, amg_coarse_max
    o.amg_aggregation = amg_aggregation
    o.learned_weights = learned_weights.encode() if learned_weights else None
    return o


class Precond:
    """A device preconditioner (b2s_pc) built from a CSR or BAIJ matrix."""

    def __init__(self, ctx: Context, A, kind, **opts):
        if isinstance(kind, str):
            kind = PC_NAMES[kind]
        self.ctx, self.kind, self.n = ctx, kind, A.n
        o = pc_opts(**opts)
        h = C.c_void_p()
        fn = lib().b2s_pc_create_baij if isinstance(A, BAIJ) else lib().b2s_pc_create
        ctx.check(fn(ctx.h, A.h, kind, C.byref(o), C.byref(h)), "pc_create")
        self.h = h

    def apply(self, r):
        z = np.zeros(self.n)
        self.ctx.check(lib().b2s_pc_apply(self.ctx.h, self.h, _f64(r), z), "pc_apply")
        return z

    def sizes(self, what: str):
        """The three sizes b2s_pc_export reports for `what` (no arrays)."""
        sizes = (C.c_uint64 * 3)()
        self.ctx.check(lib().b2s_pc_export(self.ctx.h, self.h, what.encode(), sizes, None, None, None), "pc_export")
        return tuple(int(x) for x in sizes)

    def export(self, what: str):
        """(rp, ci, v) arrays of an internal factor (see b2s_pc_export)."""
        sizes = (C.c_uint64 * 3)()
        self.ctx.check(lib().b2s_pc_export(self.ctx.h, self.h, what.encode(), sizes, None, None, None), "pc_export")
        rp = np.zeros(sizes[0], np.uint32)
        ci = np.zeros(sizes[1], np.uint32)
        v = np.zeros(sizes[2], np.float64)
        self.ctx.check(lib().b2s_pc_export(self.ctx.h, self.h, what.encode(), sizes, _ptr(rp), _ptr(ci), _ptr(v)),
                       "pc_export")
        return rp, ci, v

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.ctx.h:
                lib().b2s_pc_destroy(self.h)
        except Exception:
            pass


class SchurPrecond(Precond):
    """make_schur_preconditioner (blockMatrix.hpp:637-685) on the device:
    A_pc for the velocity block, S_pc (None = identity) for the pressure
    block, B (n_pres x n_vel) and Bt (n_vel x n_pres) CSR handles."""

    def __init__(self, ctx: Context, n_vel: int, n_pres: int, B: "CSR", Bt: "CSR", A_pc, S_pc=None):
        self.ctx, self.kind, self.n = ctx, PC_SCHUR, int(n_vel) + int(n_pres)
        self._keep = (B, Bt, A_pc, S_pc)  # the parts must outlive the composition
        h = C.c_void_p()
        ctx.check(lib().b2s_pc_create_schur(ctx.h, int(n_vel), int(n_pres), B.h, Bt.h, A_pc.h,
                                            S_pc.h if S_pc is not None else None, C.byref(h)), "pc_create_schur")
        self.h = h


class ScaledPrecond(Precond):
    """z = alpha * M^-1 r for a device preconditioner M."""

    def __init__(self, ctx: Context, inner, alpha: float):
        self.ctx, self.kind, self.n = ctx, PC_SCALED, inner.n
        self._keep = inner
        h = C.c_void_p()
        ctx.check(lib().b2s_pc_create_scaled(ctx.h, inner.h, float(alpha), C.byref(h)), "pc_create_scaled")
        self.h = h


class HostPrecond:
    """Preconditioner that calls a Python function z = f(r) on the host."""

    def __init__(self, ctx: Context, n: int, fn):
        self.ctx, self.n, self._fn = ctx, n, fn
        CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_uint64)

        def tramp(user, r, z, nn):
            try:
                rv = np.ctypeslib.as_array(r, shape=(nn,))
                zv = np.ctypeslib.as_array(z, shape=(nn,))
                zv[:] = fn(rv.copy())
                return 0
            except Exception:
                return 1

        self._cb = CB(tramp)
        h = C.c_void_p()
        ctx.check(lib().b2s_pc_create_host(ctx.h, n, C.cast(self._cb, C.c_void_p), None, C.byref(h)), "pc_create_host")
        self.h = h

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.ctx.h:
                lib().b2s_pc_destroy(self.h)
        except Exception:
            pass


WEIGHTS = os.path.join(HERE, "weights", "learned_ic0.bin")
LOSS_PRECOND, LOSS_FACTOR, LOSS_SWEEPS = 0, 1, 2


class Learner:
    """The learned-IC(0) message-passing network (b2s_learner)."""

    def __init__(self, ctx: Context, seed: int = 0, weights: str | None = None, loss: int = LOSS_PRECOND):
        self.ctx = ctx
        h = C.c_void_p()
        ctx.check(lib().b2s_learner_create(ctx.h, seed, C.byref(h)), "learner_create")
        self.h = h
        self.set_loss(loss)
        if weights:
            self.load(weights)

    def set_loss(self, kind: int):
        self.ctx.check(lib().b2s_learner_set_loss(self.h, int(kind)), "learner_set_loss")

    def set_sweeps(self, trsv_sweeps: int = 6, factor_sweeps: int = 0):
        """LOSS_SWEEPS' sweeps per triangle; the base factor (0: exact IC(0), k: k fixed-point sweeps)."""
        self.ctx.check(lib().b2s_learner_set_sweeps(self.h, int(trsv_sweeps), int(factor_sweeps)),
                       "learner_set_sweeps")

    @property
    def nparams(self) -> int:
        c = C.c_uint64()
        lib().b2s_learner_params(self.h, None, C.byref(c), 0)
        return c.value

    def params(self) -> np.ndarray:
        c = C.c_uint64(self.nparams)
        out = np.zeros(c.value, np.float32)
        self.ctx.check(lib().b2s_learner_params(self.h, _ptr(out), C.byref(c), 0), "learner_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        c = C.c_uint64(len(p))
        self.ctx.check(lib().b2s_learner_params(self.h, _ptr(p), C.byref(c), 1), "learner_params")

    def load(self, path: str):
        self.ctx.check(lib().b2s_learner_load(self.h, path.encode()), "learner_load")

    def save(self, path: str):
        self.ctx.check(lib().b2s_learner_save(self.h, path.encode()), "learner_save")

    def step(self, A: CSR, nprobes=4, seed=0, probes=None, lr=1e-3, update=True, want_grad=False):
        loss = C.c_double()
        grad = np.zeros(self.nparams, np.float32) if want_grad else None
        pr = None if probes is None else np.ascontiguousarray(probes, np.float64)
        self.ctx.check(lib().b2s_learner_step(self.ctx.h, self.h, A.h, int(nprobes), int(seed), _ptr(pr), float(lr),
                                              1 if update else 0, C.byref(loss), _ptr(grad)), "learner_step")
        return (loss.value, grad) if want_grad else loss.value

    def precond(self, A: CSR, **opts) -> "Precond":
        o = pc_opts(**opts)
        P = Precond.__new__(Precond)
        P.ctx, P.kind, P.n = self.ctx, PC_LEARNED_IC0, A.n
        h = C.c_void_p()
        self.ctx.check(lib().b2s_pc_create_learned(self.ctx.h, A.h, self.h, C.byref(o), C.byref(h)), "pc_learned")
        P.h = h
        return P

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.ctx.h:
                lib().b2s_learner_destroy(self.h)
        except Exception:
            pass


PERSIST_AUTO, PERSIST_STRIPS, PERSIST_OFF = range(3)


def solve_opts(tol=1e-10, maxit=2000, restart=30, orth=ORTH_MGS, ir_steps=0, ir_inner_tol=0.0, check_every=0,
               use_graphs=1, stall_window=0, persistent=PERSIST_AUTO) -> SolveOpts:
    o = SolveOpts()
    lib().b2s_solve_opts_default(C.byref(o))
    o.tol, o.maxit, o.restart, o.orth = tol, maxit, restart, orth
    o.ir_steps, o.ir_inner_tol, o.check_every, o.use_graphs = ir_steps, ir_inner_tol, check_every, use_graphs
    o.stall_window = stall_window
    o.persistent = persistent
    return o


def solve(ctx: Context, A, b, method=PCG, pc=None, raise_on_error=True, **opts):
    """x, stats = solve(ctx, A, b, method, pc, tol=..., maxit=..., restart=...)."""
    o = solve_opts(**opts)
    st = Stats()
    x = np.zeros(A.n)
    fn = lib().b2s_solve_baij if isinstance(A, BAIJ) else lib().b2s_solve
    rc = fn(ctx.h, A.h, pc.h if pc is not None else None, method, C.byref(o), _f64(b), x, C.byref(st))
    if rc != OK and raise_on_error:
        ctx.check(rc, "solve")
    return x, st.as_dict()


def sor(ctx: Context, A, b, omega, tol=1e-10, maxit=2000, red_black=False):
    """x, stats = sor(ctx, A, b, omega, tol, maxit, red_black): SMatrix::sor / sor_rb."""
    st = Stats()
    x = np.zeros(A.n)
    ctx.check(lib().b2s_sor(ctx.h, A.h, 1 if red_black else 0, float(omega), float(tol), int(maxit), _f64(b), x,
                            C.byref(st)), "sor_rb" if red_black else "sor")
    return x, st.as_dict()


def solve_device(ctx: Context, A, b_ptr: int, x_ptr: int, method=PCG, pc=None, **opts):
    """Solve with device pointers (e.g. torch tensors' data_ptr()) on ctx's stream."""
    o = solve_opts(**opts)
    st = Stats()
    fn = lib().b2s_solve_baij_device if isinstance(A, BAIJ) else lib().b2s_solve_device
    ctx.check(fn(ctx.h, A.h, pc.h if pc is not None else None, method, C.byref(o), C.c_void_p(b_ptr),
                 C.c_void_p(x_ptr), C.byref(st)), "solve")
    return st.as_dict()


def dot_device(ctx: Context, n: int, a_ptr: int, b_ptr: int) -> float:
    """SMatrix::dot of two device vectors (fixed-order reduction, on ctx's stream)."""
    out = C.c_double()
    ctx.check(lib().b2s_dot_device(ctx.h, int(n), C.c_void_p(a_ptr), C.c_void_p(b_ptr), C.byref(out)), "dot")
    return out.value


def dot(ctx: Context, a, b) -> float:
    out = C.c_double()
    a, b = _f64(a), _f64(b)
    ctx.check(lib().b2s_dot(ctx.h, len(a), a, b, C.byref(out)), "dot")
    return out.value


def pc_kind_from_name(method: int, name: str) -> int:
    k = C.c_int()
    st = lib().b2s_pc_kind_from_name(method, name.encode(), C.byref(k))
    if st != OK:
        raise B2SInvalidArgument(st, f"unknown preconditioner type: {name}")
    return k.value


# ------------------------------------------------------------------ generators

def _gen_csr(fn, *args):
    n, nnz = C.c_uint32(), C.c_uint32()
    st = fn(*args, C.byref(n), C.byref(nnz), None, None, None)
    if st != OK:
        _raise(st, "generator")
    rp = np.zeros(n.value + 1, np.uint32)
    ci = np.zeros(nnz.value, np.uint32)
    v = np.zeros(nnz.value, np.float64)
    fn(*args, C.byref(n), C.byref(nnz), _ptr(rp), _ptr(ci), _ptr(v))
    return n.value, rp, ci, v


def gen_poisson2d(N):
    """2-D 5-point Poisson, N x N interior grid: (n, rp, ci, v)."""
    return _gen_csr(lib().b2s_gen_poisson2d, N)


def gen_poisson3d(N):
    """3-D 7-point Poisson on N^3: (n, rp, ci, v)."""
    return _gen_csr(lib().b2s_gen_poisson3d, N)


def gen_convdiff3d(N, vx=10.0, vy=5.0, vz=2.5):
    """3-D upwind convection-diffusion on N^3: (n, rp, ci, v)."""
    return _gen_csr(lib().b2s_gen_convdiff3d, N, vx, vy, vz)


def gen_elasticity_q1(NE, E=1.0, nu=0.3):
    """Q1 hex elasticity, NE^3 elements, x=0 face clamped: (nbr, rp, ci, v) with 3x3 blocks."""
    nbr, nnzb = C.c_uint32(), C.c_uint32()
    st = lib().b2s_gen_elasticity_q1(NE, E, nu, C.byref(nbr), C.byref(nnzb), None, None, None)
    if st != OK:
        _raise(st, "generator")
    rp = np.zeros(nbr.value + 1, np.uint32)
    ci = np.zeros(nnzb.value, np.uint32)
    v = np.zeros(nnzb.value * 9, np.float64)
    lib().b2s_gen_elasticity_q1(NE, E, nu, C.byref(nbr), C.byref(nnzb), _ptr(rp), _ptr(ci), _ptr(v))
    return nbr.value, rp, ci, v


def grf_variance(seed: int) -> float:
    """Per-instance log-k variance, uniform in [1, 4], drawn from the seed."""
    u = uniform(seed ^ 0x7F4A7C15, 1)[0]
    return 1.0 + 1.5 * (u + 1.0)


def gen_grf_diffusion(N, seed, corr=0.05, var=None, with_k=False):
    """-div(k grad u) on N x N with log k a squared-exponential GRF: (n, rp, ci, v[, k])."""
    if var is None:
        var = grf_variance(seed)
    n, nnz = C.c_uint32(), C.c_uint32()
    L = lib()
    st = L.b2s_gen_grf_diffusion(N, corr, var, seed, C.byref(n), C.byref(nnz), None, None, None, None)
    if st != OK:
        _raise(st, "generator")
    rp = np.zeros(n.value + 1, np.uint32)
    ci = np.zeros(nnz.value, np.uint32)
    v = np.zeros(nnz.value, np.float64)
    k = np.zeros(n.value, np.float64)
    L.b2s_gen_grf_diffusion(N, corr, var, seed, C.byref(n), C.byref(nnz), _ptr(rp), _ptr(ci), _ptr(v), _ptr(k))
    return (n.value, rp, ci, v, k) if with_k else (n.value, rp, ci, v)


def uniform(seed: int, n: int) -> np.ndarray:
    """Counter-based uniform[-1, 1) vector (splitmix64)."""
    out = np.zeros(n, np.float64)
    lib().b2s_gen_uniform(seed, n, out)
    return out


# ------------------------------------------------- reference-facing mirror

_METHOD_OF = {"pcg": PCG, "bicgstab": BICGSTAB, "gmres": GMRES}


class SMatrix:
    """Mirror of sparse::SMatrix (array.hpp:266-373) on the GPU.

    Built from COO (sorted, duplicates merged, zeros dropped as the reference's
    constructor does) or from CSR arrays; solvers are static methods that
    return ``(x, it)`` with the reference's iteration conventions.
    """

    _ctx: Context | None = None

    @classmethod
    def context(cls) -> Context:
        if cls._ctx is None:
            cls._ctx = Context(int(os.environ.get("B2S_DEVICE", "0")))
        return cls._ctx

    def __init__(self, rows, cols, values=None, rowlist=None, collist=None, *, row_ptr=None, col_idx=None):
        self._rows, self._cols = int(rows), int(cols)
        if row_ptr is not None:
            self._rp, self._ci, self._v = _u32(row_ptr), _u32(col_idx), _f64(values)
        else:
            v, r, c = _f64(values), np.asarray(rowlist, np.int64), np.asarray(collist, np.int64)
            if not (len(v) == len(r) == len(c)):
                raise ValueError("COO input error: values, rowlist, collist differ in length")
            if len(r) and (r.min() < 0 or c.min() < 0 or r.max() >= rows or c.max() >= cols):
                raise IndexError("COO input error: row or column out of range")
            keep = v != 0.0
            r, c, v = r[keep], c[keep], v[keep]
            order = np.lexsort((np.arange(len(r)), c, r))
            r, c, v = r[order], c[order], v[order]
            if len(r):
                key = r * cols + c
                first = np.concatenate(([True], key[1:] != key[:-1]))
                grp = np.cumsum(first) - 1
                vs = np.zeros(int(grp[-1]) + 1)
                for k in range(len(v)):  # input-order summation of duplicates
                    vs[grp[k]] += v[k]
                r, c, v = r[first], c[first], vs
                nz = v != 0.0
                r, c, v = r[nz], c[nz], v[nz]
            self._rp = np.zeros(rows + 1, np.uint32)
            np.add.at(self._rp, r + 1, 1)
            self._rp = np.cumsum(self._rp, dtype=np.uint64).astype(np.uint32)
            self._ci, self._v = c.astype(np.uint32), v.astype(np.float64)
        self._dev = None

    def rows(self):
        return self._rows

    def cols(self):
        return self._cols

    def nnz(self):
        return len(self._v)

    def values(self):
        return self._v

    def row_ptr(self):
        return self._rp

    def col_idx(self):
        return self._ci

    def device(self) -> CSR:
        if self._dev is None:
            self._dev = CSR(self.context(), self._rows, self._cols, self._rp, self._ci, self._v)
        return self._dev

    @staticmethod
    def dot(a, b):
        if len(a) != len(b):
            raise ValueError("dot: vector lengths differ")
        return dot(SMatrix.context(), a, b)

    @staticmethod
    def spmv(A: "SMatrix", x):
        if A._cols != len(x):
            raise ValueError("spmv: matrix columns differ from vector length")
        return A.device().spmv(x)

    @staticmethod
    def _solve(A, b, method, precond, tol, max_iter, restart=30):
        if A._rows != A._cols:
            raise ValueError("solver needs a square matrix")
        if A._cols != len(b):
            raise ValueError("matrix columns differ from vector length")
        ctx = SMatrix.context()
        b = _f64(b)
        normb = float(np.sqrt(np.dot(b, b)))
        if normb < 1e-300:
            return np.zeros(len(b)), 0
        if method != GMRES and 1.0 < tol:
            return np.zeros(len(b)), 0
        if isinstance(precond, str):
            kind = pc_kind_from_name(method, precond)
            pc = Precond(ctx, A.device(), kind) if kind != PC_NONE else None
        elif callable(precond):
            pc = HostPrecond(ctx, A._rows, lambda r: precond(r))
        else:
            pc = precond
        x, st = solve(ctx, A.device(), b, method, pc, raise_on_error=False, tol=tol, maxit=max_iter,
                      restart=restart)
        if st["status"] not in (OK, DIVERGED):
            ctx.check(st["status"], "solve")
        return x, st["it"]

    @staticmethod
    def pcg(A, b, precond="none", tol=1e-10, max_iter=2000):
        return SMatrix._solve(A, b, PCG, precond, tol, max_iter)

    @staticmethod
    def bicgstab(A, b, precond, tol=1e-10, max_iter=2000):
        return SMatrix._solve(A, b, BICGSTAB, precond, tol, max_iter)

    @staticmethod
    def gmres(A, b, precond, restart, tol=1e-10, max_iter=2000):
        return SMatrix._solve(A, b, GMRES, precond, tol, max_iter, restart)

    @staticmethod
    def sor(A, b, omega, tol=1e-10, max_iter=2000):
        if A._rows != A._cols:
            raise ValueError("SOR needs a square matrix")
        x, st = sor(SMatrix.context(), A.device(), _f64(b), omega, tol, max_iter)
        return x, st["it"]

    @staticmethod
    def sor_rb(A, b, omega, tol=1e-10, max_iter=2000):
        if A._rows != A._cols:
            raise ValueError("red-black SOR needs a square matrix")
        x, st = sor(SMatrix.context(), A.device(), _f64(b), omega, tol, max_iter, red_black=True)
        return x, st["it"]

    @staticmethod
    def amg(A, b, tol=1e-10, max_iter=2000):
        """SMatrix::amg (array.cpp:4534-4563): x += one V-cycle of the residual
        from x = 0 until ||b - A x|| / ||b|| < tol; smoothed aggregation."""
        if A._rows != A._cols:
            raise ValueError("AMG needs a square matrix")
        if A._cols != len(b):
            raise ValueError("AMG: matrix columns differ from vector length")
        b = _f64(b)
        if float(np.sqrt(np.dot(b, b))) < 1e-300:
            return np.zeros(len(b)), 0
        ctx = SMatrix.context()
        pc = Precond(ctx, A.device(), PC_SA_AMG)
        x, st = solve(ctx, A.device(), b, STATIONARY, pc, raise_on_error=False, tol=tol, maxit=max_iter)
        if st["status"] not in (OK, DIVERGED):
            ctx.check(st["status"], "amg")
        return x, st["it"]

    def transpose(self) -> "SMatrix":
        T = self.device().transpose()
        return SMatrix(self._cols, self._rows, T.v, row_ptr=T.rp, col_idx=T.ci)

    def __mul__(self, B: "SMatrix") -> "SMatrix":
        if self._cols != B._rows:
            raise ValueError("matrix product: columns of A differ from rows of B")
        P = self.device().matmul(B.device())
        return SMatrix(self._rows, B._cols, P.v, row_ptr=P.rp, col_idx=P.ci)


def load_extension() -> str:
    """Path of the loaded native library (fails loudly when missing)."""
    lib()
    return LIB_PATH

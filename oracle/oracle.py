"""ctypes bindings for the two CPU oracles of the sparse solver path.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and
bench.py's reference / cpu_baseline legs import this module, as the checker
and as the timed CPU baseline.  The product (``cpp-fem-solver_b200``) never
imports it.

* ``Orc`` -- ``oracle/_ref/liborc.so``, the C restatement in
  ``oracle/b2s_oracle.c`` (each function cites the reference file:line).
* ``Ref`` -- ``oracle/_ref/libref.so``, the reference library itself
  (ode-solver/src/math/array.cpp + include/math/blockMatrix.hpp) compiled from
  its sources by ``oracle/Makefile`` through ``oracle/ref_harness.cpp``.
* ``Gen`` -- ``oracle/_ref/libgen.so``, the library's CPU problem generators
  built on their own, so that the benchmark's reference arm makes the same
  systems without loading the product library.

Both expose the same Python surface so tests can run one case through either.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class OracleError(Exception):
    """Raised with the oracle's status code: 1 invalid argument, 2 breakdown."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


def build(quiet: bool = True) -> None:
    """Build oracle/_ref/liborc.so and libgen.so (always) and libref.so (when
    B2S_REFERENCE_SRC names the reference's ode-solver directory)."""
    subprocess.run(["make", "-C", HERE], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class _CSR:
    """CSR matrix owned by one oracle library."""

    def __init__(self, lib, handle, n, m):
        self._lib, self.h, self.n, self.m = lib, handle, n, m

    def __del__(self):
        try:
            self._lib._csr_free(self.h)
        except Exception:
            pass

    def export(self):
        nnz = self._lib._csr_nnz(self.h)
        rp = np.zeros(self.n + 1, np.uint32)
        ci = np.zeros(nnz, np.uint32)
        v = np.zeros(nnz, np.float64)
        self._lib._csr_export(self.h, rp, ci, v)
        return rp, ci, v


class _Blk:
    def __init__(self, lib, handle, bs, nbr):
        self._lib, self.h, self.bs, self.nbr = lib, handle, bs, nbr

    def __del__(self):
        try:
            self._lib._blk_free(self.h)
        except Exception:
            pass

    def export(self):
        nnzb = self._lib._blk_nnzb(self.h)
        rp = np.zeros(self.nbr + 1, np.uint32)
        ci = np.zeros(nnzb, np.uint32)
        v = np.zeros(nnzb * self.bs * self.bs, np.float64)
        self._lib._blk_export(self.h, rp, ci, v)
        return rp, ci, v


class _PC:
    def __init__(self, lib, handle, n, kind):
        self._lib, self.h, self.n, self.kind = lib, handle, n, kind

    def __del__(self):
        try:
            self._lib._pc_free(self.h)
        except Exception:
            pass

    def apply(self, r):
        z = np.zeros(self.n, np.float64)
        self._lib._pc_apply(self.h, _f64(r), z)
        return z


class _Lib:
    prefix = ""

    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        self.path = path
        self._bind()

    def _f(self, name, res, *args):
        fn = getattr(self.lib, self.prefix + name)
        fn.restype = res
        fn.argtypes = list(args)
        return fn

    def _bind(self):
        vp, u32, f64, i32, u64, cp = C.c_void_p, C.c_uint32, C.c_double, C.c_int, C.c_uint64, C.c_char_p
        self._csr_free = self._f("csr_free", None, vp)
        self._csr_nnz = self._f("csr_nnz", u32, vp)
        self._csr_export = self._f("csr_export", None, vp, u32p, u32p, f64p)
        self._csr_transpose = self._f("csr_transpose", vp, vp)
        self._csr_matmul = self._f("csr_matmul", vp, vp, vp)
        self._pc_apply = self._f("pc_apply", None, vp, f64p, f64p)
        self._pc_free = self._f("pc_free", None, vp)
        self._blk_free = self._f("blk_free", None, vp)
        self._blk_nnzb = self._f("blk_nnzb", u32, vp)
        self._blk_export = self._f("blk_export", None, vp, u32p, u32p, f64p)
        self._blk_transpose = self._f("blk_transpose", vp, vp)
        self._blk_rows = self._f("blk_rows", u32, vp)
        self._blk_matvec = self._f("blk_matvec", None, vp, f64p, f64p)
        self._blk_gmres = self._f("blk_gmres", i32, vp, f64p, cp, f64, i32, i32, f64p, C.POINTER(C.c_int), cp, i32)

    @staticmethod
    def _check(st, err):
        if st != 0:
            raise OracleError(st, err.value.decode(errors="replace"))

    # ---- CSR ----
    def csr(self, n, m, rp, ci, v):
        raise NotImplementedError

    def csr_from_coo(self, n, m, v, r, c):
        raise NotImplementedError

    def transpose(self, A):
        return _CSR(self, self._csr_transpose(A.h), A.m, A.n)

    def matmul(self, A, B):
        return _CSR(self, self._csr_matmul(A.h, B.h), A.n, B.m)

    # ---- block ----
    def blk_export(self, B):
        return B.export()

    def blk_transpose(self, B):
        h = self._blk_transpose(B.h)
        return _Blk(self, h, B.bs, self._blk_rows(h))

    def blk_matvec(self, B, x):
        y = np.zeros(B.nbr * B.bs, np.float64)
        self._blk_matvec(B.h, _f64(x), y)
        return y

    def blk_gmres(self, B, b, precond, tol, maxit, restart):
        x = np.zeros(B.nbr * B.bs, np.float64)
        it = C.c_int(0)
        err = C.create_string_buffer(512)
        st = self._blk_gmres(B.h, _f64(b), precond.encode(), tol, maxit, restart, x, C.byref(it), err, 512)
        self._check(st, err)
        return x, it.value


class Orc(_Lib):
    """The C restatement (oracle/b2s_oracle.c)."""

    prefix = "orc_"

    def __init__(self, path=os.path.join(REF_DIR, "liborc.so")):
        super().__init__(path)
        vp, u32, f64, i32, u64, cp = C.c_void_p, C.c_uint32, C.c_double, C.c_int, C.c_uint64, C.c_char_p
        ip = C.POINTER(C.c_int)
        self._csr_from_coo = self._f("csr_from_coo", vp, u32, u32, u64, f64p, u32p, u32p, ip)
        self._csr_copy = self._f("csr_copy", vp, u32, u32, u32p, u32p, f64p)
        self._spmv = self._f("spmv", None, vp, f64p, f64p)
        self._dot = self._f("dot", f64, u64, f64p, f64p)
        self._pc_create = self._f("pc_create", vp, vp, cp, f64, ip, cp, i32)
        self._solve = self._f("solve", i32, vp, i32, cp, i32, f64, i32, f64p, f64p, ip, cp, i32)
        self._solve_pc = self._f("solve_pc", i32, vp, i32, vp, i32, f64, i32, f64p, f64p, ip, cp, i32)
        self._levels = self._f("levels", u32, u32, u32p, u32p, i32, u32p)
        self._ic0_export = self._f("ic0_export", i32, vp, u32p, vp, vp, vp, vp, vp, vp, vp)
        self._ilu0_export = self._f("ilu0_export", i32, vp, u32p, vp, vp, vp, vp, vp, vp, vp)
        self._colour_export = self._f("colour_export", i32, vp, u32p, u32p, u32p, u32p, f64p)
        self._blk_create = self._f("blk_create", vp, i32, u32, u32, u32p, u32p, f64p)
        self._blk_condense = self._f("blk_condense", vp, i32, vp, u32, u32)
        self._blk_matmul = self._f("blk_matmul", vp, vp, vp)
        self._blk_pc_create = self._f("blk_pc_create", vp, vp, cp, ip, cp, i32)
        self._blk_ilu0_export = self._f("blk_ilu0_export", i32, vp, u32p, vp, vp, vp, vp, vp, vp, vp, vp)
        self._blk_amg_export = self._f("blk_amg_export", i32, vp, i32, u32p, vp, vp, vp, vp, vp, vp, vp)
        self._blk_amg_aggregates = self._f("blk_amg_aggregates", i32, vp, i32, i32p)
        self._blk_solve_pc = self._f("blk_solve_pc", i32, vp, i32, vp, i32, f64, i32, f64p, f64p, ip, cp, i32)
        self._blk_dist_matvec = self._f("blk_dist_matvec", None, i32, u32, u32p, u32p, f64p, u32, f64p, f64p)

    def csr(self, n, m, rp, ci, v):
        return _CSR(self, self._csr_copy(n, m, _u32(rp), _u32(ci), _f64(v)), n, m)

    def blk_dist_matvec(self, bs, rp, lci, v, n_owned, x_full):
        """BlockMatrix::distributed_matvec after the exchange (owned pass, then ghosts)."""
        nbr = len(rp) - 1
        y = np.zeros(nbr * bs, np.float64)
        self._blk_dist_matvec(bs, nbr, _u32(rp), _u32(lci), _f64(v), n_owned, _f64(x_full), y)
        return y

    def csr_from_coo(self, n, m, v, r, c):
        st = C.c_int(0)
        v, r, c = _f64(v), _u32(r), _u32(c)
        h = self._csr_from_coo(n, m, len(v), v, r, c, C.byref(st))
        if not h:
            raise OracleError(st.value, "COO input out of range")
        return _CSR(self, h, n, m)

    def spmv(self, A, x):
        y = np.zeros(A.n, np.float64)
        self._spmv(A.h, _f64(x), y)
        return y

    def dot(self, a, b):
        a, b = _f64(a), _f64(b)
        return self._dot(len(a), a, b)

    def levels(self, n, rp, ci, upper=False):
        lev = np.zeros(n, np.uint32)
        nl = self._levels(n, _u32(rp), _u32(ci), 1 if upper else 0, lev)
        return lev, nl

    def pc(self, A, kind, omega=1.2):
        st, err = C.c_int(0), C.create_string_buffer(512)
        h = self._pc_create(A.h, kind.encode(), omega, C.byref(st), err, 512)
        if not h:
            self._check(st.value or 1, err)
        return _PC(self, h, A.n, kind)

    def blk_pc(self, B, kind):
        st, err = C.c_int(0), C.create_string_buffer(512)
        h = self._blk_pc_create(B.h, kind.encode(), C.byref(st), err, 512)
        if not h:
            self._check(st.value or 1, err)
        return _PC(self, h, B.nbr * B.bs, "blk_" + kind)

    def solve(self, A, method, precond, b, tol=1e-10, maxit=2000, restart=30):
        x = np.zeros(A.n, np.float64)
        it, err = C.c_int(0), C.create_string_buffer(512)
        st = self._solve(A.h, method, precond.encode(), restart, tol, maxit, _f64(b), x, C.byref(it), err, 512)
        self._check(st, err)
        return x, it.value

    def solve_pc(self, A, method, pc, b, tol=1e-10, maxit=2000, restart=30):
        x = np.zeros(A.n, np.float64)
        it, err = C.c_int(0), C.create_string_buffer(512)
        st = self._solve_pc(A.h, method, pc.h if pc is not None else None, restart, tol, maxit, _f64(b), x,
                            C.byref(it), err, 512)
        self._check(st, err)
        return x, it.value

    def blk(self, bs, nbr, nbc, rp, ci, v):
        return _Blk(self, self._blk_create(bs, nbr, nbc, _u32(rp), _u32(ci), _f64(v)), bs, nbr)

    def blk_condense(self, bs, A, nbr, nbc):
        return _Blk(self, self._blk_condense(bs, A.h, nbr, nbc), bs, nbr)

    def blk_matmul(self, A, B):
        return _Blk(self, self._blk_matmul(A.h, B.h), A.bs, A.nbr)

    def blk_solve_pc(self, B, method, pc, b, tol=1e-10, maxit=2000, restart=30):
        x = np.zeros(B.nbr * B.bs, np.float64)
        it, err = C.c_int(0), C.create_string_buffer(512)
        st = self._blk_solve_pc(B.h, method, pc.h if pc is not None else None, restart, tol, maxit, _f64(b), x,
                                C.byref(it), err, 512)
        self._check(st, err)
        return x, it.value

    def amg_aggregates(self, pc, level, nrows):
        agg = np.zeros(nrows, np.int32)
        if self._blk_amg_aggregates(pc.h, level, agg) != 0:
            raise OracleError(1, "no aggregates on that level")
        return agg

    # exports shared with Ref
    ic0_export = lambda self, pc: _ic0_export(self._ic0_export, pc)
    ilu0_export = lambda self, pc: _ilu0_export(self._ilu0_export, pc)
    colour_export = lambda self, pc, A=None: _colour_export_orc(self._colour_export, pc)
    blk_ilu0_export = lambda self, pc, bs: _blk_ilu0_export(lambda *a: self._blk_ilu0_export(*a), pc, bs)
    amg_export = lambda self, pc, bs: _amg_export(lambda *a: self._blk_amg_export(*a), pc, bs)


class Ref(_Lib):
    """The reference library compiled from its own sources (oracle/_ref/libref.so)."""

    prefix = "ref_"

    def __init__(self, path=os.path.join(REF_DIR, "libref.so")):
        super().__init__(path)
        vp, u32, f64, i32, u64, cp = C.c_void_p, C.c_uint32, C.c_double, C.c_int, C.c_uint64, C.c_char_p
        ip = C.POINTER(C.c_int)
        self._set_threads = self._f("set_threads", None, i32)
        self.max_threads = self._f("max_threads", i32)
        self._csr_coo = self._f("csr_coo", vp, u32, u32, u64, f64p, u32p, u32p, cp, i32)
        self._csr_direct = self._f("csr_direct", vp, u32, u32, u32p, u32p, f64p)
        self._spmv = self._f("spmv", None, vp, f64p, f64p)
        self._dot = self._f("dot", f64, f64p, f64p, u64)
        self._solve = self._f("solve", i32, vp, i32, cp, i32, f64, i32, f64p, f64p, ip, cp, i32)
        self._sor = self._f("sor", i32, vp, i32, f64, f64, i32, f64p, f64p, ip, cp, i32)
        self._pc_create = self._f("pc_create", vp, vp, cp, f64, cp, i32)
        self._gmres_pc = self._f("gmres_pc", i32, vp, vp, i32, f64, i32, f64p, f64p, ip, cp, i32)
        self._ic0_export = self._f("ic0_export", i32, vp, u32p, vp, vp, vp, vp, vp, vp, vp)
        self._ilu0_export = self._f("ilu0_export", i32, vp, u32p, vp, vp, vp, vp, vp, vp, vp)
        self._redblack = self._f("redblack", i32, vp, u32p, u32p, u32p, u32p, f64p, cp, i32)
        self._blk_create = self._f("blk_create", vp, i32, u32, u32, u32p, u32p, f64p)
        self._blk_condense = self._f("blk_condense", vp, i32, vp, u32, u32)
        self._blk_pc_create = self._f("blk_pc_create", vp, vp, cp, cp, i32)
        self._blk_ilu0_export = self._f("blk_ilu0_export", i32, vp, i32, u32p, vp, vp, vp, vp, vp, vp, vp, vp)
        self._blk_amg_export = self._f("blk_amg_export", i32, vp, i32, i32, u32p, vp, vp, vp, vp, vp, vp, vp)
        self._schur_create = self._f("schur_create", vp, u32, u32, vp, vp, vp, vp, f64)

    def set_threads(self, t: int):
        self._set_threads(int(t))

    def csr(self, n, m, rp, ci, v):
        return _CSR(self, self._csr_direct(n, m, _u32(rp), _u32(ci), _f64(v)), n, m)

    def csr_from_coo(self, n, m, v, r, c):
        err = C.create_string_buffer(512)
        v, r, c = _f64(v), _u32(r), _u32(c)
        h = self._csr_coo(n, m, len(v), v, r, c, err, 512)
        if not h:
            raise OracleError(1, err.value.decode(errors="replace"))
        return _CSR(self, h, n, m)

    def spmv(self, A, x):
        y = np.zeros(A.n, np.float64)
        self._spmv(A.h, _f64(x), y)
        return y

    def dot(self, a, b):
        a, b = _f64(a), _f64(b)
        return self._dot(a, b, len(a))

    def pc(self, A, kind, omega=1.2):
        err = C.create_string_buffer(512)
        h = self._pc_create(A.h, kind.encode(), omega, err, 512)
        if not h:
            raise OracleError(2, err.value.decode(errors="replace"))
        return _PC(self, h, A.n, kind)

    def blk_pc(self, B, kind):
        err = C.create_string_buffer(512)
        h = self._blk_pc_create(B.h, kind.encode(), err, 512)
        if not h:
            raise OracleError(2, err.value.decode(errors="replace"))
        return _PC(self, h, B.nbr * B.bs, "blk_" + kind)

    def solve(self, A, method, precond, b, tol=1e-10, maxit=2000, restart=30):
        x = np.zeros(A.n, np.float64)
        it, err = C.c_int(0), C.create_string_buffer(512)
        st = self._solve(A.h, method, precond.encode(), restart, tol, maxit, _f64(b), x, C.byref(it), err, 512)
        self._check(st, err)
        return x, it.value

    def sor(self, A, b, omega, tol=1e-10, maxit=2000, red_black=False):
        """SMatrix::sor / sor_rb of the compiled reference: (x, it)."""
        x = np.zeros(A.n, np.float64)
        it, err = C.c_int(0), C.create_string_buffer(512)
        st = self._sor(A.h, 1 if red_black else 0, omega, tol, maxit, _f64(b), x, C.byref(it), err, 512)
        self._check(st, err)
        return x, it.value

    def gmres_pc(self, A, pc, b, restart=30, tol=1e-10, maxit=2000):
        x = np.zeros(A.n, np.float64)
        it, err = C.c_int(0), C.create_string_buffer(512)
        st = self._gmres_pc(A.h, pc.h, restart, tol, maxit, _f64(b), x, C.byref(it), err, 512)
        self._check(st, err)
        return x, it.value

    def schur(self, n_vel, n_pres, B, Bt, A_pc, S_pc=None, scale=1.0):
        """The reference's make_schur_preconditioner with these parts (S_pc
        None: identity; else z = scale * S_pc(r))."""
        h = self._schur_create(n_vel, n_pres, B.h, Bt.h, A_pc.h, S_pc.h if S_pc is not None else None, scale)
        pc = _PC(self, h, n_vel + n_pres, "schur")
        pc._keep = (B, Bt, A_pc, S_pc)
        return pc

    def redblack(self, A):
        n = A.n
        nc = np.zeros(1, np.uint32)
        cp_ = np.zeros(n + 1, np.uint32)
        nid = np.zeros(n, np.uint32)
        perm = np.zeros(n, np.uint32)
        d2 = np.zeros(n, np.float64)
        err = C.create_string_buffer(512)
        self._check(self._redblack(A.h, nc, cp_, nid, perm, d2, err, 512), err)
        return int(nc[0]), cp_[: int(nc[0]) + 1].copy(), nid, perm, d2

    def blk(self, bs, nbr, nbc, rp, ci, v):
        return _Blk(self, self._blk_create(bs, nbr, nbc, _u32(rp), _u32(ci), _f64(v)), bs, nbr)

    def blk_condense(self, bs, A, nbr, nbc):
        return _Blk(self, self._blk_condense(bs, A.h, nbr, nbc), bs, nbr)

    ic0_export = lambda self, pc: _ic0_export(self._ic0_export, pc)
    ilu0_export = lambda self, pc: _ilu0_export(self._ilu0_export, pc)
    blk_ilu0_export = lambda self, pc, bs: _blk_ilu0_export(lambda h, *a: self._blk_ilu0_export(h, bs, *a), pc, bs)
    amg_export = lambda self, pc, bs: _amg_export(lambda h, lvl, *a: self._blk_amg_export(h, bs, lvl, *a), pc, bs)


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _ic0_export(fn, pc):
    sizes = np.zeros(2, np.uint32)
    if fn(pc.h, sizes, None, None, None, None, None, None, None) != 0:
        raise OracleError(1, "not an IC(0) preconditioner")
    n = pc.n
    Lrp, Lci, Lv = np.zeros(n + 1, np.uint32), np.zeros(sizes[0], np.uint32), np.zeros(sizes[0])
    Trp, Tci, Tv = np.zeros(n + 1, np.uint32), np.zeros(sizes[1], np.uint32), np.zeros(sizes[1])
    d = np.zeros(n)
    fn(pc.h, sizes, *map(_ptr, (Lrp, Lci, Lv, Trp, Tci, Tv, d)))
    return dict(Lrp=Lrp, Lci=Lci, Lv=Lv, LTrp=Trp, LTci=Tci, LTv=Tv, diag=d)


def _ilu0_export(fn, pc):
    sizes = np.zeros(2, np.uint32)
    if fn(pc.h, sizes, None, None, None, None, None, None, None) != 0:
        raise OracleError(1, "not an ILU(0) preconditioner")
    n = pc.n
    Lrp, Lci, Lv = np.zeros(n + 1, np.uint32), np.zeros(sizes[0], np.uint32), np.zeros(sizes[0])
    Urp, Uci, Uv = np.zeros(n + 1, np.uint32), np.zeros(sizes[1], np.uint32), np.zeros(sizes[1])
    di = np.zeros(n, np.uint32)
    fn(pc.h, sizes, *map(_ptr, (Lrp, Lci, Lv, Urp, Uci, Uv, di)))
    return dict(Lrp=Lrp, Lci=Lci, Lv=Lv, Urp=Urp, Uci=Uci, Uv=Uv, diag_idx=di)


def _colour_export_orc(fn, pc):
    n = pc.n
    nc = np.zeros(1, np.uint32)
    cp_ = np.zeros(n + 1, np.uint32)
    nid, perm, d2 = np.zeros(n, np.uint32), np.zeros(n, np.uint32), np.zeros(n)
    if fn(pc.h, nc, cp_, nid, perm, d2) != 0:
        raise OracleError(1, "not an SSOR preconditioner")
    return int(nc[0]), cp_[: int(nc[0]) + 1].copy(), nid, perm, d2


def _blk_ilu0_export(fn, pc, bs):
    sizes = np.zeros(2, np.uint32)
    if fn(pc.h, sizes, None, None, None, None, None, None, None, None) != 0:
        raise OracleError(1, "not a block ILU(0) preconditioner")
    nb, bv = pc.n // bs, bs * bs
    Lrp, Lci, Lv = np.zeros(nb + 1, np.uint32), np.zeros(sizes[0], np.uint32), np.zeros(int(sizes[0]) * bv)
    Urp, Uci, Uv = np.zeros(nb + 1, np.uint32), np.zeros(sizes[1], np.uint32), np.zeros(int(sizes[1]) * bv)
    Ud, inv = np.zeros(nb, np.uint32), np.zeros(nb * bv)
    fn(pc.h, sizes, *map(_ptr, (Lrp, Lci, Lv, Urp, Uci, Uv, Ud, inv)))
    return dict(Lrp=Lrp, Lci=Lci, Lv=Lv, Urp=Urp, Uci=Uci, Uv=Uv, Udiag=Ud, inv_diag=inv)


def _amg_export(fn, pc, bs):
    """List of levels: dict(nrows, Arp, Aci, Av, Prp, Pci, Pv, ncols_P, diag_inv)."""
    sizes = np.zeros(4, np.uint32)
    nlev = fn(pc.h, -1, sizes, None, None, None, None, None, None, None)
    if nlev < 0:
        raise OracleError(1, "not an AMG preconditioner")
    out = []
    bv = bs * bs
    for lvl in range(nlev):
        fn(pc.h, lvl, sizes, None, None, None, None, None, None, None)
        nr, nnzA, ncP, nnzP = (int(s) for s in sizes)
        Arp, Aci, Av = np.zeros(nr + 1, np.uint32), np.zeros(nnzA, np.uint32), np.zeros(nnzA * bv)
        Prp, Pci, Pv = np.zeros(nr + 1, np.uint32), np.zeros(max(nnzP, 1), np.uint32), np.zeros(max(nnzP, 1) * bv)
        dinv = np.zeros(nr * bv)
        fn(pc.h, lvl, sizes, *map(_ptr, (Arp, Aci, Av, Prp, Pci, Pv, dinv)))
        lv = dict(nrows=nr, Arp=Arp, Aci=Aci, Av=Av, diag_inv=dinv, ncols_P=ncP)
        if nnzP:
            lv.update(Prp=Prp, Pci=Pci[:nnzP], Pv=Pv[: nnzP * bv])
        out.append(lv)
    return out


class Gen:
    """The problem generators of ``cpp-fem-solver_b200/csrc/gen.cpp`` from
    ``oracle/_ref/libgen.so`` (same source and flags as the product build, so
    the same systems bit for bit)."""

    def __init__(self, path=os.path.join(REF_DIR, "libgen.so")):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        self.path = path
        vp, u32, f64, u64 = C.c_void_p, C.c_uint32, C.c_double, C.c_uint64
        pu = C.POINTER(C.c_uint32)
        self._grf = self.lib.b2s_gen_grf_diffusion
        self._grf.restype = C.c_int
        self._grf.argtypes = [u32, f64, f64, u64, pu, pu, vp, vp, vp, vp]
        self._uni = self.lib.b2s_gen_uniform
        self._uni.restype = C.c_int
        self._uni.argtypes = [u64, u64, vp]

    def uniform(self, seed: int, n: int) -> np.ndarray:
        """Counter-based uniform[-1, 1) vector (splitmix64), as b2s.uniform."""
        out = np.zeros(n, np.float64)
        if self._uni(seed, n, _ptr(out)) != 0:
            raise OracleError(1, "uniform generator failed")
        return out

    def grf_variance(self, seed: int) -> float:
        """Per-instance log-k variance in [1, 4], as b2s.grf_variance."""
        u = self.uniform(seed ^ 0x7F4A7C15, 1)[0]
        return 1.0 + 1.5 * (u + 1.0)

    def grf_diffusion(self, N: int, seed: int, corr: float = 0.05):
        """512^2-style GRF diffusion system: (n, rp, ci, v), as b2s.gen_grf_diffusion."""
        var = self.grf_variance(seed)
        n, nnz = C.c_uint32(), C.c_uint32()
        if self._grf(N, corr, var, seed, C.byref(n), C.byref(nnz), None, None, None, None) != 0:
            raise OracleError(1, "GRF generator failed")
        rp = np.zeros(n.value + 1, np.uint32)
        ci = np.zeros(nnz.value, np.uint32)
        v = np.zeros(nnz.value, np.float64)
        self._grf(N, corr, var, seed, C.byref(n), C.byref(nnz), _ptr(rp), _ptr(ci), _ptr(v), None)
        return n.value, rp, ci, v

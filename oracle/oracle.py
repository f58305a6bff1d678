"""ctypes front end of the oracle library (oracle/liblfg_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, never by the product package.  It builds the
oracle from source on first use if the shared library is missing.

Two builds of the same C sources:
* lib() -- the strict build the tests check against (-O2, no FMA
  contraction);
* lib(native=True) -- the CPU baseline the benchmark times (-O3
  -march=native -fopenmp), built on the host that runs it under a name keyed
  by the host's CPU model and instruction-set flags, so a library built on
  one machine is never loaded on another.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import platform
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liblfg_oracle.so"

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


def build(force: bool = False) -> Path:
    srcs = [HERE / f for f in ("ora_kernels.c", "ora_solvers.c", "ora_real.inc", "lfg_oracle.h")]
    if force or not LIB_PATH.exists() or any(
            s.stat().st_mtime > LIB_PATH.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def _cpu_tag() -> str:
    """Short hash of the CPU model, its instruction-set flags and the
    compiler: what -march=native code depends on."""
    info = platform.processor() or ""
    try:
        txt = Path("/proc/cpuinfo").read_text()
        keep = [ln for ln in txt.splitlines() if ln.startswith(("model name", "flags"))]
        info += "\n".join(sorted(set(keep)))
    except OSError:
        pass
    try:
        info += subprocess.run(["gcc", "--version"], capture_output=True, text=True).stdout
    except OSError:
        pass
    return hashlib.sha1(info.encode()).hexdigest()[:12]


def build_native(force: bool = False) -> Path:
    """The -O3 -march=native -fopenmp build for this host's CPU."""
    out = HERE / "_native" / f"liblfg_oracle_{_cpu_tag()}.so"
    srcs = [HERE / f for f in ("ora_kernels.c", "ora_solvers.c", "ora_real.inc", "lfg_oracle.h")]
    if force or not out.exists() or any(s.stat().st_mtime > out.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE), "native", f"NATIVE_OUT={out}"],
                       check=True)
    return out


_libs = {}


def lib(native: bool = False) -> C.CDLL:
    if native not in _libs:
        path = build_native() if native else build()
        L = C.CDLL(str(path))
        L.ora_dot_d.restype = C.c_double
        L.ora_norm_d.restype = C.c_double
        L.ora_dot_f.restype = C.c_double
        L.ora_norm_f.restype = C.c_double
        L.ora_mg_work_size_d.restype = C.c_long
        L.ora_mg_work_size_f.restype = C.c_long
        _setup_signatures(L)
        _libs[native] = L
    return _libs[native]


def ptr(a: np.ndarray):
    """ctypes pointer to a contiguous numpy array (int32, float32 or float64)."""
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be contiguous")
    if a.dtype == np.float64:
        return a.ctypes.data_as(_dp)
    if a.dtype == np.float32:
        return a.ctypes.data_as(_fp)
    if a.dtype == np.int32:
        return a.ctypes.data_as(_ip)
    raise TypeError(a.dtype)


class HelmOp(C.Structure):
    _fields_ = [("ncol", C.c_int), ("nl", C.c_int), ("cm", C.c_void_p), ("hf", C.c_void_p),
                ("links", C.c_void_p)]


MAX_LEVELS = 8


class MGStruct(C.Structure):
    _fields_ = [("nlevels", C.c_int), ("n_pre", C.c_int), ("n_post", C.c_int),
                ("n_coarse", C.c_int), ("omega", C.c_double),
                ("op", HelmOp * MAX_LEVELS), ("child", C.c_void_p * MAX_LEVELS),
                ("work", C.c_void_p)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("final_err", C.c_double)]


class MixedInfo(C.Structure):
    _fields_ = [("outer_iterations", C.c_int), ("inner_iterations", C.c_int),
                ("final_rel_residual", C.c_double)]


class Helmholtz:
    """Oracle view of a HelmholtzProblem: operators of every MG level."""

    def __init__(self, prob, dtype=np.float64, native: bool = False):
        """native: run on the -O3 -march=native build (CPU timing) instead
        of the strict build the tests check against."""
        L = lib(native)
        self.L = L
        self.prob = prob
        self.nl = prob.nlayers
        self.keep = []
        # Galerkin coarse operators are built in double, then cast.
        cms = [np.ascontiguousarray(prob.cm, dtype=np.float64)]
        hfs = [np.ascontiguousarray(prob.hf, dtype=np.float64)]
        links = [np.ascontiguousarray(prob.links, dtype=np.int32)]
        for l, child in enumerate(prob.mg_child):
            child = np.ascontiguousarray(child, dtype=np.int32)
            lc = np.ascontiguousarray(prob.mg_links[l], dtype=np.int32)
            nc = lc.shape[0]
            fine = HelmOp(links[-1].shape[0], self.nl, cms[-1].ctypes.data, hfs[-1].ctypes.data,
                          links[-1].ctypes.data)
            cm_c = np.zeros(3 * self.nl * nc)
            hf_c = np.zeros(4 * self.nl * nc)
            L.ora_galerkin_coarsen(C.byref(fine), nc, ptr(child), ptr(lc), ptr(cm_c), ptr(hf_c))
            cms.append(cm_c)
            hfs.append(hf_c)
            links.append(lc)
        self.cm64, self.hf64, self.links = cms, hfs, links
        self.child = [np.ascontiguousarray(c, dtype=np.int32) for c in prob.mg_child]
        self.cm32 = [c.astype(np.float32) for c in cms]
        self.hf32 = [h.astype(np.float32) for h in hfs]

    def op(self, level: int = 0, dtype=np.float64) -> HelmOp:
        cm = self.cm64 if dtype == np.float64 else self.cm32
        hf = self.hf64 if dtype == np.float64 else self.hf32
        return HelmOp(self.links[level].shape[0], self.nl, cm[level].ctypes.data,
                      hf[level].ctypes.data, self.links[level].ctypes.data)

    def mg(self, dtype=np.float64, n_pre=2, n_post=2, n_coarse=8, omega=0.8, nlevels=None):
        nlev = len(self.links) if nlevels is None else nlevels
        s = MGStruct()
        s.nlevels, s.n_pre, s.n_post, s.n_coarse, s.omega = nlev, n_pre, n_post, n_coarse, omega
        for l in range(nlev):
            s.op[l] = self.op(l, dtype)
        for l in range(nlev - 1):
            s.child[l] = self.child[l].ctypes.data
        L = self.L
        sfx = "d" if dtype == np.float64 else "f"
        nwork = getattr(L, f"ora_mg_work_size_{sfx}")(C.byref(s))
        work = np.zeros(nwork, dtype=dtype)
        self.keep.append(work)
        s.work = work.ctypes.data
        return s

    def apply(self, x: np.ndarray, level: int = 0) -> np.ndarray:
        dtype = x.dtype
        y = np.zeros_like(x)
        op = self.op(level, dtype)
        fn = self.L.ora_helm_apply_d if dtype == np.float64 else self.L.ora_helm_apply_f
        fn(C.byref(op), ptr(x), ptr(y))
        return y

    def smooth(self, x_in, b, omega=0.8, level: int = 0):
        dtype = b.dtype
        op = self.op(level, dtype)
        out = np.zeros_like(b)
        work = np.zeros(b.size + 2 * self.nl, dtype=dtype)
        fn = self.L.ora_helm_smooth_d if dtype == np.float64 else self.L.ora_helm_smooth_f
        fn(C.byref(op), C.c_double(omega), None if x_in is None else ptr(x_in), ptr(b),
           ptr(out), ptr(work))
        return out

    def mg_apply(self, b: np.ndarray, **kw) -> np.ndarray:
        s = self.mg(b.dtype, **kw)
        x = np.zeros_like(b)
        fn = self.L.ora_mg_apply_d if b.dtype == np.float64 else self.L.ora_mg_apply_f
        fn(C.byref(s), ptr(b), ptr(x))
        return x

    def gcr_mg_solve(self, b, gcrk=10, r_tol=1e-8, max_iter=20, dtype=np.float64, **mgkw):
        L = self.L
        sfx = "d" if dtype == np.float64 else "f"
        b = np.ascontiguousarray(b, dtype=dtype)
        n = b.size
        op = self.op(0, dtype)
        mg = self.mg(dtype, **mgkw)
        x = np.zeros_like(b)
        work = np.zeros((2 * gcrk + 3) * n, dtype=dtype)
        info = SolveInfo()
        apply_cb = C.cast(getattr(L, f"ora_helm_apply_cb_{sfx}"), C.c_void_p)
        mg_cb = C.cast(getattr(L, f"ora_mg_apply_cb_{sfx}"), C.c_void_p)
        st = getattr(L, f"ora_gcr_solve_{sfx}")(
            C.c_long(n), apply_cb, C.byref(op), mg_cb, C.byref(mg), gcrk, C.c_double(r_tol),
            C.c_double(0.0), max_iter, 1, ptr(x), ptr(b), ptr(work), C.byref(info))
        return x, st, info

    def mixed_solve(self, b, tol=1e-8, max_outer=10, gcrk=10, inner_tol=1e-4,
                    inner_max_iter=2, **mgkw):
        L = self.L
        b = np.ascontiguousarray(b, dtype=np.float64)
        op = self.op(0, np.float64)
        mg = self.mg(np.float32, **mgkw)
        x = np.zeros_like(b)
        info = MixedInfo()
        st = L.ora_mixed_gcr_mg_solve(C.byref(op), C.byref(mg), ptr(b), ptr(x),
                                      C.c_double(tol), max_outer, gcrk, C.c_double(inner_tol),
                                      inner_max_iter, C.byref(info))
        return x, st, info


    def mixed_cg_col_solve(self, b, tol=1e-8, max_outer=10, inner_tol=1e-5, max_inner=200):
        """Refinement with an inner FP32 CG preconditioned by T'^{-1}."""
        L = self.L
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        info = MixedInfo()
        op64, op32 = self.op(0, np.float64), self.op(0, np.float32)
        st = L.ora_mixed_cg_col_solve(C.byref(op64), C.byref(op32), ptr(b), ptr(x),
                                      C.c_double(tol), max_outer, C.c_double(inner_tol),
                                      max_inner, C.byref(info))
        return x, st, info


class Lma(C.Structure):
    """ora_lma: an LMA operator (local_stencil(ncell*nlayers, ndf, ndf),
    1-based map(ndf, ncell))."""
    _fields_ = [("ncell", C.c_int), ("nlayers", C.c_int), ("ndf", C.c_int), ("undf", C.c_int),
                ("matrix", C.c_void_p), ("map", C.c_void_p)]


class DiagPrec(C.Structure):
    _fields_ = [("n", C.c_long), ("diag", C.c_void_p)]


class W0:
    """Oracle view of a W0 LMA problem (mass + stiffness): the matrix_vector
    apply over every cell, mm_diagonal and the Jacobi-preconditioned
    cg_solve, as the reference's mass_matrix_solver_alg composes them."""

    def __init__(self, prob, matrix=None, native: bool = False):
        self.L = lib(native)
        self.prob = prob
        self.A = np.ascontiguousarray(prob.matrix() if matrix is None else matrix,
                                      dtype=np.float64)
        self.map1 = np.ascontiguousarray(prob.map + 1, dtype=np.int32)
        self.lma = Lma(prob.ncell, prob.nlayers, self.map1.shape[1], prob.ndof,
                       self.A.ctypes.data, self.map1.ctypes.data)
        self.diag = np.zeros(prob.ndof)
        self.L.ora_lma_diagonal(C.byref(self.lma), ptr(self.diag))
        self.dprec = DiagPrec(prob.ndof, self.diag.ctypes.data)

    def apply(self, x: np.ndarray) -> np.ndarray:
        y = np.zeros(self.prob.ndof)
        self.L.ora_lma_apply_cb(C.byref(self.lma), ptr(np.ascontiguousarray(x)), ptr(y))
        return y

    def cg_solve(self, b, r_tol=1e-8, max_iter=2000):
        n = self.prob.ndof
        x = np.zeros(n)
        work = np.zeros(3 * n)
        info = SolveInfo()
        L = self.L
        st = L.ora_cg_solve_d(C.c_long(n), C.cast(L.ora_lma_apply_cb, C.c_void_p),
                              C.byref(self.lma), C.cast(L.ora_diag_prec_apply, C.c_void_p),
                              C.byref(self.dprec), C.c_double(r_tol), C.c_double(0.0), max_iter,
                              1, ptr(x), ptr(np.ascontiguousarray(b, dtype=np.float64)), ptr(work),
                              C.byref(info))
        return x, st, info


def _setup_signatures(L):
    L.ora_gcr_solve_d.argtypes = [C.c_long, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp,
                                  _dp, C.c_void_p]
    L.ora_gcr_solve_f.argtypes = [C.c_long, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, _fp, _fp,
                                  _fp, C.c_void_p]
    for nm in ("gmres", "fgmres"):
        getattr(L, f"ora_{nm}_solve_d").argtypes = [
            C.c_long, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
            C.c_double, C.c_int, C.c_int, _dp, _dp, _dp, C.c_void_p]
    L.ora_block_gcr_solve_d.argtypes = [C.c_long, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int,
                                        C.c_int, C.c_int, C.POINTER(C.c_int), _dp, _dp, _dp,
                                        C.c_void_p]
    L.ora_bicgstab_solve_d.argtypes = [C.c_long, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp, _dp,
                                       C.c_void_p]
    L.ora_cg_solve_d.argtypes = [C.c_long, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp, _dp,
                                 C.c_void_p]



MAX_W2_LEVELS = 8


class W2MgStruct(C.Structure):
    _fields_ = [("nlevels", C.c_int), ("n_pre", C.c_int), ("n_post", C.c_int),
                ("n_coarse", C.c_int), ("omega", C.c_double),
                ("op", Lma * MAX_W2_LEVELS), ("ncoarse", C.c_int * MAX_W2_LEVELS),
                ("cell_map", C.c_void_p * MAX_W2_LEVELS),
                ("sel_ew", C.c_void_p * MAX_W2_LEVELS), ("sel_ns", C.c_void_p * MAX_W2_LEVELS),
                ("work", C.c_void_p)]


class W2Multigrid:
    """Oracle view of a W2 hierarchy (problems.W2Hierarchy): flat W2 fields
    in the reference's dof order, each level's LMA operator with 1-based
    dofmaps, and the V-cycle of ora_w2mg_apply_cb as a preconditioner of
    the reference's cg_solve."""

    def __init__(self, hier, n_pre=2, n_post=2, n_coarse=8, omega=0.6, native: bool = False):
        L = lib(native)
        self.L, self.hier = L, hier
        self.keep = []
        s = W2MgStruct()
        nlev = len(hier.levels)
        s.nlevels, s.n_pre, s.n_post, s.n_coarse, s.omega = nlev, n_pre, n_post, n_coarse, omega
        for l, lev in enumerate(hier.levels):
            A = self._flat_matrix(lev)
            m1 = np.ascontiguousarray(lev.flat_map + 1, dtype=np.int32)
            self.keep += [A, m1]
            s.op[l] = Lma(lev.ncell, lev.nlayers, 6, lev.flat_ndof, A.ctypes.data, m1.ctypes.data)
        for l, cm in enumerate(hier.cell_maps):
            cmf = np.ascontiguousarray(np.asarray(cm).reshape(cm.shape[0], 4) + 1, dtype=np.int32)
            coarse = hier.levels[l + 1]
            ew = np.ascontiguousarray(coarse.ew, dtype=np.int32)
            ns = np.ascontiguousarray(coarse.ns, dtype=np.int32)
            self.keep += [cmf, ew, ns]
            s.ncoarse[l] = cm.shape[0]
            s.cell_map[l], s.sel_ew[l], s.sel_ns[l] = cmf.ctypes.data, ew.ctypes.data, ns.ctypes.data
        L.ora_w2mg_work_size.restype = C.c_long
        work = np.zeros(L.ora_w2mg_work_size(C.byref(s)))
        self.keep.append(work)
        s.work = work.ctypes.data
        L.ora_w2mg_setup(C.byref(s))
        self.s = s
        self.op0 = s.op[0]

    @staticmethod
    def _flat_matrix(lev):
        # local_stencil as stored: Fortran (ncell*nl, 6, 6) flattened
        return np.ascontiguousarray(lev.matrix, dtype=np.float64)

    def apply(self, x: np.ndarray) -> np.ndarray:
        y = np.zeros(self.hier.levels[0].flat_ndof)
        self.L.ora_lma_apply_cb(C.byref(self.op0), ptr(np.ascontiguousarray(x)), ptr(y))
        return y

    def vcycle(self, b: np.ndarray) -> np.ndarray:
        x = np.zeros_like(b)
        self.L.ora_w2mg_apply_cb(C.byref(self.s), ptr(np.ascontiguousarray(b)), ptr(x))
        return x

    def cg_solve(self, b, r_tol=1e-8, max_iter=500, multigrid=True):
        """cg_solve preconditioned by the V-cycle (or by the diagonal)."""
        L = self.L
        n = b.size
        x = np.zeros(n)
        work = np.zeros(3 * n)
        info = SolveInfo()
        if multigrid:
            prec, pctx = C.cast(L.ora_w2mg_apply_cb, C.c_void_p), C.byref(self.s)
        else:
            d = np.zeros(n)
            L.ora_lma_diagonal(C.byref(self.op0), ptr(d))
            self.keep.append(d)
            dp = DiagPrec(n, d.ctypes.data)
            self.keep.append(dp)
            prec, pctx = C.cast(L.ora_diag_prec_apply, C.c_void_p), C.byref(dp)
        st = L.ora_cg_solve_d(C.c_long(n), C.cast(L.ora_lma_apply_cb, C.c_void_p),
                              C.byref(self.op0), prec, pctx, C.c_double(r_tol), C.c_double(0.0),
                              max_iter, 1, ptr(x), ptr(np.ascontiguousarray(b, dtype=np.float64)),
                              ptr(work), C.byref(info))
        return x, st, info


def _w2_gcr(self, b, gcrk=10, r_tol=1e-8, max_iter=100, multigrid=True):
    """gcr_solve (right-preconditioned GCR(k)) with the V-cycle or the diagonal."""
    L = self.L
    n = b.size
    x = np.zeros(n)
    work = np.zeros((2 * gcrk + 3) * n)
    info = SolveInfo()
    if multigrid:
        prec, pctx = C.cast(L.ora_w2mg_apply_cb, C.c_void_p), C.byref(self.s)
    else:
        d = np.zeros(n)
        L.ora_lma_diagonal(C.byref(self.op0), ptr(d))
        dp = DiagPrec(n, d.ctypes.data)
        self.keep += [d, dp]
        prec, pctx = C.cast(L.ora_diag_prec_apply, C.c_void_p), C.byref(dp)
    st = L.ora_gcr_solve_d(C.c_long(n), C.cast(L.ora_lma_apply_cb, C.c_void_p),
                           C.byref(self.op0), prec, pctx, gcrk, C.c_double(r_tol),
                           C.c_double(0.0), max_iter, 1, ptr(x),
                           ptr(np.ascontiguousarray(b, dtype=np.float64)), ptr(work),
                           C.byref(info))
    return x, st, info


W2Multigrid.gcr_solve = _w2_gcr

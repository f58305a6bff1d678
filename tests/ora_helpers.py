"""Whole-mesh drivers of the oracle's per-cell kernels (test support).

Each helper loops over cells in order and calls the oracle's restatement
of one reference kernel with the reference's calling convention (1-based
dofmaps, Fortran-ordered arrays), as the PSy layer does.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from oracle.oracle import lib, ptr

_dp, _fp, _ip = C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int)


def _sfx(dtype):
    return "r_double" if np.dtype(dtype) == np.float64 else "r_single"


def _p(a):
    return ptr(np.ascontiguousarray(a))


def lma_apply(kind: str, ls, map1, map2, ncell, nl, x, y0=None, undf1=None):
    """matrix_vector / dg_matrix_vector / transpose_matrix_vector over all cells.

    ls: local_stencil flattened Fortran (ncell*nl, ndf1, ndf2) (transpose:
    (ncell*nl, ndf2, ndf1)); map1/map2: (ncell, ndf) 1-based first dofs."""
    L = lib()
    dt = x.dtype
    map1 = np.ascontiguousarray(map1, dtype=np.int32)
    map2 = np.ascontiguousarray(map2, dtype=np.int32)
    ndf1, ndf2 = map1.shape[1], map2.shape[1]
    undf1 = undf1 if undf1 is not None else (y0.size if y0 is not None else None)
    y = np.zeros(undf1, dtype=dt) if y0 is None else np.array(y0, dtype=dt)
    ls = np.ascontiguousarray(ls, dtype=dt)
    fn = getattr(L, f"ora_{kind}_code_{_sfx(dt)}")
    for cell in range(1, ncell + 1):
        fn(cell, nl, _p(y), _p(x), ncell * nl, _p(ls), ndf1, y.size,
           _p(map1[cell - 1]), ndf2, x.size, _p(map2[cell - 1]))
    return y


def mm_diagonal(ls, map1, ncell, nl, undf, dtype=np.float64):
    L = lib()
    d = np.zeros(undf, dtype=dtype)
    map1 = np.ascontiguousarray(map1, dtype=np.int32)
    ls = np.ascontiguousarray(ls, dtype=dtype)
    fn = getattr(L, f"ora_mm_diagonal_code_{_sfx(dtype)}")
    for cell in range(1, ncell + 1):
        fn(cell, nl, _p(d), ncell * nl, _p(ls), map1.shape[1], undf, _p(map1[cell - 1]))
    return d


def cma_app(cm, ncol, nrow, ncolumn, bw, alpha, beta, gm, gp, ind_to, ind_from, x, lhs0,
            nlev_to, nlev_from):
    """columnwise_op_app over all columns; fields column-contiguous."""
    L = lib()
    dt = x.dtype
    lhs = np.array(lhs0, dtype=dt)
    fn = getattr(L, f"ora_columnwise_op_app_code_{_sfx(dt)}")
    it = np.ascontiguousarray(ind_to, dtype=np.int32)
    iff = np.ascontiguousarray(ind_from, dtype=np.int32)
    cm = np.ascontiguousarray(cm, dtype=dt)
    for c in range(1, ncol + 1):
        m1 = np.array([(c - 1) * nlev_to + 1], dtype=np.int32)
        m2 = np.array([(c - 1) * nlev_from + 1], dtype=np.int32)
        fn(c, ncol, _p(lhs), _p(x), _p(cm), nrow, ncolumn, bw, alpha, beta, gm, gp, 1, lhs.size,
           _p(m1), _p(it), 1, x.size, _p(m2), _p(iff))
    return lhs


def cma_appinv(cm, ncol, nrow, ind, x, nlev):
    L = lib()
    dt = x.dtype
    lhs = np.zeros_like(x)
    fn = getattr(L, f"ora_columnwise_op_appinv_code_{_sfx(dt)}")
    it = np.ascontiguousarray(ind, dtype=np.int32)
    cm = np.ascontiguousarray(cm, dtype=dt)
    cp = np.zeros(nrow, dtype=dt)
    dp = np.zeros(nrow, dtype=dt)
    for c in range(1, ncol + 1):
        m = np.array([(c - 1) * nlev + 1], dtype=np.int32)
        fn(c, ncol, _p(lhs), _p(x), _p(cm), nrow, 3, 1, 1, 1, 1, 1, lhs.size, _p(m), _p(it),
           _p(cp), _p(dp))
    return lhs


def tri_solve(x, t0, tp, tm, ncol, nl):
    L = lib()
    dt = x.dtype
    y = np.zeros_like(x)
    fn = getattr(L, f"ora_tri_solve_code_{_sfx(dt)}")
    w1 = np.zeros(nl, dtype=dt)
    w2 = np.zeros(nl, dtype=dt)
    for c in range(ncol):
        m = np.array([c * nl + 1], dtype=np.int32)
        fn(nl, _p(y), _p(x), _p(t0), _p(tp), _p(tm), 1, x.size, _p(m), _p(w1), _p(w2))
    return y


def operator_tri_solve(matrix, x, ncell, nl):
    """matrix: (ncell*nl, 2, 2) Fortran-flattened; fields (nl+1) per cell."""
    L = lib()
    y = np.zeros_like(x)
    work = np.zeros(5 * (nl + 1))
    mat = np.ascontiguousarray(matrix, dtype=np.float64)
    for cell in range(1, ncell + 1):
        m = np.array([(cell - 1) * (nl + 1) + 1, (cell - 1) * (nl + 1) + 2], dtype=np.int32)
        L.ora_operator_tri_solve_code(cell, nl, _p(y), _p(x), ncell * nl, _p(mat), 2, x.size,
                                      _p(m), _p(work))
    return y


def restrict(mode: str, child, fine, nlev, weights=None):
    """child: (ncoarse, ny, nx) 0-based; scalar fields column-contiguous."""
    L = lib()
    dt = fine.dtype
    ncoarse, ny, nx = child.shape
    nfine = fine.size // nlev
    coarse = np.zeros(ncoarse * nlev, dtype=dt)
    work = np.zeros(nlev + 1, dtype=dt)
    map_fine = (np.arange(nfine, dtype=np.int32) * nlev + 1)
    ndf = 1 if nlev > 0 else 1
    top_nl = nlev  # W3 convention: nlayers = nlev, ndf = 1
    for C_ in range(ncoarse):
        cell_map = np.ascontiguousarray(child[C_].T + 1, dtype=np.int32)  # (nx, ny) Fortran
        cell_map_f = np.asfortranarray(cell_map).ravel(order="F")
        cmap = np.ascontiguousarray(cell_map_f, dtype=np.int32)
        mc = np.array([C_ * nlev + 1], dtype=np.int32)
        if mode == "unweighted":
            getattr(L, f"ora_restrict_scalar_unweighted_code_{_sfx(dt)}")(
                top_nl, _p(cmap), nx, ny, nfine, _p(coarse), _p(fine), coarse.size, _p(mc), ndf,
                fine.size, _p(map_fine), _p(work))
        elif mode == "weighted":
            getattr(L, f"ora_restrict_scalar_weighted_code_{_sfx(dt)}")(
                top_nl, _p(cmap), nx, ny, nfine, _p(coarse), _p(fine), _p(weights), coarse.size,
                _p(mc), ndf, fine.size, _p(map_fine), _p(work))
        else:
            getattr(L, f"ora_restrict_mass_w3_code_{_sfx(dt)}")(
                top_nl, _p(cmap), nx, ny, nfine, _p(coarse), _p(fine), coarse.size, _p(mc), ndf,
                fine.size, _p(map_fine), _p(work))
    return coarse


def prolong(child, fine0, coarse, nlev, weights=None):
    L = lib()
    dt = coarse.dtype
    ncoarse, ny, nx = child.shape
    fine = np.array(fine0, dtype=dt)
    nfine = fine.size // nlev
    map_fine = (np.arange(nfine, dtype=np.int32) * nlev + 1)
    for C_ in range(ncoarse):
        cmap = np.ascontiguousarray(np.asfortranarray(child[C_].T + 1).ravel(order="F"),
                                    dtype=np.int32)
        mc = np.array([C_ * nlev + 1], dtype=np.int32)
        if weights is None:
            getattr(L, f"ora_prolong_scalar_unweighted_code_{_sfx(dt)}")(
                nlev, _p(cmap), nx, ny, nfine, _p(fine), _p(coarse), 1, fine.size, _p(map_fine),
                coarse.size, _p(mc))
        else:
            getattr(L, f"ora_prolong_scalar_weighted_code_{_sfx(dt)}")(
                nlev, _p(cmap), nx, ny, nfine, _p(fine), _p(coarse), _p(weights), 1, fine.size,
                _p(map_fine), coarse.size, _p(mc))
    return fine


def w0_transfer(direction: str, child, fine_corners, coarse_corners, src, nl, dst0=None):
    """restrict_w0 / prolong_w0 over all coarse cells; W0 fields have nl+1
    dofs per vertex column (column-contiguous)."""
    L = lib()
    ncoarse, ny, nx = child.shape
    nlev = nl + 1
    nvf = int(fine_corners.max()) + 1
    nvc = int(coarse_corners.max()) + 1
    # 8-dof W0 maps: bottom SW,SE,NE,NW then top, 1-based
    mf = np.concatenate([fine_corners * nlev + 1, fine_corners * nlev + 2], axis=1).astype(np.int32)
    mc = np.concatenate([coarse_corners * nlev + 1, coarse_corners * nlev + 2], axis=1).astype(np.int32)
    mf = np.ascontiguousarray(mf)
    if direction == "restrict":
        out = np.zeros(nvc * nlev) if dst0 is None else np.array(dst0, dtype=np.float64)
    else:
        out = np.zeros(nvf * nlev) if dst0 is None else np.array(dst0, dtype=np.float64)
    for C_ in range(ncoarse):
        cmap = np.ascontiguousarray(np.asfortranarray(child[C_].T + 1).ravel(order="F"),
                                    dtype=np.int32)
        mcc = np.ascontiguousarray(mc[C_])
        if direction == "restrict":
            L.ora_restrict_w0_code(nl, _p(cmap), nx, ny, mf.shape[0], _p(out), _p(src), out.size,
                                   _p(mcc), 8, src.size, _p(mf))
        else:
            L.ora_prolong_w0_code(nl, _p(cmap), nx, ny, mf.shape[0], _p(out), _p(src), 8,
                                  out.size, _p(mf), src.size, _p(mcc))
    return out


# ---------------------------------------------------------------- CMA assembly
def _pF(a):
    """Pointer to a Fortran-ordered array (through a 1-D view, so writes land
    in the array)."""
    v = a.ravel(order="F")
    assert np.shares_memory(v, a)
    return ptr(v)


from lfric_core_b200.problems import banded_dofmap, cma_prod_size, cma_size  # noqa: E402,F401


def _cma_args(p):
    return [p["nrow"], p["ncol"], p["bw"], p["alpha"], p["beta"], p["gm"], p["gp"]]


def cma_asm(ls, p, ncell, nlayers, cb_to, cb_from, dtype=np.float64):
    """columnwise_op_asm over all cells; ls: (ncell*nlayers, ndf_to, ndf_from) F order."""
    L = lib()
    ls = np.asfortranarray(ls, dtype=dtype)
    cm = np.zeros((p["bw"], p["nrow"], ncell), dtype=dtype, order="F")
    fn = getattr(L, f"ora_columnwise_op_asm_code_{_sfx(dtype)}")
    cbt, cbf = np.asfortranarray(cb_to, np.int32), np.asfortranarray(cb_from, np.int32)
    for cell in range(1, ncell + 1):
        fn(cell, nlayers, ncell, ncell * nlayers, _pF(ls), _pF(cm), p["nrow"], p["ncol"],
           p["bw"], p["alpha"], p["beta"], p["gm"], p["gp"], cbt.shape[0],
           cbt.ctypes.data_as(_ip), cbf.shape[0], cbf.ctypes.data_as(_ip))
    return cm


def cma_mul(A, pa, B, pb, C0, pc, ncell):
    """C += A B over all cells (columnwise_op_mul)."""
    L = lib()
    dt = A.dtype
    out = np.array(C0, dtype=dt, order="F")
    fn = getattr(L, f"ora_columnwise_op_mul_code_{_sfx(dt)}")
    A, B = np.asfortranarray(A), np.asfortranarray(B)
    for cell in range(1, ncell + 1):
        fn(cell, ncell, _pF(A), pa["nrow"], pa["ncol"], pa["bw"], pa["alpha"], pa["beta"],
           pa["gm"], pa["gp"], _pF(B), pb["nrow"], pb["ncol"], pb["bw"], pb["alpha"],
           pb["beta"], pb["gm"], pb["gp"], _pF(out), pc["nrow"], pc["ncol"], pc["bw"],
           pc["alpha"], pc["beta"], pc["gm"], pc["gp"])
    return out


def cma_scaledadd(A, pa, B, pb, pc, ncell, alpha, beta):
    """C = alpha A + beta B over all cells (columnwise_op_scaledadd)."""
    L = lib()
    dt = A.dtype
    out = np.zeros((pc["bw"], pc["nrow"], ncell), dtype=dt, order="F")
    fn = getattr(L, f"ora_columnwise_op_scaledadd_code_{_sfx(dt)}")
    ct = C.c_double if dt == np.float64 else C.c_float
    A, B = np.asfortranarray(A), np.asfortranarray(B)
    for cell in range(1, ncell + 1):
        fn(cell, ncell, _pF(A), pa["nrow"], pa["ncol"], pa["bw"], pa["alpha"], pa["beta"],
           pa["gm"], pa["gp"], _pF(B), pb["nrow"], pb["ncol"], pb["bw"], pb["alpha"],
           pb["beta"], pb["gm"], pb["gp"], _pF(out), pc["nrow"], pc["ncol"], pc["bw"],
           pc["alpha"], pc["beta"], pc["gm"], pc["gp"], ct(alpha), ct(beta))
    return out


def cma_hmht(dh, m2h, p, ncell, nlayers, cb, dtype=np.float64):
    """columnwise_op_asm_diag_hmht over all cells."""
    L = lib()
    dh, m2h = np.asfortranarray(dh, dtype=dtype), np.asfortranarray(m2h, dtype=dtype)
    cm = np.zeros((p["bw"], p["nrow"], ncell), dtype=dtype, order="F")
    fn = getattr(L, f"ora_columnwise_op_asm_diag_hmht_code_{_sfx(dtype)}")
    cb = np.asfortranarray(cb, np.int32)
    for cell in range(1, ncell + 1):
        fn(cell, nlayers, ncell, ncell * nlayers, _pF(dh), _pF(m2h), _pF(cm), p["nrow"], p["bw"],
           p["alpha"], p["beta"], p["gm"], p["gp"], cb.shape[0], cb.ctypes.data_as(_ip),
           dh.shape[2])
    return cm


def cma_m2v(ls, p, ncell, nlayers, cb, dtype=np.float64):
    """columnwise_op_asm_m2v_lumped_inv over all cells."""
    L = lib()
    ls = np.asfortranarray(ls, dtype=dtype)
    cm = np.zeros((p["bw"], p["nrow"], ncell), dtype=dtype, order="F")
    fn = getattr(L, f"ora_columnwise_op_asm_m2v_lumped_inv_code_{_sfx(dtype)}")
    cb = np.asfortranarray(cb, np.int32)
    for cell in range(1, ncell + 1):
        fn(cell, nlayers, ncell, ncell * nlayers, _pF(ls), _pF(cm), p["nrow"], p["bw"],
           cb.shape[0], cb.ctypes.data_as(_ip))
    return cm


def cma_dense(cm, p, cell=0):
    """The dense nrow x ncol matrix of one column of a CMA operator."""
    D = np.zeros((p["nrow"], p["ncol"]))
    for i in range(1, p["nrow"] + 1):
        jm = int(np.ceil((p["alpha"] * i - p["gp"]) / p["beta"]))
        jp = int(np.floor((p["alpha"] * i + p["gm"]) / p["beta"]))
        for j in range(max(1, jm), min(p["ncol"], jp) + 1):
            D[i - 1, j - 1] = cm[j - jm, i - 1, cell]
    return D


# ------------------------------------------------------- W2 intergrid drivers
def _cellmap(nx, ny):
    """cell_map(x, y) = x + (y-1) nx of the reference tests, Fortran order."""
    return np.asfortranarray(np.array([[x + (y - 1) * nx for y in range(1, ny + 1)]
                                       for x in range(1, nx + 1)], dtype=np.int32))


def w2_restrict(kind, nl, nx, ny, map_f, map_c, fine, undf_c, sel_ew=2, sel_ns=2,
                dtype=np.float64, cell_map=None):
    """restrict_w2 / restrict_w2h / restrict_w2v over one coarse cell; maps
    1-based, map_f (ncell_f, ndf) and map_c (ndf,)."""
    L = lib()
    cm = _cellmap(nx, ny) if cell_map is None else np.asfortranarray(cell_map, np.int32)
    mf = np.ascontiguousarray(map_f, dtype=np.int32)      # (ncell, ndf) == Fortran (ndf, ncell)
    mc = np.ascontiguousarray(map_c, dtype=np.int32)
    fine = np.ascontiguousarray(fine, dtype=dtype)
    coarse = np.zeros(undf_c, dtype=dtype)
    work = np.zeros(nl + 1, dtype=dtype)
    sfx = _sfx(dtype)
    ip = lambda a: a.ctypes.data_as(_ip)
    if kind == "w2v":
        getattr(L, f"ora_restrict_w2v_code_{sfx}")(nl, ip(cm), nx, ny, nx * ny, ptr(coarse),
                                                   ptr(fine), ip(mc), mf.shape[1], ip(mf),
                                                   ptr(work))
    else:
        ew, ns = np.array([sel_ew], np.int32), np.array([sel_ns], np.int32)
        one = np.array([1], np.int32)
        getattr(L, f"ora_restrict_w2_code_{sfx}")(nl, ip(cm), nx, ny, nx * ny, ptr(coarse),
                                                  ptr(fine), ip(ew), ip(ns), ip(mc),
                                                  mf.shape[1], ip(mf), ip(one),
                                                  1 if kind == "w2" else 0, ptr(work))
    return coarse


def w2_weights(nl, nx, ny, map_f, undf_f, w0=None, cell_map=None):
    L = lib()
    cm = _cellmap(nx, ny) if cell_map is None else np.asfortranarray(cell_map, np.int32)
    mf = np.ascontiguousarray(map_f, dtype=np.int32)
    w = np.zeros(undf_f) if w0 is None else np.array(w0, dtype=np.float64)
    L.ora_weights_prolong_w2_code(nl, cm.ctypes.data_as(_ip), nx, ny, nx * ny, ptr(w),
                                  mf.shape[1], mf.ctypes.data_as(_ip))
    return w


def w2_prolong(nl, nx, ny, map_f, map_c, coarse, weights, fine0, cell_map=None):
    L = lib()
    cm = _cellmap(nx, ny) if cell_map is None else np.asfortranarray(cell_map, np.int32)
    mf = np.ascontiguousarray(map_f, dtype=np.int32)
    mc = np.ascontiguousarray(map_c, dtype=np.int32)
    fine = np.array(fine0, dtype=np.float64)
    L.ora_prolong_w2_code(nl, cm.ctypes.data_as(_ip), nx, ny, nx * ny, ptr(fine),
                          ptr(np.ascontiguousarray(coarse, np.float64)),
                          ptr(np.ascontiguousarray(weights, np.float64)), mf.shape[1],
                          mf.ctypes.data_as(_ip), mc.ctypes.data_as(_ip))
    return fine

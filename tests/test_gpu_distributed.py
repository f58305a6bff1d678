"""The partitioned solve's device side on one GPU: the halo plumbing entry
points (pack, unpack, zero columns) and the rank-local GCR with the column
preconditioner through the C ABI, against the oracle's single-domain GCR.
(More ranks need more GPUs; the partition, halo exchange and global sums
are covered on CPU ranks in test_distributed.py.)"""
import ctypes as C

import numpy as np
import pytest

from lfric_core_b200 import api
from lfric_core_b200.api import R_DOUBLE, Field
from lfric_core_b200.problems import helmholtz_problem

pytestmark = pytest.mark.gpu


def test_halo_pack_unpack_zero(ctx):
    import torch
    ncol, nl = 300, 7
    rng = np.random.default_rng(2)
    v = rng.standard_normal(ncol * nl)
    F = Field(ctx, R_DOUBLE, ncol, nl).import_(v)
    cols = np.array([5, 0, 299, 17, 18], dtype=np.int32)
    dcols = torch.tensor(cols, device="cuda")
    buf = torch.empty(cols.size * nl, dtype=torch.float64, device="cuda")
    ip = C.cast(dcols.data_ptr(), C.POINTER(C.c_int))
    ctx.check(ctx.lib.lfg_field_pack_columns(F.h, ip, int(cols.size),
                                             C.c_void_p(buf.data_ptr())))
    ctx.synchronize()
    vv = v.reshape(ncol, nl)
    assert np.array_equal(buf.cpu().numpy().reshape(nl, cols.size), vv[cols].T)
    G = Field(ctx, R_DOUBLE, ncol, nl)
    ctx.check(ctx.lib.lfg_field_unpack_columns(G.h, ip, int(cols.size),
                                               C.c_void_p(buf.data_ptr())))
    g = G.export().reshape(ncol, nl)
    assert np.array_equal(g[cols], vv[cols])
    assert not np.any(np.delete(g, cols, axis=0))
    ctx.check(ctx.lib.lfg_field_zero_columns(F.h, 290, 10))
    f = F.export().reshape(ncol, nl)
    assert not np.any(f[290:]) and np.array_equal(f[:290], vv[:290])
    assert ctx.lib.lfg_field_zero_columns(F.h, 295, 10) == 3      # LFG_ERR_ARG


def test_rank_local_gcr_matches_the_oracle(ctx):
    import ctypes
    from lfric_core_b200.distributed import LibrarySpace, gcr_solve
    from oracle.oracle import Helmholtz as OraHelm, SolveInfo, ptr
    p = helmholtz_problem(12, 8, seed=23, mg_levels=1)
    sp = LibrarySpace(ctx, p, rank=0, world=1)
    b = sp.field_from_global(p.rhs)
    x = sp.new()
    res = gcr_solve(sp, x, b, gcrk=10, r_tol=1e-9, max_iter=40)
    ora = OraHelm(p)
    L = ora.L
    op = ora.op(0)
    mg = ora.mg(np.float64, n_pre=0, n_post=0, n_coarse=1, omega=1.0, nlevels=1)
    n = p.ndof
    x1 = np.zeros(n)
    work = np.zeros(23 * n)
    info = SolveInfo()
    st = L.ora_gcr_solve_d(ctypes.c_long(n), ctypes.cast(L.ora_helm_apply_cb_d, ctypes.c_void_p),
                           ctypes.byref(op), ctypes.cast(L.ora_mg_apply_cb_d, ctypes.c_void_p),
                           ctypes.byref(mg), 10, ctypes.c_double(1e-9), ctypes.c_double(0.0), 40,
                           1, ptr(x1), ptr(np.ascontiguousarray(p.rhs)), ptr(work),
                           ctypes.byref(info))
    assert res.status == st == 0
    assert res.iterations == info.iterations
    xg = sp.owned_values(x).ravel()
    assert np.linalg.norm(xg - x1) / np.linalg.norm(x1) < 1e-12

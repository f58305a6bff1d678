"""The partitioned solve's device side on one GPU: the halo plumbing entry
points (pack, unpack, zero columns), the rank-local GCR with the column
preconditioner through the C ABI against the oracle's single-domain GCR,
and GCR with the partitioned multigrid V-cycle.  Several ranks of the
multigrid run here as one process on the one device: each rank's
hierarchy is its own set of library objects, and the halo exchange copies
columns between the ranks' fields on the device, ordered by the host (no
kernel waits on another).  The partition, the exchange over
torch.distributed and the global sums are covered on CPU ranks in
test_distributed.py."""
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


MG = dict(n_pre=2, n_post=2, n_coarse=8, omega=0.8)


class GroupLevels:
    """mg_vcycle's level interface over several ranks' LibraryLevels in one
    process: fields are lists (one per rank), every step runs rank by rank,
    and the halo exchange packs each sender's columns and unpacks them into
    the receiver's halo on the device."""

    def __init__(self, ranks):
        self.r, self.nlevels = ranks, ranks[0].nlevels

    def smooth(self, l, omega, x_in, b, x_out):
        for i, lv in enumerate(self.r):
            lv.smooth(l, omega, None if x_in is None else x_in[i], b[i], x_out[i])

    def copy(self, l, dst, src):
        for d, s_ in zip(dst, src):
            d.copy(s_)

    def set0(self, l, f):
        for g in f:
            g.set_scalar(0.0)

    def exchange(self, l, f):
        for p, lv in enumerate(self.r):
            for q, cols in sorted(lv.plans[l].recv.items()):
                src = self.r[q]
                buf = src.columns.pack(f[q], src.plans[l].send[p])
                lv.columns.unpack(f[p], cols, buf)

    def resid_restrict(self, l, x, b, bc):
        for i, lv in enumerate(self.r):
            lv.resid_restrict(l, x[i], b[i], bc[i])

    def prolong_add(self, l, fine, coarse):
        for i, lv in enumerate(self.r):
            lv.prolong_add(l, fine[i], coarse[i])

    def work(self, l):
        w = [lv.work(l) for lv in self.r]
        return tuple(None if w[0][j] is None else [wi[j] for wi in w] for j in range(3))


class GroupSpace:
    """gcr_solve's space over several ranks' LibraryMgSpaces in one process:
    vectors are lists, inner products the sum of the ranks' shares."""

    def __init__(self, spaces):
        self.s = spaces
        self.levels = GroupLevels([sp.levels for sp in spaces])

    def new(self):
        return [sp.new() for sp in self.s]

    def set(self, v, a):
        for f in v:
            f.set_scalar(a)

    def copy(self, d, s_):
        for a, b in zip(d, s_):
            a.copy(b)

    def axpy(self, y, a, x):
        for u, v in zip(y, x):
            u.axpy(a, v)

    def scale(self, v, a):
        for f in v:
            f.scale(a)

    def dot(self, u, v):
        return float(sum(a.dot(b) for a, b in zip(u, v)))

    def norm(self, v):
        return float(np.sqrt(self.dot(v, v)))

    def apply(self, x, y):
        self.levels.exchange(0, x)
        for sp, a, b in zip(self.s, x, y):
            sp.op.apply(b, a)
            sp.zero_halo(a)
            sp.zero_halo(b)

    def prec(self, x, y):
        from lfric_core_b200.distributed import mg_vcycle
        mg_vcycle(self.levels, x, y, **MG)
        for sp, f in zip(self.s, y):
            sp.zero_halo(f)


@pytest.mark.parametrize("world", [1, 2, 3])
def test_partitioned_multigrid_gcr_matches_the_oracle(ctx, world):
    """GCR(10) with the partitioned 3-level V-cycle (C12 -> C6 -> C3 x 8,
    nested ownership; the coarse operators from the library's Galerkin
    coarsening of each rank's local operator) takes the single-domain
    oracle GCR + multigrid's iteration count and reaches its solution."""
    from lfric_core_b200.distributed import LibraryMgSpace, gcr_solve
    from oracle.oracle import Helmholtz as OraHelm
    p = helmholtz_problem(12, 8, seed=23, mg_levels=3)
    x1, st1, info = OraHelm(p).gcr_mg_solve(p.rhs, gcrk=10, r_tol=1e-9, max_iter=40, **MG)
    assert st1 == 0
    spaces = [LibraryMgSpace(ctx, p, r, world, exchange=False, **MG) for r in range(world)]
    sp = GroupSpace(spaces)
    b = [s_.field_from_global(p.rhs) for s_ in spaces]
    x = sp.new()
    sp.set(x, 0.0)
    res = gcr_solve(sp, x, b, gcrk=10, r_tol=1e-9, max_iter=40)
    assert res.status == 0
    assert res.iterations == info.iterations
    xg = np.zeros((p.ncol, p.nlayers))
    for s_, f in zip(spaces, x):
        xg[s_.plan.owned] = s_.owned_values(f)
    xg = xg.ravel()
    assert np.linalg.norm(xg - x1) / np.linalg.norm(x1) < 1e-10

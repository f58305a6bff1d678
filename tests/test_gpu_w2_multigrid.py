"""Vector-space (W2) multigrid on the device against the oracle.

A W2 hierarchy on the cubed sphere (C24/C12/C6 x 4 layers, rediscretised
RT0 mass + divergence-divergence operator on every level) is held in the
library's column layout; its transfers, operator applies, the V-cycle and
GCR(10) preconditioned by the V-cycle are compared with the oracle, which
works on the same spaces in the reference's flat dof order."""
import numpy as np
import pytest

from lfric_core_b200 import api
from lfric_core_b200.api import R_DOUBLE, Field
from lfric_core_b200.problems import w2_hierarchy
from oracle.oracle import W2Multigrid

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def w2(ctx):
    H = w2_hierarchy(24, 4, 3, seed=1, top=4e5, tau=1e9, radius=6.371e5)
    return H, api.W2System(ctx, H), W2Multigrid(H, omega=0.6)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_w2_column_transfers_match_the_oracle(ctx, w2):
    import ctypes as C
    from oracle.oracle import lib, ptr
    H, S, ora = w2
    fine, coarse = H.levels[0], H.levels[1]
    rng = np.random.default_rng(3)
    v = rng.standard_normal(fine.flat_ndof)
    F = S.field(v, 0)
    Cc = S.field(None, 1)
    S.maps[0].restrict(api.W2_FULL, Cc, F)
    L = lib()
    cm = np.ascontiguousarray(H.cell_maps[0].reshape(-1, 4) + 1, dtype=np.int32)
    mf = np.ascontiguousarray(fine.flat_map + 1, dtype=np.int32)
    mc = np.ascontiguousarray(coarse.flat_map + 1, dtype=np.int32)
    ew = np.ascontiguousarray(coarse.ew, dtype=np.int32)
    ns = np.ascontiguousarray(coarse.ns, dtype=np.int32)
    want = np.zeros(coarse.flat_ndof)
    work = np.zeros(fine.nlayers + 1)
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    for c in range(coarse.ncell):
        one = np.array([c + 1], dtype=np.int32)
        L.ora_restrict_w2_code_r_double(fine.nlayers, ip(cm[c]), 2, 2, 4, ptr(want), ptr(v),
                                        ip(ew), ip(ns), ip(mc[c]), 6, ip(mf), ip(one), 1,
                                        ptr(work))
    assert np.array_equal(S.flat(Cc, 1), want)
    # prolongation of a coarse field with the weights of weights_prolong_w2
    u = rng.standard_normal(coarse.flat_ndof)
    Uc, Wf, Pf = S.field(u, 1), S.field(None, 0), S.field(None, 0)
    S.maps[0].prolong_weights(Wf)
    S.maps[0].prolong(Pf, Uc, Wf)
    w = np.zeros(fine.flat_ndof)
    p = np.zeros(fine.flat_ndof)
    for c in range(coarse.ncell):
        L.ora_weights_prolong_w2_code(fine.nlayers, ip(cm[c]), 2, 2, 4, ptr(w), 6, ip(mf))
    for c in range(coarse.ncell):
        L.ora_prolong_w2_code(fine.nlayers, ip(cm[c]), 2, 2, 4, ptr(p), ptr(u), ptr(w), 6,
                              ip(mf), ip(mc[c]))
    assert np.array_equal(S.flat(Wf, 0), w)
    assert rel(S.flat(Pf, 0), p) < 1e-15


def test_w2_operator_and_vcycle_match_the_oracle(ctx, w2):
    H, S, ora = w2
    rng = np.random.default_rng(4)
    x = rng.standard_normal(H.levels[0].flat_ndof)
    X, Y = S.field(x), S.field()
    S.ops[0].apply(api.LMA_WRITE, Y, X)
    assert rel(S.flat(Y), ora.apply(x)) < 1e-13
    Z = S.field()
    S.prec.apply(X, Z)
    assert rel(S.flat(Z), ora.vcycle(x)) < 1e-12


def test_w2_multigrid_gcr_parity(ctx, w2):
    """GCR(10) preconditioned by the W2 V-cycle: the oracle's iteration count
    and solution (1e-12); fewer iterations than with the diagonal."""
    H, S, ora = w2
    x_ref, st, info = ora.gcr_solve(H.rhs, gcrk=10, r_tol=1e-8, max_iter=100)
    sol = api.IterativeSolver(api.LinearOperator.from_lma(S.ops[0]), S.prec, S.field(), "gcr",
                              r_tol=1e-8, max_iter=100, gcrk=10)
    B, X = S.field(H.rhs), S.field()
    out = sol.apply(X, B)
    assert out.status == st == 0
    assert out.iterations == info.iterations
    assert rel(S.flat(X), x_ref) < 1e-12
    _, _, info_d = ora.gcr_solve(H.rhs, gcrk=10, r_tol=1e-8, max_iter=400, multigrid=False)
    assert out.iterations < info_d.iterations

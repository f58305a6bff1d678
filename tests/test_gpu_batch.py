"""Batched persistent solves (lfg_batch_*) against the oracle's
ora_mixed_cg_col_solve, problem by problem, and the full batched workload
(64 right-hand sides on C48 x 30 plus 32 uneven problems)."""
import numpy as np
import pytest

from lfric_core_b200 import api
from lfric_core_b200.api import R_DOUBLE, BatchedHelmholtz, Helmholtz, Mesh
from lfric_core_b200.problems import batch_workload
from oracle.oracle import Helmholtz as OraHelm

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def build(ctx, wl):
    ops = []
    for p in wl.operators:
        mesh = Mesh(ctx, p.links)
        ops.append(Helmholtz(ctx, R_DOUBLE, mesh, p.nlayers, p.cm, p.hf))
    return ops


def small_workload():
    return batch_workload(seed=5, n_rhs=3, n_shared=8, l_shared=10, n_uneven=5,
                          n_range=(3, 16), l_range=(2, 24))


def true_residual(ora, x, b):
    r = b - ora.apply(x)
    return np.linalg.norm(r) / np.linalg.norm(b)


def test_batch_parity_small(ctx):
    wl = small_workload()
    ops = build(ctx, wl)
    B = BatchedHelmholtz(ctx, [ops[j] for j in wl.problem_op])
    for i, b in enumerate(wl.rhs):
        B.rhs[i].import_(b)
    assert B.solve() == 0
    oras = [OraHelm(p) for p in wl.operators]
    for i, b in enumerate(wl.rhs):
        ora = oras[wl.problem_op[i]]
        x_ref, st, info = ora.mixed_cg_col_solve(b)
        res = B.result(i)
        x = B.sol[i].export()
        assert res.status == st == 0
        assert res.outer_iterations == info.outer_iterations
        # FP32 inner arithmetic rounds differently from the oracle's; an inner
        # stopping test may flip by one iteration
        assert abs(res.inner_iterations - info.inner_iterations) <= res.outer_iterations
        assert res.rel_residual <= 1e-8
        assert true_residual(ora, x, b) <= 1e-8
        assert rel(x, x_ref) < 1e-6


def test_batch_replay_is_deterministic(ctx):
    wl = small_workload()
    ops = build(ctx, wl)
    B = BatchedHelmholtz(ctx, [ops[j] for j in wl.problem_op])
    for i, b in enumerate(wl.rhs):
        B.rhs[i].import_(b)
    B.solve()
    first = [B.sol[i].export() for i in range(len(B))]
    r1 = [B.result(i) for i in range(len(B))]
    B.solve()
    for i in range(len(B)):
        assert np.array_equal(B.sol[i].export(), first[i])
        assert B.result(i) == r1[i]


@pytest.mark.parametrize("tc,bpsm,graph", [(64, 1, True), (128, 2, False), (256, 1, True)])
def test_batch_launch_shapes_agree(ctx, tc, bpsm, graph):
    wl = small_workload()
    ops = build(ctx, wl)
    B = BatchedHelmholtz(ctx, [ops[j] for j in wl.problem_op], tile_cols=tc, blocks_per_sm=bpsm,
                         use_graph=graph)
    for i, b in enumerate(wl.rhs):
        B.rhs[i].import_(b)
    assert B.solve() == 0
    t = B.tuning()
    assert (t["tile_cols"], t["blocks_per_sm"]) == (tc, bpsm)
    assert t["phases"] > 0
    oras = [OraHelm(p) for p in wl.operators]
    for i, b in enumerate(wl.rhs):
        assert true_residual(oras[wl.problem_op[i]], B.sol[i].export(), b) <= 1e-8


def test_batch_zero_rhs_and_not_converged(ctx):
    wl = small_workload()
    ops = build(ctx, wl)
    B = BatchedHelmholtz(ctx, [ops[j] for j in wl.problem_op], tol=1e-14, max_outer=1)
    for i, b in enumerate(wl.rhs):
        B.rhs[i].import_(np.zeros_like(b) if i == 1 else b)
    nf = B.solve()
    assert nf == len(B) - 1
    z = B.result(1)
    assert z.status == api.OK and z.outer_iterations == 0
    assert not np.any(B.sol[1].export())
    for i in (0, 2, 3):
        r = B.result(i)
        assert r.status == api.NOT_CONVERGED and r.outer_iterations == 1


def test_batch_barrier_wait_runs_out(ctx):
    """The grid barrier waits for one CTA more than launched: every wait
    gives up after spin_limit spins, the solve reports LFG_ERR_STATE and the
    context stays usable."""
    wl = small_workload()
    ops = build(ctx, wl)
    B = BatchedHelmholtz(ctx, [ops[j] for j in wl.problem_op], spin_limit=2000,
                         tile_cols=128, blocks_per_sm=1)
    for i, b in enumerate(wl.rhs):
        B.rhs[i].import_(b)
    B.test_stall(1)
    with pytest.raises(api.LfgError) as e:
        B.solve()
    assert e.value.status == 6
    B.test_stall(0)
    assert B.solve() == 0


def test_batch_full_workload(ctx):
    """64 seeded right-hand sides on C48 x 30 plus 32 problems with n in
    12..96 and 10..70 levels: all reach 1e-8 in FP64 (checked by the
    oracle's FP64 operator), two match the oracle's own solve."""
    wl = batch_workload()
    ops = build(ctx, wl)
    B = BatchedHelmholtz(ctx, [ops[j] for j in wl.problem_op])
    for i, b in enumerate(wl.rhs):
        B.rhs[i].import_(b)
    assert B.solve() == 0
    oras = {}
    for i, b in enumerate(wl.rhs):
        j = wl.problem_op[i]
        if j not in oras:
            oras[j] = OraHelm(wl.operators[j])
        assert true_residual(oras[j], B.sol[i].export(), b) <= 1e-8, i
    for i in (5, 64 + int(np.argmin([wl.operators[j].ncol for j in wl.problem_op[64:]]))):
        j = wl.problem_op[i]
        x_ref, st, info = oras[j].mixed_cg_col_solve(wl.rhs[i])
        assert st == 0
        assert B.result(i).outer_iterations == info.outer_iterations
        assert rel(B.sol[i].export(), x_ref) < 1e-6

"""The structured panel kernels against the per-column kernels and the oracle.

On a cubed-sphere mesh numbered panel by panel, row-major, the Helmholtz
apply, residual, sweep right-hand side and fused residual + restriction take
their interior neighbours by arithmetic and read V adjacent columns per
thread; the panel borders run the per-column code through the links table.
Fields that do not start on a 16-byte boundary (views into a larger
allocation) take the per-column kernels for every column, so the two forms
are compared on the same operator: they perform the same operations in the
same order and must agree bit for bit.  Both are also compared with the
oracle.
"""
import numpy as np
import pytest

from lfric_core_b200 import api
from lfric_core_b200.api import R_DOUBLE, R_SINGLE, Field
from lfric_core_b200.problems import helmholtz_problem
from oracle.oracle import Helmholtz as OraHelm

pytestmark = pytest.mark.gpu


def _view(ctx, kind, ncol, nl, keep):
    """A field view 1 element past a 16-byte boundary (per-column kernels)."""
    base = Field(ctx, kind, ncol * nl + 4, 1)
    keep.append(base)
    return Field(ctx, kind, ncol, nl, device_ptr=base.device_ptr() + kind, keep=[base])


@pytest.mark.parametrize("kind", [R_SINGLE, R_DOUBLE])
# C176 x 64 is large enough for the panel form of the fused residual +
# restriction (at least 8 waves of coarse columns x levels on 148 SMs); the
# smaller meshes take the lane-per-child kernel for it in both layouts
@pytest.mark.parametrize("n,nl", [(12, 5), (48, 9), (176, 64)])
def test_panel_kernels_equal_per_column_kernels(ctx, kind, n, nl):
    p = helmholtz_problem(n, nl, seed=41, mg_levels=2)
    mesh, cmesh = api.Mesh(ctx, p.links), api.Mesh(ctx, p.mg_links[0])
    H = api.Helmholtz(ctx, kind, mesh, nl, p.cm, p.hf)
    ig = api.Intergrid(ctx, p.mg_child[0], p.ncol)
    nc = p.mg_child[0].shape[0]
    rng = np.random.default_rng(7)
    xh, bh = rng.standard_normal(p.ndof), rng.standard_normal(p.ndof)
    keep = []
    xa, ba, ya = H.field(xh), H.field(bh), H.field()
    xu, bu, yu = (_view(ctx, kind, p.ncol, nl, keep) for _ in range(3))
    xu.import_(xh)
    bu.import_(bh)
    ca, cu = Field(ctx, kind, nc, nl), Field(ctx, kind, nc, nl)
    ora = OraHelm(p)
    tol = 1e-12 if kind == R_DOUBLE else 2e-5
    dt = np.float64 if kind == R_DOUBLE else np.float32
    # y = A x
    H.apply(ya, xa)
    H.apply(yu, xu)
    a, u = ya.export(), yu.export()
    assert np.array_equal(a, u)
    ref = ora.apply(xh.astype(dt).astype(np.float64))
    assert np.linalg.norm(a - ref) / np.linalg.norm(ref) < tol
    # r = b + H_off x
    H.sweep_rhs(xa, ba, ya)
    H.sweep_rhs(xu, bu, yu)
    assert np.array_equal(ya.export(), yu.export())
    # b - A x summed over each coarse cell's children
    H.residual_restrict(ig, xa, ba, ca)
    H.residual_restrict(ig, xu, bu, cu)
    a, u = ca.export(), cu.export()
    assert np.array_equal(a, u)
    r = bh.astype(dt).astype(np.float64) - ref
    want = np.zeros(nc * nl)
    child = np.asarray(p.mg_child[0]).reshape(nc, -1)
    rr = r.reshape(p.ncol, nl)
    for q in range(child.shape[1]):
        want += rr[child[:, q]].ravel()
    assert np.linalg.norm(a - want) / np.linalg.norm(want) < 10 * tol
    ctx.synchronize()


def test_panel_apply_with_inner_product(ctx):
    """The GCR step's fused apply + inner product through the panel kernel
    and through the per-column kernel give the same bits."""
    p = helmholtz_problem(24, 7, seed=43, mg_levels=2)
    S = api.HelmholtzSystem(ctx, p, fp64=True, mixed=False)
    r1 = S.solve_fp64(p.rhs)
    x1 = S.solution()
    ora = OraHelm(p)
    x_ref, st, info = ora.gcr_mg_solve(p.rhs, gcrk=10, r_tol=1e-8, max_iter=20)
    assert r1.status == st == 0 and r1.iterations == info.iterations
    assert np.linalg.norm(x1 - x_ref) / np.linalg.norm(x_ref) < 1e-12


@pytest.mark.parametrize("nl", [1, 3, 70, 80])
def test_sweep_forms_give_the_same_bits(ctx, nl):
    """On a structured FP32 mesh with many columns (C96) the sweep from a
    guess runs as the panel right-hand side kernel and the TMA-staged
    substitution; fields off a 16-byte boundary take the per-column
    right-hand side and substitution kernels.  Both give the same bits and
    match the oracle."""
    p = helmholtz_problem(96, nl, seed=45, mg_levels=1)
    H = api.Helmholtz(ctx, R_SINGLE, api.Mesh(ctx, p.links), nl, p.cm, p.hf)
    rng = np.random.default_rng(46)
    xh = rng.standard_normal(p.ndof).astype(np.float32)
    bh = rng.standard_normal(p.ndof).astype(np.float32)
    keep = []
    xa, ba, ya = H.field(xh), H.field(bh), H.field()
    xu, bu, yu = (_view(ctx, R_SINGLE, p.ncol, nl, keep) for _ in range(3))
    xu.import_(xh)
    bu.import_(bh)
    H.smooth(0.8, xa, ba, ya)
    H.smooth(0.8, xu, bu, yu)
    a = ya.export()
    assert np.array_equal(a, yu.export())
    ref = OraHelm(p).smooth(xh.astype(np.float64), bh.astype(np.float64), 0.8)
    assert np.linalg.norm(a - ref) / np.linalg.norm(ref) < 2e-5
    ctx.synchronize()   # no bounded wait ran out

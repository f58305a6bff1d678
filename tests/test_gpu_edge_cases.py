"""Edge cases of the device path against the oracle: one- and two-level
columns, columns taller than the register/shared-memory tiles (the fallback
kernels), zero right-hand sides (the solvers' early return), ragged sizes
(vector tails, odd column counts) and unaligned field views (the scalar
path of the packed vector kernels)."""
import numpy as np
import pytest

from lfric_core_b200 import api
from lfric_core_b200.api import R_DOUBLE, R_SINGLE, ColumnwiseOperator, Field, field_from
from lfric_core_b200.problems import helmholtz_problem
from oracle.oracle import Helmholtz as OraHelm
from tests import ora_helpers as oh

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.mark.parametrize("n,nl,kind", [(8, 1, R_DOUBLE), (8, 2, R_SINGLE), (8, 150, R_DOUBLE),
                                       (96, 150, R_SINGLE), (96, 1, R_SINGLE),
                                       (96, 100, R_SINGLE), (96, 100, R_DOUBLE)])
def test_helmholtz_column_heights(ctx, n, nl, kind):
    """apply and both sweep forms for columns of 1 to 150 levels, on a mesh
    with few columns (segmented sweep, or its per-column fallback above 384
    levels) and on C96: the TMA substitution with d' in registers up to 80
    levels (FP32 and FP64), with d' in shared memory for 81-128 FP32
    levels, one thread per column above that and for taller FP64 columns."""
    p = helmholtz_problem(n, nl, seed=21, mg_levels=1)
    dt = np.float64 if kind == R_DOUBLE else np.float32
    ora = OraHelm(p)
    H = api.Helmholtz(ctx, kind, api.Mesh(ctx, p.links), nl, p.cm, p.hf)
    rng = np.random.default_rng(22)
    x = rng.standard_normal(p.ndof).astype(dt)
    b = rng.standard_normal(p.ndof).astype(dt)
    X, B, Y = H.field(x), H.field(b), H.field()
    tol = 1e-12 if kind == R_DOUBLE else 2e-6
    H.apply(Y, X)
    assert rel(Y.export(np.float64), ora.apply(x.astype(np.float64))) < tol
    H.smooth(0.8, None, B, Y)
    assert rel(Y.export(np.float64), ora.smooth(None, b, 0.8)) < tol
    H.smooth(0.8, X, B, Y)
    assert rel(Y.export(np.float64), ora.smooth(x, b, 0.8)) < tol
    ctx.synchronize()


@pytest.mark.parametrize("n", [8, 96])
def test_helmholtz_nonsymmetric_couplings(ctx, n):
    """Couplings whose two sides of a face differ are read per side (the
    kernels read each face through one designated side only when every face
    agrees bit for bit): apply and both sweep forms against the oracle, on
    the segmented (C8) and the element-parallel + TMA (C96) sweep paths."""
    p = helmholtz_problem(n, 10, seed=27, mg_levels=1)
    hf = p.hf.copy().reshape(-1, 4)
    hf[5, 0] *= 1.5                        # one side of one face
    p.hf = hf.ravel()
    ora = OraHelm(p)
    H = api.Helmholtz(ctx, R_DOUBLE, api.Mesh(ctx, p.links), p.nlayers, p.cm, p.hf)
    rng = np.random.default_rng(28)
    x, b = rng.standard_normal(p.ndof), rng.standard_normal(p.ndof)
    X, B, Y = H.field(x), H.field(b), H.field()
    H.apply(Y, X)
    assert rel(Y.export(), ora.apply(x)) < 1e-12
    H.smooth(0.8, X, B, Y)
    assert rel(Y.export(), ora.smooth(x, b, 0.8)) < 1e-12
    H.smooth(0.8, None, B, Y)
    assert rel(Y.export(), ora.smooth(None, b, 0.8)) < 1e-12


@pytest.mark.parametrize("nl,kind", [(1, R_DOUBLE), (2, R_SINGLE), (13, R_DOUBLE), (33, R_DOUBLE),
                                     (33, R_SINGLE), (70, R_DOUBLE), (100, R_DOUBLE)])
def test_cma_appinv_column_heights(ctx, nl, kind):
    """columnwise_op_appinv for 1 to 100 rows: in FP64 one thread per
    column up to 12 rows, then 2, 4 or 8 segments per column (13 rows leave
    a short last segment), and one thread per column again above 96 rows
    (d' in shared memory up to 800 FP64 rows); FP32 one thread per column."""
    ncol = 333
    dt = np.float64 if kind == R_DOUBLE else np.float32
    rng = np.random.default_rng(23)
    sub, sup = -rng.random((ncol, nl)), -rng.random((ncol, nl))
    diag = (np.abs(sub) + np.abs(sup) + 0.5) * (1.5 + rng.random((ncol, nl)))
    cm = np.stack([sub, diag, sup], axis=-1).astype(dt)
    ind = np.arange(1, nl + 1, dtype=np.int32)
    A = ColumnwiseOperator(ctx, kind, ncol, nl, nl, 3, 1, 1, 1, 1, ind, ind, cm.ravel())
    x = rng.standard_normal(ncol * nl).astype(dt)
    X, Y = field_from(ctx, x, ncol, nl, kind=kind), Field(ctx, kind, ncol, nl)
    A.apply_inverse(Y, X)
    ref = oh.cma_appinv(cm.ravel(), ncol, nl, ind, x, nl)
    assert rel(Y.export(), ref) < (1e-13 if kind == R_DOUBLE else 2e-6)
    # a second solve reuses the operator's cached factors
    A.apply_inverse(Y, X)
    assert rel(Y.export(), ref) < (1e-13 if kind == R_DOUBLE else 2e-6)


@pytest.mark.parametrize("method", ["gcr", "cg", "bicgstab", "gmres", "fgmres"])
def test_zero_rhs_returns_at_once(ctx, method):
    """b = 0 from x = 0: every Krylov solve returns at once with x = 0 (the
    reference's |r0| < EPS exits; block_gcr has none and divides by a zero
    norm, as the reference would)."""
    p = helmholtz_problem(8, 10, seed=24, mg_levels=2)
    S = api.HelmholtzSystem(ctx, p, mixed=False)
    sol = api.IterativeSolver(api.LinearOperator.from_helmholtz(S.op64), S.mg64, S.x64, method,
                              r_tol=1e-8, max_iter=10, gcrk=4)
    B, X = S.op64.field(np.zeros(p.ndof)), S.op64.field(np.zeros(p.ndof))
    out = sol.apply(X, B)
    assert out.status == api.OK and out.iterations == 0
    assert not np.any(X.export())


def test_zero_rhs_mixed(ctx):
    p = helmholtz_problem(8, 10, seed=25, mg_levels=2)
    S = api.HelmholtzSystem(ctx, p, fp64=False)
    m = S.solve_mixed(np.zeros(p.ndof))
    assert m.status == api.OK and m.outer_iterations == 0
    assert not np.any(S.solution())


@pytest.mark.parametrize("ncol,nlev", [(1, 1), (33, 7), (1001, 3), (4097, 2)])
def test_field_roundtrip_and_vector_tails(ctx, ncol, nlev):
    """Import/export of ragged shapes (transposition tiles cut), and the
    vector algebra on sizes that leave a tail after the 16-byte packs."""
    rng = np.random.default_rng(ncol)
    for kind, dt in ((R_DOUBLE, np.float64), (R_SINGLE, np.float32)):
        x = rng.standard_normal(ncol * nlev).astype(dt)
        y = rng.standard_normal(ncol * nlev).astype(dt)
        X, Y = field_from(ctx, x, ncol, nlev, kind=kind), field_from(ctx, y, ncol, nlev, kind=kind)
        assert np.array_equal(X.export(), x)
        tol = 1e-14 if kind == R_DOUBLE else 1e-6
        Y.axpy(0.75, X)
        assert np.allclose(Y.export(), y + dt(0.75) * x, rtol=tol, atol=tol)
        d = X.dot(X)
        assert abs(d - float(np.dot(x.astype(np.float64), x.astype(np.float64)))) <= 1e-12 * d
        Y.axpby(2.0, X, -1.0, X)
        assert np.allclose(Y.export(), x, rtol=tol, atol=tol)


def test_unaligned_views_take_the_scalar_path(ctx):
    """Field views that start 4 and 12 bytes into an allocation (not 16-byte
    aligned) run the scalar path of the packed vector kernels."""
    n = 1001
    base = Field(ctx, R_SINGLE, 2 * n + 8, 1)
    ref = np.random.default_rng(26).standard_normal(2 * n + 8).astype(np.float32)
    base.import_(ref)
    p = base.device_ptr()
    V = Field(ctx, R_SINGLE, n, 1, device_ptr=p + 4, keep=[base])            # [1, n+1)
    W = Field(ctx, R_SINGLE, n, 1, device_ptr=p + 4 * (n + 3), keep=[base])  # [n+3, 2n+3)
    V.axpy(0.5, W)
    out = base.export()
    want = ref.copy()
    want[1:n + 1] = ref[1:n + 1] + np.float32(0.5) * ref[n + 3:2 * n + 3]
    assert np.allclose(out, want, rtol=1e-6, atol=1e-6)
    d = V.dot(W)
    assert abs(d - float(np.dot(want[1:n + 1].astype(np.float64),
                                want[n + 3:2 * n + 3].astype(np.float64)))) <= 1e-9 * (1 + abs(d))

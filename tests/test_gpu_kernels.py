"""CUDA kernels through the C ABI against the oracle and the golden vectors.

FP64 results must agree with the oracle to a relative 1e-12 (the kernels
may contract multiply-adds into FMAs and sum in another order); FP32 results
to the tolerance stated per test.
"""
import json

import numpy as np
import pytest

from lfric_core_b200 import api
from lfric_core_b200.api import R_DOUBLE, R_SINGLE, Field, field_from
from lfric_core_b200.mesh import coarsen_map, cubed_sphere
from lfric_core_b200.problems import helmholtz_problem, w0_problem
from oracle.oracle import Helmholtz as OraHelm
from tests import ora_helpers as oh
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def load(name):
    return json.loads((GOLDEN / name).read_text())


# ----------------------------------------------------------------- fields
@pytest.mark.parametrize("kind", [R_DOUBLE, R_SINGLE])
def test_field_roundtrip(ctx, kind):
    rng = np.random.default_rng(0)
    x = rng.standard_normal(37 * 11)
    f = field_from(ctx, x.astype(np.float64), 37, 11, kind=kind)
    back = f.export(np.float64)
    dt = np.float64 if kind == R_DOUBLE else np.float32
    assert np.array_equal(back, x.astype(dt).astype(np.float64))
    assert np.array_equal(f.export(np.float32), x.astype(dt).astype(np.float32))


def test_vector_algebra(ctx):
    rng = np.random.default_rng(1)
    n, nl = 1000, 7
    xs = [rng.standard_normal(n * nl) for _ in range(3)]
    X, Y, Z = (field_from(ctx, v, n, nl) for v in xs)
    X.axpy(0.3, Y)
    assert rel(X.export(), xs[0] + 0.3 * xs[1]) < 1e-15
    X.aypx(-1.7, Y)
    ref = -1.7 * (xs[0] + 0.3 * xs[1]) + xs[1]
    assert rel(X.export(), ref) < 1e-15
    Z.axpby(2.0, X, -0.5, Y)
    assert rel(Z.export(), 2.0 * ref - 0.5 * xs[1]) < 1e-15
    Z.scale(0.25)
    assert rel(Z.export(), 0.25 * (2.0 * ref - 0.5 * xs[1])) < 1e-15
    d = Y.dot(X)
    assert abs(d - np.dot(xs[1], ref)) / abs(np.dot(xs[1], ref)) < 1e-13
    assert abs(Y.norm() - np.linalg.norm(xs[1])) / np.linalg.norm(xs[1]) < 1e-14
    Y.set_scalar(2.0)
    Z.divide(X, Y)
    assert np.array_equal(Z.export(), X.export() / 2.0)   # X_divideby_Y is exact here
    W = X.duplicate()
    W.copy(X)
    assert np.array_equal(W.export(), X.export())


def test_inner_products_are_deterministic_and_fp64(ctx):
    rng = np.random.default_rng(2)
    n, nl = 221184 // 16, 70
    v = rng.standard_normal(n * nl).astype(np.float32)
    X = field_from(ctx, v, n, nl, kind=R_SINGLE)
    a, b = X.dot(X), X.dot(X)
    assert a == b
    ref = np.dot(v.astype(np.float64), v.astype(np.float64))
    assert abs(a - ref) / ref < 1e-12        # FP64 accumulation of FP32 data


def test_mixed_kind_copy_and_increment(ctx):
    rng = np.random.default_rng(3)
    x = rng.standard_normal(500)
    e = rng.standard_normal(500).astype(np.float32)
    X = field_from(ctx, x, 50, 10)
    E = field_from(ctx, e, 50, 10, kind=R_SINGLE)
    X.axpy(1.0, E)                              # r_def += r_solver
    assert rel(X.export(), x + e.astype(np.float64)) < 1e-16
    R32 = Field(ctx, R_SINGLE, 50, 10)
    R32.copy(X)
    assert np.array_equal(R32.export(np.float32), (x + e.astype(np.float64)).astype(np.float32))


# ----------------------------------------------------------------- column solves
def test_tri_solve_golden(ctx):
    g = load("tri_solve_kat.json")
    nl = g["nlayers"]
    x = field_from(ctx, np.array(g["x"], float), 1, nl)
    t0 = field_from(ctx, np.full(nl, g["tri_0"]), 1, nl)
    tp = field_from(ctx, np.full(nl, g["tri_plus"]), 1, nl)
    tm = field_from(ctx, np.full(nl, g["tri_minus"]), 1, nl)
    y = Field(ctx, R_DOUBLE, 1, nl)
    api.tri_solve(y, x, t0, tp, tm)
    ans = np.array(g["answer"])
    assert np.max(np.abs(y.export() - ans) / np.abs(ans)) < g["pinned_rel_tol"]


@pytest.mark.parametrize("ncol,nl", [(384, 10), (55, 70), (33, 100)])
@pytest.mark.parametrize("kind", [R_DOUBLE, R_SINGLE])
def test_tri_solve_random(ctx, ncol, nl, kind):
    rng = np.random.default_rng(ncol + nl)
    tm = -rng.uniform(0, 1, ncol * nl)
    tp = -rng.uniform(0, 1, ncol * nl)
    t0 = rng.uniform(1.5, 3, ncol * nl) * (np.abs(tm) + np.abs(tp))
    x = rng.standard_normal(ncol * nl)
    dt = np.float64 if kind == R_DOUBLE else np.float32
    ref = oh.tri_solve(x.astype(dt), t0.astype(dt), tp.astype(dt), tm.astype(dt), ncol, nl)
    F = [field_from(ctx, a, ncol, nl, kind=kind) for a in (x, t0, tp, tm)]
    y = Field(ctx, kind, ncol, nl)
    api.tri_solve(y, *F)
    assert rel(y.export(np.float64), ref) < (TOL64 if kind == R_DOUBLE else 1e-5)


def _cma_problem(ncol, nl, seed):
    rng = np.random.default_rng(seed)
    cm = np.zeros((ncol, nl, 3))
    cm[:, 1:, 0] = -rng.uniform(0, 1, (ncol, nl - 1))
    cm[:, :-1, 2] = -rng.uniform(0, 1, (ncol, nl - 1))
    cm[:, :, 1] = rng.uniform(1.5, 3, (ncol, nl)) * (np.abs(cm[:, :, 0]) + np.abs(cm[:, :, 2]))
    return cm


@pytest.mark.parametrize("nl", [3, 20, 70, 90])
@pytest.mark.parametrize("kind", [R_DOUBLE, R_SINGLE])
def test_cma_app_appinv(ctx, nl, kind):
    """W3->W3 tridiagonal CMA (alpha = beta = 1, gamma = 1, bandwidth 3)."""
    ncol = 6 * 8 * 8
    cm = _cma_problem(ncol, nl, nl)
    ind = np.arange(1, nl + 1, dtype=np.int32)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(ncol * nl)
    lhs0 = rng.standard_normal(ncol * nl)
    dt = np.float64 if kind == R_DOUBLE else np.float32
    A = api.ColumnwiseOperator(ctx, kind, ncol, nl, nl, 3, 1, 1, 1, 1, ind, ind, cm)
    X = field_from(ctx, x, ncol, nl, kind=kind)
    L = field_from(ctx, lhs0, ncol, nl, kind=kind)
    A.apply(L, X)
    ref = oh.cma_app(cm.ravel().astype(dt), ncol, nl, nl, 3, 1, 1, 1, 1, ind, ind, x.astype(dt),
                     lhs0.astype(dt), nl, nl)
    tol = TOL64 if kind == R_DOUBLE else 1e-5
    assert rel(L.export(np.float64), ref) < tol
    Y = Field(ctx, kind, ncol, nl)
    A.apply_inverse(Y, X)
    ref = oh.cma_appinv(cm.ravel().astype(dt), ncol, nl, ind, x.astype(dt), nl)
    assert rel(Y.export(np.float64), ref) < tol


def test_cma_wtheta_m3x3_golden(ctx):
    g = load("cma_m3x3_kat.json")
    nl = g["nlayers"]
    nrow = nl + 1
    cm = np.zeros((1, nrow, 3))
    cm[0, 0], cm[0, 1:-1], cm[0, -1] = g["band_first_row"], g["band_interior"], g["band_last_row"]
    dense = np.diag(cm[0, :, 1]) + np.diag(cm[0, :-1, 2], 1) + np.diag(cm[0, 1:, 0], -1)
    ind = np.arange(1, nrow + 1, dtype=np.int32)
    A = api.ColumnwiseOperator(ctx, R_DOUBLE, 1, nrow, nrow, g["asserted"]["bw"],
                               g["asserted"]["alpha"], 1, g["asserted"]["g_m"], 1, ind, ind, cm)
    rhs = np.random.default_rng(11).uniform(size=nrow)
    X = field_from(ctx, rhs, 1, nrow)
    L = Field(ctx, R_DOUBLE, 1, nrow)
    A.apply(L, X)
    assert np.allclose(L.export(), dense @ rhs, atol=g["tol"] * 1e-8)
    A.apply_inverse(L, X)
    assert np.allclose(dense @ L.export(), rhs, atol=1e-14)


def test_operator_tri_solve(ctx):
    g = load("operator_tri_solve_kat.json")
    nl = g["nlayers"]
    mat = np.array(g["tri_as_passed_fortran_order"])
    x = np.array(g["x"], float)
    ref = oh.operator_tri_solve(mat, x, 1, nl)
    m = np.array([[0, 1]], dtype=np.int32)                  # Wtheta: bottom, top
    lma = api.LocalOperator(ctx, R_DOUBLE, 1, nl, mat, m, 1, nl + 1)
    X = field_from(ctx, x, 1, nl + 1)
    Y = Field(ctx, R_DOUBLE, 1, nl + 1)
    lma.operator_tri_solve(Y, X)
    assert rel(Y.export(), ref) < TOL64


# ----------------------------------------------------------------- LMA
@pytest.mark.parametrize("name,mode", [("matrix_vector", api.LMA_INC),
                                       ("dg_matrix_vector", api.LMA_WRITE)])
def test_lma_golden(ctx, name, mode):
    g = load(f"{name}_kat.json")
    lma = api.LocalOperator(ctx, R_DOUBLE, 1, 1, np.array(g["matrix_fortran_order"]),
                            np.array([[0, 1, 2, 3]]), 4, 1, np.array([[0, 1]]), 2, 1)
    X = field_from(ctx, np.array(g["x"]), 2, 1)
    Y = field_from(ctx, np.full(4, 5.0 if mode == api.LMA_WRITE else 0.0), 4, 1)
    lma.apply(mode, Y, X)
    assert np.allclose(Y.export(), g["answer"], rtol=0, atol=g["tol_r_double"])


def test_lma_transpose_golden(ctx):
    g = load("transpose_matrix_vector_kat.json")
    # matrix(ncell_3d, ndf2=4 (x space), ndf1=2 (lhs space)): an operator
    # from the 2-dof space to the 4-dof space, applied transposed
    lma = api.LocalOperator(ctx, R_DOUBLE, 1, 1, np.array(g["matrix_fortran_order"]),
                            np.array([[0, 1, 2, 3]]), 4, 1, np.array([[0, 1]]), 2, 1)
    X = field_from(ctx, np.array(g["x"]), 4, 1)
    Y = Field(ctx, R_DOUBLE, 2, 1)
    lma.apply(api.LMA_TRANSPOSE, Y, X)
    assert np.allclose(Y.export(), g["answer"], rtol=0, atol=g["tol_r_double"])


@pytest.mark.parametrize("kind,tol", [(R_DOUBLE, TOL64), (R_SINGLE, 5e-6)])
@pytest.mark.parametrize("n,nl", [(4, 3), (8, 10)])
def test_lma_w0_against_oracle(ctx, n, nl, kind, tol):
    """The W0 8x8 applies (FP32 fields against the FP64 oracle at 5e-6)."""
    p = w0_problem(n, nl, seed=n, top=nl * 1e3, kappa_sigma=0.5)
    A = p.matrix()
    nent, nlev = p.nvert, nl + 1
    lma = api.LocalOperator(ctx, kind, p.ncell, nl, A, p.map, nent, nlev)
    rng = np.random.default_rng(4)
    x = rng.standard_normal(p.ndof)
    y0 = rng.standard_normal(p.ndof)
    if kind == R_SINGLE:   # the oracle sees the values the device holds
        x, y0 = x.astype(np.float32).astype(np.float64), y0.astype(np.float32).astype(np.float64)
        A = A.astype(np.float32).astype(np.float64)
    m1 = (p.map + 1).astype(np.int32)
    X = field_from(ctx, x, nent, nlev, kind=kind)
    Y = field_from(ctx, y0, nent, nlev, kind=kind)
    lma.apply(api.LMA_INC, Y, X)
    ref = oh.lma_apply("matrix_vector", A, m1, m1, p.ncell, nl, x, y0=y0)
    assert rel(Y.export(np.float64), ref) < tol
    lma.apply(api.LMA_WRITE, Y, X)
    ref0 = oh.lma_apply("matrix_vector", A, m1, m1, p.ncell, nl, x, y0=np.zeros(p.ndof))
    assert rel(Y.export(np.float64), ref0) < tol
    Y.import_(y0)
    lma.apply(api.LMA_TRANSPOSE, Y, X)
    # transpose_matrix_vector reads matrix(ik, df2, df1) = A(ik, df_to, df_from)
    ref = oh.lma_apply("transpose_matrix_vector", A, m1, m1, p.ncell, nl, x, y0=y0)
    assert rel(Y.export(np.float64), ref) < tol
    D = field_from(ctx, y0, nent, nlev, kind=kind)
    lma.diagonal(D)
    ref = y0 + oh.mm_diagonal(A, m1, p.ncell, nl, p.ndof)
    assert rel(D.export(np.float64), ref) < tol


def test_lma_wide_incidence_lists(ctx):
    """An entity shared by 24 cells, more than the padded incidence table's
    16 slots: the applies take the one-pass gathers over the incidence
    lists (forward, write and transposed) and match the oracle."""
    ncell, nl, nlev = 24, 5, 6
    m = np.zeros((ncell, 3), dtype=np.int32)
    for c in range(ncell):      # df 0 on the hub entity 0, dfs 1-2 on entity c+1
        m[c] = [0, (c + 1) * nlev, (c + 1) * nlev + 1]
    nent = ncell + 1
    ndof = nent * nlev
    rng = np.random.default_rng(51)
    A = rng.standard_normal((ncell * nl, 3, 3)).ravel(order="F")
    lma = api.LocalOperator(ctx, R_DOUBLE, ncell, nl, A, m, nent, nlev)
    x, y0 = rng.standard_normal(ndof), rng.standard_normal(ndof)
    m1 = m + 1
    X, Y = field_from(ctx, x, nent, nlev), field_from(ctx, y0, nent, nlev)
    lma.apply(api.LMA_INC, Y, X)
    assert rel(Y.export(), oh.lma_apply("matrix_vector", A, m1, m1, ncell, nl, x, y0=y0)) < TOL64
    lma.apply(api.LMA_WRITE, Y, X)
    ref0 = oh.lma_apply("matrix_vector", A, m1, m1, ncell, nl, x, y0=np.zeros(ndof))
    assert rel(Y.export(), ref0) < TOL64
    Y.import_(y0)
    lma.apply(api.LMA_TRANSPOSE, Y, X)
    ref = oh.lma_apply("transpose_matrix_vector", A, m1, m1, ncell, nl, x, y0=y0)
    assert rel(Y.export(), ref) < TOL64


# ----------------------------------------------------------------- intergrid
def test_intergrid_scalar_golden(ctx):
    g = load("intergrid_kat.json")
    child = np.array([[[0, 1], [2, 3]]], dtype=np.int32)
    ig = api.Intergrid(ctx, child, 4)
    k = g["restrict_scalar_unweighted"]
    nl = k["nlayers"]
    C_, Fi = Field(ctx, R_DOUBLE, 1, nl), field_from(ctx, np.full(4 * nl, k["fine"]), 4, nl)
    ig.restrict(api.RESTRICT_UNWEIGHTED, C_, Fi)
    assert np.allclose(C_.export(), k["coarse"], atol=1e-12)
    ig.restrict(api.RESTRICT_MASS_W3, C_, Fi)
    assert np.allclose(C_.export(), g["restrict_mass_w3"]["coarse"], atol=1e-12)
    k = g["prolong_scalar_unweighted"]
    Fo = Field(ctx, R_DOUBLE, 4, nl)
    ig.prolong(Fo, field_from(ctx, np.full(nl, k["coarse"]), 1, nl))
    assert np.allclose(Fo.export(), k["coarse"], atol=1e-12)
    k = g["restrict_scalar_weighted"]
    C1 = Field(ctx, R_DOUBLE, 1, 1)
    W = field_from(ctx, np.array(k["weights"]), 4, 1)
    ig.restrict(api.RESTRICT_WEIGHTED, C1, field_from(ctx, np.array(k["fine"]), 4, 1), W)
    assert np.allclose(C1.export(), k["coarse"], atol=1e-12)
    k = g["prolong_scalar_weighted"]
    F1 = Field(ctx, R_DOUBLE, 4, 1)
    ig.prolong(F1, field_from(ctx, np.array([k["coarse"]]), 1, 1), W)
    assert np.allclose(F1.export(), k["fine"], atol=1e-12)


def test_intergrid_scalar_random(ctx):
    nf, nl = 8, 12
    child = coarsen_map(nf)
    ncoarse, nfine = child.shape[0], 6 * nf * nf
    ig = api.Intergrid(ctx, child, nfine)
    rng = np.random.default_rng(8)
    fine = rng.standard_normal(nfine * nl)
    w = rng.uniform(0.5, 2, nfine * nl)
    Fi, Wf = field_from(ctx, fine, nfine, nl), field_from(ctx, w, nfine, nl)
    Co = Field(ctx, R_DOUBLE, ncoarse, nl)
    for mode, name in [(api.RESTRICT_UNWEIGHTED, "unweighted"), (api.RESTRICT_WEIGHTED, "weighted"),
                       (api.RESTRICT_MASS_W3, "mass")]:
        ig.restrict(mode, Co, Fi, Wf if name == "weighted" else None)
        ref = oh.restrict(name, child, fine, nl, weights=w)
        assert rel(Co.export(), ref) < TOL64, name
    coarse = rng.standard_normal(ncoarse * nl)
    Cc = field_from(ctx, coarse, ncoarse, nl)
    for wt in (None, w):
        Fo = field_from(ctx, fine, nfine, nl)
        ig.prolong(Fo, Cc, None if wt is None else Wf)
        assert rel(Fo.export(), oh.prolong(child, fine, coarse, nl, weights=wt)) < TOL64


def _w0_golden_tables(k):
    nx, ny, nl = k["nx"], k["ny"], k["nlayers"]
    cm_xy = np.array(k["cell_map_xy"])
    child = np.zeros((1, ny, nx), dtype=np.int32)
    for x in range(nx):
        for y in range(ny):
            child[0, y, x] = cm_xy[x][y] - 1
    mf = np.array(k["map_fine"])
    fc = ((mf[:, :4] - 1) // (nl + 1)).astype(np.int32)
    cc = (((np.array(k["map_coarse"])[:4] - 1) // (nl + 1))[None, :]).astype(np.int32)
    return child, fc, cc


def test_w0_golden(ctx):
    g = load("intergrid_kat.json")
    k = g["restrict_w0"]
    child, fc, cc = _w0_golden_tables(k)
    nl = k["nlayers"]
    ig = api.Intergrid(ctx, child, child.size, cc, fc)
    nvc, nvf = int(cc.max()) + 1, int(fc.max()) + 1
    Co = Field(ctx, R_DOUBLE, nvc, nl + 1)
    ig.restrict_w0(Co, field_from(ctx, np.array(k["fine"]), nvf, nl + 1))
    assert np.allclose(Co.export(), k["coarse"], atol=k["tol"])
    k = g["prolong_w0"]
    Fo = Field(ctx, R_DOUBLE, nvf, nl + 1)
    ig.prolong_w0(Fo, field_from(ctx, np.array(k["coarse"]), nvc, nl + 1))
    assert np.allclose(Fo.export(), k["fine"], atol=k["tol"])


def test_w0_random_against_oracle(ctx):
    nf, nl = 8, 5
    child = coarsen_map(nf)
    fine, coarse = cubed_sphere(nf), cubed_sphere(nf // 2)
    ig = api.Intergrid(ctx, child, fine.ncell, coarse.cell_vertices, fine.cell_vertices)
    rng = np.random.default_rng(9)
    src = rng.standard_normal(fine.nvert * (nl + 1))
    Co = Field(ctx, R_DOUBLE, coarse.nvert, nl + 1)
    ig.restrict_w0(Co, field_from(ctx, src, fine.nvert, nl + 1))
    ref = oh.w0_transfer("restrict", child, fine.cell_vertices, coarse.cell_vertices, src, nl)
    assert np.array_equal(Co.export(), ref)
    csrc = rng.standard_normal(coarse.nvert * (nl + 1))
    Fo = Field(ctx, R_DOUBLE, fine.nvert, nl + 1)
    ig.prolong_w0(Fo, field_from(ctx, csrc, coarse.nvert, nl + 1))
    ref = oh.w0_transfer("prolong", child, fine.cell_vertices, coarse.cell_vertices, csrc, nl)
    assert rel(Fo.export(), ref) < 1e-15


# ----------------------------------------------------------------- Helmholtz
@pytest.fixture(scope="module")
def helm_small():
    return helmholtz_problem(8, 20, seed=3, mg_levels=3)


@pytest.mark.parametrize("kind", [R_DOUBLE, R_SINGLE])
def test_helmholtz_apply_and_smooth(ctx, helm_small, kind):
    p = helm_small
    dt = np.float64 if kind == R_DOUBLE else np.float32
    ora = OraHelm(p)
    mesh = api.Mesh(ctx, p.links)
    H = api.Helmholtz(ctx, kind, mesh, p.nlayers, p.cm, p.hf)
    rng = np.random.default_rng(12)
    x = rng.standard_normal(p.ndof).astype(dt)
    b = rng.standard_normal(p.ndof).astype(dt)
    X, B, Y = H.field(x), H.field(b), H.field()
    H.apply(Y, X)
    tol = TOL64 if kind == R_DOUBLE else 2e-6
    assert rel(Y.export(np.float64), ora.apply(x)) < tol
    H.smooth(0.8, None, B, Y)
    assert rel(Y.export(np.float64), ora.smooth(None, b, 0.8)) < tol
    H.smooth(0.8, X, B, Y)
    assert rel(Y.export(np.float64), ora.smooth(x, b, 0.8)) < tol


@pytest.mark.parametrize("kind", [R_SINGLE, R_DOUBLE])
@pytest.mark.parametrize("nx,ny", [(1, 1), (2, 1), (3, 1), (2, 2)])
def test_residual_restrict_any_child_count(ctx, kind, nx, ny):
    """The fused residual + restriction on maps of 1 to 4 children per
    coarse column (the lane-per-child kernel leaves the lanes past the
    map's children idle): b_c = the sum of the children's b - A x."""
    p = helmholtz_problem(6, 7, seed=47, mg_levels=1)
    ncol, nl = p.ncol, p.nlayers
    H = api.Helmholtz(ctx, kind, api.Mesh(ctx, p.links), nl, p.cm, p.hf)
    nq = nx * ny
    nc = ncol // nq
    child = np.arange(ncol, dtype=np.int32).reshape(nc, ny, nx)   # 216 columns
    ig = api.Intergrid(ctx, child, ncol)
    rng = np.random.default_rng(48)
    dt = np.float64 if kind == R_DOUBLE else np.float32
    x = rng.standard_normal(p.ndof).astype(dt)
    b = rng.standard_normal(p.ndof).astype(dt)
    X, B, Y = H.field(x), H.field(b), H.field()
    H.apply(Y, X)
    r = (b.astype(np.float64) - Y.export(np.float64)).reshape(ncol, nl)
    CB = Field(ctx, kind, nc, nl)
    H.residual_restrict(ig, X, B, CB)
    want = np.zeros((nc, nl))
    for q in range(nq):
        want += r[child.reshape(nc, nq)[:, q]]
    tol = 1e-13 if kind == R_DOUBLE else 1e-5
    assert rel(CB.export(np.float64), want.ravel()) < tol


@pytest.mark.parametrize("n,kind", [(12, R_SINGLE), (16, R_DOUBLE), (24, R_SINGLE),
                                    (48, R_DOUBLE), (96, R_SINGLE), (96, R_DOUBLE)])
def test_helmholtz_smooth_each_launch_path(ctx, n, kind):
    """The sweep runs as the segmented one-kernel sweep on meshes with few
    columns (70 levels as 32 x 3 on C12, 16 x 5 on C16, 8 x 9 on C24 and
    4 x 18 on C48: threads per column x levels per thread), and as
    right-hand side + substitution on C96 (the FP32 substitution through
    TMA-staged tiles): all against the oracle."""
    p = helmholtz_problem(n, 70, seed=11, mg_levels=1)
    dt = np.float64 if kind == R_DOUBLE else np.float32
    ora = OraHelm(p)
    H = api.Helmholtz(ctx, kind, api.Mesh(ctx, p.links), p.nlayers, p.cm, p.hf)
    rng = np.random.default_rng(13)
    x = rng.standard_normal(p.ndof).astype(dt)
    b = rng.standard_normal(p.ndof).astype(dt)
    X, B, Y = H.field(x), H.field(b), H.field()
    tol = TOL64 if kind == R_DOUBLE else 2e-6
    H.smooth(0.8, None, B, Y)
    assert rel(Y.export(np.float64), ora.smooth(None, b, 0.8)) < tol
    H.smooth(0.8, X, B, Y)
    assert rel(Y.export(np.float64), ora.smooth(x, b, 0.8)) < tol
    ctx.synchronize()   # no bounded wait ran out


def test_galerkin_coarse_operator(ctx, helm_small):
    p = helm_small
    ora = OraHelm(p)
    meshes = [api.Mesh(ctx, p.links)] + [api.Mesh(ctx, l) for l in p.mg_links]
    H = api.Helmholtz(ctx, R_DOUBLE, meshes[0], p.nlayers, p.cm, p.hf)
    rng = np.random.default_rng(13)
    for l, ch in enumerate(p.mg_child):
        ig = api.Intergrid(ctx, ch, meshes[l].ncol)
        Hc = H.coarsen(ig, meshes[l + 1], R_DOUBLE)
        x = rng.standard_normal(meshes[l + 1].ncol * p.nlayers)
        Y = Hc.field()
        Hc.apply(Y, Hc.field(x))
        assert rel(Y.export(), ora.apply(x, level=l + 1)) < TOL64
        H = Hc


@pytest.mark.parametrize("kind", [R_DOUBLE, R_SINGLE])
def test_multigrid_vcycle(ctx, helm_small, kind):
    p = helm_small
    ora = OraHelm(p)
    sysm = api.HelmholtzSystem(ctx, p, mixed=(kind == R_SINGLE), fp64=True)
    b = np.random.default_rng(14).standard_normal(p.ndof)
    if kind == R_DOUBLE:
        B, Y = sysm.op64.field(b), sysm.op64.field()
        sysm.mg64.apply(B, Y)
        assert rel(Y.export(), ora.mg_apply(b)) < TOL64
    else:
        op = sysm.levels32[0]
        B, Y = op.field(b.astype(np.float32)), op.field()
        sysm.mg32.apply(B, Y)
        assert rel(Y.export(np.float64), ora.mg_apply(b.astype(np.float32))) < 1e-5


@pytest.mark.parametrize("n,sweep_words", [(8, 6), (96, 9)])
@pytest.mark.parametrize("kind,w", [(R_DOUBLE, 8), (R_SINGLE, 4)])
def test_algorithmic_byte_counter(ctx, kind, w, n, sweep_words):
    """lfg_ctx_algorithmic_bytes adds each kernel's arrays once per launch:
    5 words per dof plus the couplings for the Helmholtz apply, 3 for axpy,
    2 for a dot, 5 for the smoother sweep from zero; the sweep from a guess
    is 6 words plus the couplings as one segmented kernel (C8) and 3 + 6
    plus the couplings as right-hand side + substitution (C96).  The
    couplings count 2 words per dof for the FP64 operator (symmetric, each
    face read through one side) and 4 for the FP32 one."""
    p = helmholtz_problem(n, 12, seed=41, mg_levels=1)
    H = api.Helmholtz(ctx, kind, api.Mesh(ctx, p.links), p.nlayers, p.cm, p.hf)
    X, Y, B = H.field(p.rhs), H.field(), H.field(p.rhs)
    ndof = p.ndof
    hw = 2 if kind == R_DOUBLE else 4
    for fn, words in ((lambda: H.apply(Y, X), 5 + hw), (lambda: Y.axpy(0.5, X), 3),
                      (lambda: X.dot(Y), 2), (lambda: H.smooth(0.8, None, B, Y), 5),
                      (lambda: H.smooth(0.8, X, B, Y), sweep_words + hw)):
        b0 = ctx.algorithmic_bytes()
        fn()
        assert ctx.algorithmic_bytes() - b0 == words * ndof * w

"""The oracle against the reference's own unit-test vectors (CPU only).

Fixtures in tests/golden were read out of the reference's pFUnit tests by
tests/golden/make_golden.py; each test cites the reference test it pins.
"""
import json

import numpy as np
import pytest

from tests.conftest import GOLDEN
from tests import ora_helpers as oh


def load(name):
    return json.loads((GOLDEN / name).read_text())


def test_tri_solve_kat_pinned():
    # sci_tri_solve_kernel_mod_test.pf: the reference's tolerance is 1e10
    # (void); the stated answer is pinned here at 1e-12 relative.
    g = load("tri_solve_kat.json")
    assert g["reference_tol"] >= 1e9
    nl = g["nlayers"]
    x = np.array(g["x"], dtype=np.float64)
    t0 = np.full(nl, g["tri_0"])
    tp = np.full(nl, g["tri_plus"])
    tm = np.full(nl, g["tri_minus"])
    y = oh.tri_solve(x, t0, tp, tm, 1, nl)
    ans = np.array(g["answer"])
    assert np.max(np.abs(y - ans) / np.abs(ans)) < 1e-12
    # and it is the dense solution
    A = np.diag(t0) + np.diag(tp[:-1], 1) + np.diag(tm[1:], -1)
    assert np.allclose(A @ y, x, rtol=0, atol=1e-13)


def test_tri_solve_kat_single():
    g = load("tri_solve_kat.json")
    nl = g["nlayers"]
    x = np.array(g["x"], dtype=np.float32)
    y = oh.tri_solve(x, np.full(nl, g["tri_0"], np.float32), np.full(nl, g["tri_plus"], np.float32),
                     np.full(nl, g["tri_minus"], np.float32), 1, nl)
    assert np.max(np.abs(y - np.array(g["answer"]))) < 1e-5


def test_operator_tri_solve_as_written():
    # sci_operator_tri_solve_kernel_mod_test.pf passes tri(2,2,nz-1) where the
    # kernel reads matrix(ncell=nz-1,2,2): with the reference's void tolerance
    # the stated answer is not what the kernel computes.  Pin the kernel on
    # the test's literal memory instead: it must equal the dense solve of the
    # tridiagonal the kernel assembles from that memory.
    g = load("operator_tri_solve_kat.json")
    nl = g["nlayers"]
    mat = np.array(g["tri_as_passed_fortran_order"])
    x = np.array(g["x"], dtype=np.float64)
    y = oh.operator_tri_solve(mat, x, 1, nl)
    M = mat.reshape((nl, 2, 2), order="F")
    t0 = np.zeros(nl + 1)
    tp = np.zeros(nl + 1)
    tm = np.zeros(nl + 1)
    for k in range(nl):
        t0[k] += M[k, 0, 0]
        tp[k] = M[k, 0, 1]
        tm[k + 1] = M[k, 1, 0]
        t0[k + 1] += M[k, 1, 1]
    A = np.diag(t0) + np.diag(tp[:-1], 1) + np.diag(tm[1:], -1)
    assert np.allclose(y, np.linalg.solve(A, x), rtol=1e-12, atol=1e-12)
    assert not np.allclose(y, g["answer"], atol=1e-6)


def test_operator_tri_solve_intended_layout():
    # The test's intent: halves a0/2 on the diagonal, ap above, am below.
    g = load("operator_tri_solve_kat.json")
    nl = g["nlayers"]
    M = np.zeros((nl, 2, 2))
    M[:, 0, 0] = M[:, 1, 1] = 0.5 * g["a0"]
    M[:, 0, 1] = g["ap"]
    M[:, 1, 0] = g["am"]
    x = np.array(g["x"], dtype=np.float64)
    y = oh.operator_tri_solve(M.ravel(order="F"), x, 1, nl)
    d = np.full(nl + 1, g["a0"])
    d[0] = d[-1] = 0.5 * g["a0"]
    A = np.diag(d) + np.diag(np.full(nl, g["ap"]), 1) + np.diag(np.full(nl, g["am"]), -1)
    assert np.allclose(y, np.linalg.solve(A, x), rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name,kind", [("matrix_vector", "matrix_vector"),
                                       ("dg_matrix_vector", "dg_matrix_vector")])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_lma_kats(name, kind, dtype):
    g = load(f"{name}_kat.json")
    x = np.array(g["x"], dtype=dtype)
    y0 = np.zeros(4, dtype=dtype)
    y = oh.lma_apply(kind, np.array(g["matrix_fortran_order"], dtype=dtype),
                     np.array([g["map1"]]), np.array([g["map2"]]), 1, 1, x, y0=y0)
    tol = g["tol_r_double"] if dtype == np.float64 else 1e-5
    assert np.allclose(y, g["answer"], rtol=0, atol=tol)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_transpose_kat(dtype):
    g = load("transpose_matrix_vector_kat.json")
    x = np.array(g["x"], dtype=dtype)
    y = oh.lma_apply("transpose_matrix_vector", np.array(g["matrix_fortran_order"], dtype=dtype),
                     np.array([g["map1"]]), np.array([g["map2"]]), 1, 1, x,
                     y0=np.zeros(2, dtype=dtype))
    tol = g["tol_r_double"] if dtype == np.float64 else g["tol_r_single"] * 10
    assert np.allclose(y, g["answer"], rtol=0, atol=tol)


def test_mm_diagonal_kat():
    g = load("mm_diagonal_kat.json")
    d = oh.mm_diagonal(np.array(g["matrix_fortran_order"]), np.array(g["map"]), 2, g["nlayers"],
                       g["undf"])
    assert np.allclose(d, g["answer"], rtol=0, atol=1e-12)


def _m3x3_cma(nl):
    """Wtheta->Wtheta CMA parameters the reference's canned data produce."""
    from oracle.oracle import lib
    import ctypes as C
    out = np.zeros(7, dtype=np.int32)
    ind_to = np.zeros(nl + 1, dtype=np.int32)
    ind_from = np.zeros(nl + 1, dtype=np.int32)
    offs = np.array([0, 1], dtype=np.int32)       # bottom face, top face
    lib().ora_cma_params(nl, 0, 1, 0, 1, offs.ctypes.data_as(C.POINTER(C.c_int)),
                         offs.ctypes.data_as(C.POINTER(C.c_int)),
                         out.ctypes.data_as(C.POINTER(C.c_int)),
                         ind_to.ctypes.data_as(C.POINTER(C.c_int)),
                         ind_from.ctypes.data_as(C.POINTER(C.c_int)))
    return out, ind_to, ind_from


def test_cma_params_match_reference_asserts():
    g = load("cma_m3x3_kat.json")
    out, ind_to, _ = _m3x3_cma(g["nlayers"])
    alpha, beta, gm, gp, bw, nrow, ncol = out
    a = g["asserted"]
    assert alpha == a["alpha"] and gm == a["g_m"] and bw == a["bw"] and a["ndf"] == 2
    assert nrow == ncol == g["nlayers"] + 1
    assert list(ind_to) == list(range(1, nrow + 1))


def _m3x3_bands(g, nrow, dtype):
    cm = np.zeros((1, nrow, 3), dtype=dtype)   # [cell][row][band] = Fortran (3, nrow, 1)
    cm[0, 0] = g["band_first_row"]
    cm[0, 1:-1] = g["band_interior"]
    cm[0, -1] = g["band_last_row"]
    dense = np.zeros((nrow, nrow))
    for i in range(nrow):
        for j, b in zip((i - 1, i, i + 1), cm[0, i]):
            if 0 <= j < nrow:
                dense[i, j] = b
    return cm, dense


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_cma_app_and_appinv_m3x3(dtype):
    # columnwise_op_app/appinv_kernel_mod_test.pf: apply against a dense
    # product and invert then re-apply the dense matrix, random RHS.
    g = load("cma_m3x3_kat.json")
    out, ind_to, ind_from = _m3x3_cma(g["nlayers"])
    alpha, beta, gm, gp, bw, nrow, ncol = (int(v) for v in out)
    cm, dense = _m3x3_bands(g, nrow, dtype)
    rng = np.random.default_rng(11)
    rhs = rng.uniform(size=nrow).astype(dtype)
    lhs = oh.cma_app(cm.ravel(), 1, nrow, ncol, bw, alpha, beta, gm, gp, ind_to, ind_from, rhs,
                     np.zeros(nrow, dtype=dtype), nrow, ncol)
    assert np.allclose(lhs, dense @ rhs, rtol=0, atol=g["tol"])
    inv = oh.cma_appinv(cm.ravel(), 1, nrow, ind_to, rhs, nrow)
    assert np.allclose(dense @ inv, rhs, rtol=0, atol=g["tol"])
    if dtype == np.float64:
        assert np.allclose(dense @ inv, rhs, rtol=0, atol=1e-14)


def _scalar_layout(nl):
    # cell_map(x, y) = x + (y-1)*2, map_f(1,c) = 1 + (c-1)*nlayers
    child = np.array([[[0, 1], [2, 3]]], dtype=np.int32)   # [C][y][x]
    return child


def test_intergrid_scalar_kats():
    g = load("intergrid_kat.json")
    child = _scalar_layout(3)
    k = g["restrict_scalar_unweighted"]
    c = oh.restrict("unweighted", child, np.full(4 * k["nlayers"], k["fine"]), k["nlayers"])
    assert np.allclose(c, k["coarse"], atol=1e-12)
    k = g["restrict_mass_w3"]
    c = oh.restrict("mass", child, np.full(4 * k["nlayers"], k["fine"]), k["nlayers"])
    assert np.allclose(c, k["coarse"], atol=1e-12)
    k = g["prolong_scalar_unweighted"]
    f = oh.prolong(child, np.zeros(4 * k["nlayers"]), np.full(k["nlayers"], k["coarse"]),
                   k["nlayers"])
    assert np.allclose(f[:3], k["fine"], atol=1e-12)
    assert np.allclose(f, k["coarse"], atol=1e-12)
    k = g["restrict_scalar_weighted"]
    c = oh.restrict("weighted", child, np.array(k["fine"]), 1, weights=np.array(k["weights"]))
    assert np.allclose(c, k["coarse"], atol=1e-12)
    k = g["prolong_scalar_weighted"]
    f = oh.prolong(child, np.zeros(4), np.array([k["coarse"]]), 1, weights=np.array(k["weights"]))
    assert np.allclose(f, k["fine"], atol=1e-12)


def _w0_tables(k):
    nx, ny, nl = k["nx"], k["ny"], k["nlayers"]
    cm_xy = np.array(k["cell_map_xy"])               # [x][y], 1-based fine cells
    child = np.zeros((1, ny, nx), dtype=np.int32)
    for x in range(nx):
        for y in range(ny):
            child[0, y, x] = cm_xy[x][y] - 1
    mf = np.array(k["map_fine"])                     # [cell][df] 1-based dofs
    fine_corners = (mf[:, :4] - 1) // (nl + 1)
    coarse_corners = ((np.array(k["map_coarse"])[:4] - 1) // (nl + 1))[None, :]
    return child, fine_corners.astype(np.int32), coarse_corners.astype(np.int32)


def test_w0_kats():
    g = load("intergrid_kat.json")
    k = g["restrict_w0"]
    child, fc, cc = _w0_tables(k)
    out = oh.w0_transfer("restrict", child, fc, cc, np.array(k["fine"]), k["nlayers"])
    assert np.allclose(out, k["coarse"], atol=k["tol"])
    k = g["prolong_w0"]
    child, fc, cc = _w0_tables(k)
    out = oh.w0_transfer("prolong", child, fc, cc, np.array(k["coarse"]), k["nlayers"])
    assert np.allclose(out, k["fine"], atol=k["tol"])


# ------------------------------------------------- CMA assembly and algebra
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_cma_asm_m3x3(dtype):
    # columnwise_op_asm_kernel_mod_test.pf: Wtheta -> Wtheta, 3 layers, every
    # cell stencil (1/3 1/6; 1/6 1/3): rows 1/3 1/6 | 1/6 2/3 1/6 | 1/6 1/3
    g = load("cma_assembly_kat.json")
    nl = g["nlayers"]
    p = oh.cma_size(nl, 2, 2, 1, 0, 1, 0)
    assert (p["alpha"], p["beta"], p["gm"], p["gp"], p["bw"]) == (1, 1, 1, 1, 3)
    ls = np.tile(np.array(g["asm_stencil_fortran_order"]).reshape(2, 2, order="F"), (nl, 1, 1))
    cb = oh.banded_dofmap(nl, 2, 0, 1)
    cm = oh.cma_asm(ls, p, 1, nl, cb, cb, dtype)
    tol = 1e-15 if dtype == np.float64 else 1e-7
    for i in range(p["nrow"]):
        if i == 0:
            got, want = cm[1:3, i, 0], g["asm_first_row"]
        elif i == p["nrow"] - 1:
            got, want = cm[0:2, i, 0], g["asm_last_row"]
        else:
            got, want = cm[:, i, 0], g["asm_interior_row"]
        assert np.allclose(got, want, rtol=0, atol=tol * 4)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_cma_mul_dtd(dtype):
    # columnwise_op_mul_kernel_mod_test.pf: D (W3 <- Wtheta) bands (+1,-1),
    # D^T (Wtheta <- W3) bands (-1,+1); C = D^T D against the dense product
    g = load("cma_assembly_kat.json")
    nl = g["mul_nlayers"]
    pTT = oh.cma_size(nl, 2, 2, 1, 0, 1, 0)
    pT3 = oh.cma_size(nl, 2, 1, 1, 0, 0, 1)
    p3T = oh.cma_size(nl, 1, 2, 0, 1, 1, 0)
    assert pT3["alpha"] == p3T["beta"] and pT3["bw"] == p3T["bw"]
    assert pT3["gm"] == p3T["gp"] and pT3["gp"] == p3T["gm"]
    D = np.zeros((p3T["bw"], p3T["nrow"], 1), dtype=dtype, order="F")
    D[0, :, 0], D[1, :, 0] = g["mul_D_bands"]
    DT = np.zeros((pT3["bw"], pT3["nrow"], 1), dtype=dtype, order="F")
    DT[0, :, 0], DT[1, :, 0] = g["mul_DT_bands"]
    C0 = np.zeros((pTT["bw"], pTT["nrow"], 1), dtype=dtype, order="F")
    C = oh.cma_mul(DT, pT3, D, p3T, C0, pTT, 1)
    Dd = np.zeros((p3T["nrow"], p3T["ncol"]))
    for i in range(p3T["nrow"]):
        Dd[i, i], Dd[i, i + 1] = 1.0, -1.0
    assert np.allclose(oh.cma_dense(C, pTT), Dd.T @ Dd, rtol=0, atol=g["tol"])
    assert np.array_equal(oh.cma_dense(C, pTT), Dd.T @ Dd)  # small integers: exact


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_cma_scaledadd(dtype):
    # columnwise_op_scaledadd_kernel_mod_test.pf: C = mu M + nu DTD with M = I
    # on W3 and DTD = tridiag(1, 2, 1) in the product pattern
    g = load("cma_assembly_kat.json")
    nl = g["nlayers"]
    p33 = oh.cma_size(nl, 1, 1, 0, 1, 0, 1)
    p3T = oh.cma_size(nl, 1, 2, 0, 1, 1, 0)
    pT3 = oh.cma_size(nl, 2, 1, 1, 0, 0, 1)
    pp = oh.cma_prod_size(p3T, pT3)
    M = np.zeros((p33["bw"], p33["nrow"], 1), dtype=dtype, order="F")
    M[0, :, 0] = 1.0
    DTD = np.zeros((pp["bw"], pp["nrow"], 1), dtype=dtype, order="F")
    for b, v in enumerate(g["scaledadd_DTD_bands"]):
        DTD[b, :, 0] = v
    mu, nu = g["scaledadd_mu"], g["scaledadd_nu"]
    C = oh.cma_scaledadd(M, p33, DTD, pp, pp, 1, mu, nu)
    dense = mu * np.eye(p33["nrow"]) + nu * (2 * np.eye(pp["nrow"]) + np.eye(pp["nrow"], k=1)
                                            + np.eye(pp["nrow"], k=-1))
    tol = 1e-14 if dtype == np.float64 else 2e-6
    assert np.allclose(oh.cma_dense(C, pp), dense, rtol=0, atol=tol * 10)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_cma_asm_diag_hmht(dtype):
    # columnwise_op_asm_diag_hmht_kernel_mod_test.pf: Dh = (rho), M2h =
    # diag(sigma) per cell; every diagonal entry is sum rho^2 / sigma
    g = load("cma_assembly_kat.json")
    nl = g["nlayers"]
    p = oh.cma_size(nl, 1, 1, 0, 1, 0, 1)
    rho, sigma = np.array(g["hmht_rho"]), np.array(g["hmht_sigma"])
    dh = np.tile(rho.reshape(1, 1, 4), (nl, 1, 1))
    m2h = np.tile(np.diag(sigma)[None], (nl, 1, 1))
    cb = oh.banded_dofmap(nl, 1, 1, 0)
    cm = oh.cma_hmht(dh, m2h, p, 1, nl, cb, dtype)
    answer = float(np.sum(rho ** 2 / sigma))
    tol = 1e-14 if dtype == np.float64 else 1e-6
    assert np.allclose(cm[0, :, 0], answer, rtol=tol, atol=0)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_cma_asm_m2v_lumped_inv(dtype):
    # columnwise_op_asm_m2v_lumped_inv_kernel_mod_test.pf: W2v, stencil
    # (1/3 1/6; 1/6 1/3): band 1 holds 3 on the end rows, 3/2 inside
    g = load("cma_assembly_kat.json")
    nl = g["nlayers"]
    p = oh.cma_size(nl, 2, 2, 1, 0, 1, 0)
    ls = np.tile(np.array(g["m2v_stencil_fortran_order"]).reshape(2, 2, order="F"), (nl, 1, 1))
    cb = oh.banded_dofmap(nl, 2, 0, 1)
    cm = oh.cma_m2v(ls, p, 1, nl, cb, dtype)
    want = np.full(p["nrow"], g["m2v_interior_rows"])
    want[[0, -1]] = g["m2v_end_rows"]
    tol = 1e-14 if dtype == np.float64 else 1e-6
    assert np.allclose(cm[0, :, 0], want, rtol=tol, atol=0)
    assert not np.any(cm[1:, :, 0])


# ------------------------------------------------- W2 intergrid transfers
@pytest.mark.parametrize("name,dtype", [("restrict_w2", np.float64), ("restrict_w2", np.float32),
                                        ("restrict_w2h", np.float64), ("restrict_w2v", np.float64),
                                        ("restrict_w2v", np.float32)])
def test_w2_restrict_kat(name, dtype):
    # restrict_w2{,h,v}_kernel_mod_test.pf (one coarse cell of 2 x 3 fine cells)
    g = load("w2_intergrid_kat.json")
    k = g[name]
    kind = {"restrict_w2": "w2", "restrict_w2h": "w2h", "restrict_w2v": "w2v"}[name]
    got = oh.w2_restrict(kind, k["nlayers"], k["nx"], k["ny"], k["map_f"], k["map_c"],
                         k["fine"], len(k["answer"]), dtype=dtype)
    assert np.allclose(got, k["answer"], rtol=0, atol=g["tol"])


def test_w2_weights_and_prolong_kat():
    # weights_prolong_w2_kernel_mod_test.pf and prolong_w2_kernel_mod_test.pf
    g = load("w2_intergrid_kat.json")
    k = g["weights_prolong_w2"]
    w = oh.w2_weights(k["nlayers"], k["nx"], k["ny"], k["map_f"], len(k["answer"]))
    assert np.allclose(w, k["answer"], rtol=0, atol=g["tol"])
    k = g["prolong_w2"]
    assert np.allclose(w, k["weights"], rtol=0, atol=g["tol"])
    fine = oh.w2_prolong(k["nlayers"], k["nx"], k["ny"], k["map_f"], k["map_c"], k["coarse"],
                         k["weights"], np.zeros(len(k["answer"])))
    assert np.allclose(fine, k["answer"], rtol=0, atol=g["tol"])

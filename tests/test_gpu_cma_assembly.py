"""CMA assembly and algebra on the device (lfg_cma_assemble, _multiply,
_scaled_add, _assemble_diag_hmht, _assemble_m2v_lumped_inv) against the
oracle's restatements of the reference kernels, on seeded multi-column
inputs, and the reference tests' known answers through the C ABI."""
import json

import numpy as np
import pytest

from lfric_core_b200 import api
from lfric_core_b200.api import R_DOUBLE, R_SINGLE, ColumnwiseOperator, Field, LocalOperator
from tests import ora_helpers as oh
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

NCELL, NL = 700, 20
TOL = {R_DOUBLE: 1e-13, R_SINGLE: 2e-6}
DT = {R_DOUBLE: np.float64, R_SINGLE: np.float32}


def cma(ctx, kind, p, ncell=NCELL):
    return ColumnwiseOperator(ctx, kind, ncell, p["nrow"], p["ncol"], p["bw"], p["alpha"],
                              p["beta"], p["gm"], p["gp"], np.arange(1, p["nrow"] + 1),
                              np.arange(1, p["ncol"] + 1))


def space_map(ncell, nl, ndf, nface):
    """A valid LMA dofmap (ncell, ndf) for a space with nface dofs on
    layer faces (Wtheta, W2v: nlev = nl + 1) or per-cell entities."""
    if nface:
        nlev = nl + 1
        m = np.array([[c * nlev + d for d in range(ndf)] for c in range(ncell)])
        return m, ncell, nlev
    m = np.array([[(c * ndf + d) * nl for d in range(ndf)] for c in range(ncell)])
    return m, ncell * ndf, nl


def lma(ctx, kind, ls, to, frm, ncell=NCELL, nl=NL):
    mt, et, lt = space_map(ncell, nl, *to)
    mf, ef, lf = space_map(ncell, nl, *frm)
    return LocalOperator(ctx, kind, ncell, nl, np.asfortranarray(ls).ravel(order="F"), mt, et, lt,
                         mf, ef, lf)


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("kind", [R_DOUBLE, R_SINGLE])
def test_assemble_against_oracle(ctx, kind):
    rng = np.random.default_rng(21)
    cases = [  # (ndf_to, ndf_from, to (ndf, nface), from (ndf, nface), size args)
        ((2, 1), (2, 1), (NL, 2, 2, 1, 0, 1, 0), (2, 0, 1), (2, 0, 1)),   # Wtheta -> Wtheta
        ((1, 0), (2, 1), (NL, 1, 2, 0, 1, 1, 0), (1, 1, 0), (2, 0, 1)),   # W3 <- Wtheta
        ((2, 1), (1, 0), (NL, 2, 1, 1, 0, 0, 1), (2, 0, 1), (1, 1, 0)),   # Wtheta <- W3
    ]
    for to, frm, size, cbt, cbf in cases:
        p = oh.cma_size(*size)
        ls = rng.standard_normal((NCELL * NL, to[0], frm[0]))
        A = lma(ctx, kind, ls, to, frm)
        C = cma(ctx, kind, p)
        cb_to, cb_from = oh.banded_dofmap(NL, *cbt), oh.banded_dofmap(NL, *cbf)
        C.assemble(A, cb_to, cb_from)
        ref = oh.cma_asm(ls.astype(DT[kind]), p, NCELL, NL, cb_to, cb_from, DT[kind])
        assert rel(C.get(), ref) < TOL[kind], size


def test_reassembly_reuses_the_row_lists(ctx):
    """Assembling one operator again from new element matrices on the same
    dofmaps (what every timestep does) reuses the operator's row lists and
    still matches the oracle, as does the first assembly."""
    rng = np.random.default_rng(24)
    p = oh.cma_size(NL, 1, 2, 0, 1, 1, 0)                       # W3 <- Wtheta
    cb_to, cb_from = oh.banded_dofmap(NL, 1, 1, 0), oh.banded_dofmap(NL, 2, 0, 1)
    C = cma(ctx, R_DOUBLE, p)
    for _ in range(3):
        ls = rng.standard_normal((NCELL * NL, 1, 2))
        C.assemble(lma(ctx, R_DOUBLE, ls, (1, 0), (2, 1)), cb_to, cb_from)
        ref = oh.cma_asm(ls, p, NCELL, NL, cb_to, cb_from)
        assert rel(C.get(), ref) < TOL[R_DOUBLE]


@pytest.mark.parametrize("kind", [R_DOUBLE, R_SINGLE])
def test_multiply_and_scaled_add_against_oracle(ctx, kind):
    rng = np.random.default_rng(22)
    dt = DT[kind]
    pT3 = oh.cma_size(NL, 2, 1, 1, 0, 0, 1)
    p3T = oh.cma_size(NL, 1, 2, 0, 1, 1, 0)
    pTT = oh.cma_prod_size(pT3, p3T)
    p33 = oh.cma_size(NL, 1, 1, 0, 1, 0, 1)
    p33x = oh.cma_prod_size(p3T, pT3)
    DTb = rng.standard_normal((pT3["bw"], pT3["nrow"], NCELL))
    Db = rng.standard_normal((p3T["bw"], p3T["nrow"], NCELL))
    C0 = rng.standard_normal((pTT["bw"], pTT["nrow"], NCELL))
    A = ColumnwiseOperator(ctx, kind, NCELL, pT3["nrow"], pT3["ncol"], pT3["bw"], pT3["alpha"],
                           pT3["beta"], pT3["gm"], pT3["gp"], np.arange(1, pT3["nrow"] + 1),
                           np.arange(1, pT3["ncol"] + 1), DTb.ravel(order="F"))
    B = ColumnwiseOperator(ctx, kind, NCELL, p3T["nrow"], p3T["ncol"], p3T["bw"], p3T["alpha"],
                           p3T["beta"], p3T["gm"], p3T["gp"], np.arange(1, p3T["nrow"] + 1),
                           np.arange(1, p3T["ncol"] + 1), Db.ravel(order="F"))
    C = ColumnwiseOperator(ctx, kind, NCELL, pTT["nrow"], pTT["ncol"], pTT["bw"], pTT["alpha"],
                           pTT["beta"], pTT["gm"], pTT["gp"], np.arange(1, pTT["nrow"] + 1),
                           np.arange(1, pTT["ncol"] + 1), C0.ravel(order="F"))
    C.multiply(A, B)                                  # C += D^T D
    ref = oh.cma_mul(DTb.astype(dt), pT3, Db.astype(dt), p3T, C0.astype(dt), pTT, NCELL)
    assert rel(C.get(), ref) < TOL[kind]
    # scaled add on W3: E = a M + b (D D^T)
    Mb = rng.standard_normal((p33["bw"], p33["nrow"], NCELL))
    Pb = rng.standard_normal((p33x["bw"], p33x["nrow"], NCELL))
    M = ColumnwiseOperator(ctx, kind, NCELL, p33["nrow"], p33["ncol"], p33["bw"], p33["alpha"],
                           p33["beta"], p33["gm"], p33["gp"], np.arange(1, p33["nrow"] + 1),
                           np.arange(1, p33["ncol"] + 1), Mb.ravel(order="F"))
    P = ColumnwiseOperator(ctx, kind, NCELL, p33x["nrow"], p33x["ncol"], p33x["bw"],
                           p33x["alpha"], p33x["beta"], p33x["gm"], p33x["gp"],
                           np.arange(1, p33x["nrow"] + 1), np.arange(1, p33x["ncol"] + 1),
                           Pb.ravel(order="F"))
    E = cma(ctx, kind, p33x)
    E.scaled_add(M, P, 2.4, 3.7)
    ref = oh.cma_scaledadd(Mb.astype(dt), p33, Pb.astype(dt), p33x, p33x, NCELL, 2.4, 3.7)
    assert rel(E.get(), ref) < TOL[kind]


@pytest.mark.parametrize("kind", [R_DOUBLE, R_SINGLE])
def test_products_of_wider_bands_against_oracle(ctx, kind):
    """C += A B for W3 tridiagonal factors (spans 3 and 5: the kernel with
    template span bounds 4 and 8) and for their pentadiagonal products
    (spans 5 and 9: the general kernel), against the oracle."""
    rng = np.random.default_rng(24)
    dt = DT[kind]
    p3T = oh.cma_size(NL, 1, 2, 0, 1, 1, 0)
    pT3 = oh.cma_size(NL, 2, 1, 1, 0, 0, 1)
    p3 = oh.cma_prod_size(p3T, pT3)                   # W3 <- W3, bandwidth 3
    p5 = oh.cma_prod_size(p3, p3)                     # bandwidth 5
    p9 = oh.cma_prod_size(p5, p5)                     # bandwidth 9

    def op(p, bands):
        return ColumnwiseOperator(ctx, kind, NCELL, p["nrow"], p["ncol"], p["bw"], p["alpha"],
                                  p["beta"], p["gm"], p["gp"], np.arange(1, p["nrow"] + 1),
                                  np.arange(1, p["ncol"] + 1), bands.ravel(order="F"))
    for pa, pc in ((p3, p5), (p5, p9)):
        Ab = rng.standard_normal((pa["bw"], pa["nrow"], NCELL))
        Bb = rng.standard_normal((pa["bw"], pa["nrow"], NCELL))
        C0 = rng.standard_normal((pc["bw"], pc["nrow"], NCELL))
        C = op(pc, C0)
        C.multiply(op(pa, Ab), op(pa, Bb))
        ref = oh.cma_mul(Ab.astype(dt), pa, Bb.astype(dt), pa, C0.astype(dt), pc, NCELL)
        assert rel(C.get(), ref) < TOL[kind]
        C.multiply(op(pa, Ab), op(pa, Bb))            # same shapes: the check is kept
        ref = oh.cma_mul(Ab.astype(dt), pa, Bb.astype(dt), pa, ref, pc, NCELL)
        assert rel(C.get(), ref) < TOL[kind]


@pytest.mark.parametrize("kind", [R_DOUBLE, R_SINGLE])
def test_hmht_with_two_w3_dofs_per_cell(ctx, kind):
    """asm_diag_hmht on a W3 space of two interior dofs per cell: two
    entries per row on a three-wide band (the unrolled kernel's bound of
    four entries), against the oracle."""
    rng = np.random.default_rng(25)
    dt = DT[kind]
    p = oh.cma_size(NL, 2, 2, 0, 2, 0, 2)
    dh = rng.standard_normal((NCELL * NL, 2, 4))
    m2h = rng.standard_normal((NCELL * NL, 4, 4))
    for d in range(4):
        m2h[:, d, d] = 1.0 + rng.random(NCELL * NL)
    Dh = lma(ctx, kind, dh, (2, 0), (4, 0))
    M2h = lma(ctx, kind, m2h, (4, 0), (4, 0))
    H = cma(ctx, kind, p)
    cb = oh.banded_dofmap(NL, 2, 2, 0)
    H.assemble_diag_hmht(Dh, M2h, cb)
    ref = oh.cma_hmht(dh.astype(dt), m2h.astype(dt), p, NCELL, NL, cb, dt)
    assert rel(H.get(), ref) < TOL[kind] * 10


@pytest.mark.parametrize("kind", [R_DOUBLE, R_SINGLE])
def test_hmht_and_m2v_against_oracle(ctx, kind):
    rng = np.random.default_rng(23)
    dt = DT[kind]
    p33 = oh.cma_size(NL, 1, 1, 0, 1, 0, 1)
    dh = rng.standard_normal((NCELL * NL, 1, 4))
    m2h = rng.standard_normal((NCELL * NL, 4, 4))
    for d in range(4):
        m2h[:, d, d] = 1.0 + rng.random(NCELL * NL)
    Dh = lma(ctx, kind, dh, (1, 0), (4, 0))
    M2h = lma(ctx, kind, m2h, (4, 0), (4, 0))
    H = cma(ctx, kind, p33)
    cb3 = oh.banded_dofmap(NL, 1, 1, 0)
    H.assemble_diag_hmht(Dh, M2h, cb3)
    ref = oh.cma_hmht(dh.astype(dt), m2h.astype(dt), p33, NCELL, NL, cb3, dt)
    assert rel(H.get(), ref) < TOL[kind] * 10
    # lumped inverse of a W2v mass matrix
    pvv = oh.cma_size(NL, 2, 2, 1, 0, 1, 0)
    mv = np.abs(rng.standard_normal((NCELL * NL, 2, 2))) + 0.1
    Mv = lma(ctx, kind, mv, (2, 1), (2, 1))
    L = cma(ctx, kind, pvv)
    cbv = oh.banded_dofmap(NL, 2, 0, 1)
    L.assemble_m2v_lumped_inv(Mv, cbv)
    ref = oh.cma_m2v(mv.astype(dt), pvv, NCELL, NL, cbv, dt)
    assert rel(L.get(), ref) < TOL[kind] * 10


def test_reference_known_answers_on_device(ctx):
    """The reference tests' answers through the C ABI (one column)."""
    g = json.loads((GOLDEN / "cma_assembly_kat.json").read_text())
    nl = g["nlayers"]
    pTT = oh.cma_size(nl, 2, 2, 1, 0, 1, 0)
    ls = np.tile(np.array(g["asm_stencil_fortran_order"]).reshape(2, 2, order="F"), (nl, 1, 1))
    A = lma(ctx, R_DOUBLE, ls, (2, 1), (2, 1), ncell=1, nl=nl)
    C = cma(ctx, R_DOUBLE, pTT, ncell=1)
    cb = oh.banded_dofmap(nl, 2, 0, 1)
    C.assemble(A, cb, cb)
    cm = C.get()
    assert np.allclose(cm[1:3, 0, 0], g["asm_first_row"], rtol=0, atol=1e-15)
    assert np.allclose(cm[:, 1, 0], g["asm_interior_row"], rtol=0, atol=1e-15)
    assert np.allclose(cm[0:2, -1, 0], g["asm_last_row"], rtol=0, atol=1e-15)
    # lumped inverse
    L = cma(ctx, R_DOUBLE, pTT, ncell=1)
    L.assemble_m2v_lumped_inv(A, cb)
    want = np.full(pTT["nrow"], g["m2v_interior_rows"])
    want[[0, -1]] = g["m2v_end_rows"]
    assert np.allclose(L.get()[0, :, 0], want, rtol=1e-14, atol=0)
    # diag hmht
    p33 = oh.cma_size(nl, 1, 1, 0, 1, 0, 1)
    rho, sigma = np.array(g["hmht_rho"]), np.array(g["hmht_sigma"])
    Dh = lma(ctx, R_DOUBLE, np.tile(rho.reshape(1, 1, 4), (nl, 1, 1)), (1, 0), (4, 0), 1, nl)
    M2h = lma(ctx, R_DOUBLE, np.tile(np.diag(sigma)[None], (nl, 1, 1)), (4, 0), (4, 0), 1, nl)
    H = cma(ctx, R_DOUBLE, p33, ncell=1)
    H.assemble_diag_hmht(Dh, M2h, oh.banded_dofmap(nl, 1, 1, 0))
    assert np.allclose(H.get()[0, :, 0], np.sum(rho ** 2 / sigma), rtol=1e-14, atol=0)


def test_assembled_operator_line_solve(ctx):
    """Assemble a Wtheta tridiagonal (mass-like stencils plus a diagonal
    shift) from element matrices and solve with it: appinv of the assembled
    operator against a dense solve per column."""
    rng = np.random.default_rng(24)
    p = oh.cma_size(NL, 2, 2, 1, 0, 1, 0)
    ls = rng.random((NCELL * NL, 2, 2)) * 0.2
    ls[:, 0, 0] += 1.0
    ls[:, 1, 1] += 1.0
    A = lma(ctx, R_DOUBLE, ls, (2, 1), (2, 1))
    C = cma(ctx, R_DOUBLE, p)
    cb = oh.banded_dofmap(NL, 2, 0, 1)
    C.assemble(A, cb, cb)
    nlev = NL + 1
    x = rng.standard_normal(NCELL * nlev)
    X = api.field_from(ctx, x, NCELL, nlev)
    Y = Field(ctx, R_DOUBLE, NCELL, nlev)
    C.apply_inverse(Y, X)
    y = Y.export().reshape(NCELL, nlev)
    cm = C.get()
    for c in (0, 1, NCELL // 2, NCELL - 1):
        dense = oh.cma_dense(cm, p, c)
        assert np.allclose(dense @ y[c], x.reshape(NCELL, nlev)[c], rtol=0, atol=1e-12)

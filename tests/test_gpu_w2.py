"""W2 intergrid transfers on the device (lfg_w2_*) against the oracle's
restatements of restrict_w2 / restrict_w2h / restrict_w2v / prolong_w2 /
weights_prolong_w2, on a planar mesh of coarse cells refined 2 x 2 with a
conforming W2 dofmap (shared faces, face selectors splitting them), and
the reference tests' known answers through the C ABI."""
import json

import numpy as np
import pytest

from lfric_core_b200 import api
from lfric_core_b200.api import R_DOUBLE, R_SINGLE, Field, field_from
from tests import ora_helpers as oh
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu


def w2_space(ncx, ncy, nl):
    """A conforming W2 dofmap on an ncx x ncy planar grid: x-normal faces
    (ncx+1) x ncy, y-normal faces ncx x (ncy+1), a column of nl dofs each,
    then one vertical column of nl+1 dofs per cell (B, T = B + 1).  Cell
    (i, j): i west to east, j north to south.  Returns (map (ncell, 6),
    undf, selectors ew, ns)."""
    nxf = (ncx + 1) * ncy
    nyf = ncx * (ncy + 1)
    xface = lambda i, j: j * (ncx + 1) + i
    yface = lambda i, j: nxf + j * ncx + i
    ncell = ncx * ncy
    m = np.zeros((ncell, 6), dtype=np.int32)
    ew = np.ones(ncell, dtype=np.int32)
    ns = np.ones(ncell, dtype=np.int32)
    base_v = (nxf + nyf) * nl
    for j in range(ncy):
        for i in range(ncx):
            c = j * ncx + i
            m[c] = [xface(i, j) * nl, yface(i, j + 1) * nl, xface(i + 1, j) * nl,
                    yface(i, j) * nl, base_v + c * (nl + 1), base_v + c * (nl + 1) + 1]
            ew[c] = 2 if i == ncx - 1 else 1     # the east-most cell also owns E
            ns[c] = 2 if j == 0 else 1           # the north-most cell also owns N
    return m, base_v + ncell * (nl + 1), ew, ns


def refine(ncx, ncy):
    """cell_map (ncoarse, 2, 2) [y][x] of the 2 x 2 refinement."""
    cm = np.zeros((ncx * ncy, 2, 2), dtype=np.int32)
    for j in range(ncy):
        for i in range(ncx):
            for y in range(2):
                for x in range(2):
                    cm[j * ncx + i, y, x] = (2 * j + y) * (2 * ncx) + 2 * i + x
    return cm


NCX, NCY, NL = 9, 7, 12


@pytest.fixture(scope="module")
def setup(ctx):
    mc, undf_c, ew, ns = w2_space(NCX, NCY, NL)
    mf, undf_f, _, _ = w2_space(2 * NCX, 2 * NCY, NL)
    cm = refine(NCX, NCY)
    ig = api.Intergrid(ctx, cm, mf.shape[0])
    W = api.W2Map(ig, NL, mc, undf_c, mf, undf_f, ew, ns)
    return dict(mc=mc, mf=mf, undf_c=undf_c, undf_f=undf_f, ew=ew, ns=ns, cm=cm, ig=ig, W=W)


def oracle_restrict(s, kind, fine, dtype):
    """Per coarse cell, the oracle's restriction (1-based maps)."""
    out = np.zeros(s["undf_c"], dtype=dtype)
    mf1, mc1 = s["mf"] + 1, s["mc"] + 1
    for C in range(s["cm"].shape[0]):
        cell_map = (s["cm"][C].T + 1)                # Fortran cell_map(x, y), 1-based
        part = oh.w2_restrict(kind, NL, 2, 2, mf1, mc1[C], fine, s["undf_c"],
                              s["ew"][C], s["ns"][C], dtype=dtype, cell_map=cell_map)
        touched = part != 0
        out[touched] = part[touched]
    return out


@pytest.mark.parametrize("kind,mode,dtype,tol", [
    ("w2", api.W2_FULL, np.float64, 1e-15), ("w2", api.W2_FULL, np.float32, 1e-6),
    ("w2h", api.W2_H, np.float64, 1e-15)])
def test_w2_restrict_against_oracle(ctx, setup, kind, mode, dtype, tol):
    s = setup
    rng = np.random.default_rng(31)
    fine = (rng.random(s["undf_f"]) + 0.5).astype(dtype)   # non-zero: every written dof shows
    ref = oracle_restrict(s, kind, fine, dtype)
    kindc = R_DOUBLE if dtype == np.float64 else R_SINGLE
    F = field_from(ctx, fine, s["undf_f"], 1, kind=kindc)
    Cf = Field(ctx, kindc, s["undf_c"], 1)
    Cf.set_scalar(0.0)
    s["W"].restrict(mode, Cf, F)
    got = Cf.export()
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))
    # every coarse face dof was written exactly by its owner: no zero left
    faces = np.zeros(s["undf_c"], dtype=bool)
    for C in range(s["mc"].shape[0]):
        for df in range(4 if kind == "w2h" else 5):
            n = NL + 1 if df == 4 else NL
            faces[s["mc"][C, df]:s["mc"][C, df] + n] = True
    assert np.all(got[faces] != 0)


def test_w2v_restrict_against_oracle(ctx):
    ncx, ncy = 6, 5
    nl = 10
    # W2V: one column of nl+1 dofs per cell, map (B, T)
    def v_space(nc):
        return np.array([[c * (nl + 1), c * (nl + 1) + 1] for c in range(nc)], dtype=np.int32)
    mc, mf = v_space(ncx * ncy), v_space(4 * ncx * ncy)
    cm = refine(ncx, ncy)
    ig = api.Intergrid(ctx, cm, mf.shape[0])
    W = api.W2Map(ig, nl, mc, mc.shape[0] * (nl + 1), mf, mf.shape[0] * (nl + 1))
    rng = np.random.default_rng(32)
    fine = rng.standard_normal(mf.shape[0] * (nl + 1))
    Cf = Field(ctx, R_DOUBLE, mc.shape[0] * (nl + 1), 1)
    W.restrict(api.W2_V, Cf, field_from(ctx, fine, fine.size, 1))
    ref = np.zeros(mc.shape[0] * (nl + 1))
    for C in range(mc.shape[0]):
        part = oh.w2_restrict("w2v", nl, 2, 2, mf + 1, mc[C] + 1, fine, ref.size,
                              cell_map=cm[C].T + 1)
        sl = slice(mc[C, 0], mc[C, 0] + nl + 1)
        ref[sl] = part[sl]
    assert np.max(np.abs(Cf.export() - ref)) < 1e-14


def test_w2_prolong_against_oracle(ctx, setup):
    s = setup
    rng = np.random.default_rng(33)
    Wt = Field(ctx, R_DOUBLE, s["undf_f"], 1)
    Wt.set_scalar(0.0)
    s["W"].prolong_weights(Wt)
    w = Wt.export()
    wref = np.zeros(s["undf_f"])
    for C in range(s["cm"].shape[0]):
        wref = oh.w2_weights(NL, 2, 2, s["mf"] + 1, s["undf_f"], w0=wref,
                             cell_map=s["cm"][C].T + 1)
    assert np.array_equal(w, wref)
    coarse = rng.standard_normal(s["undf_c"])
    Fo = Field(ctx, R_DOUBLE, s["undf_f"], 1)
    Fo.set_scalar(0.0)
    s["W"].prolong(Fo, field_from(ctx, coarse, s["undf_c"], 1), Wt)
    ref = np.zeros(s["undf_f"])
    for C in range(s["cm"].shape[0]):
        ref = oh.w2_prolong(NL, 2, 2, s["mf"] + 1, s["mc"][C] + 1, coarse, wref, ref,
                            cell_map=s["cm"][C].T + 1)
    assert np.max(np.abs(Fo.export() - ref)) < 1e-14


def test_w2_reference_known_answers_on_device(ctx):
    g = json.loads((GOLDEN / "w2_intergrid_kat.json").read_text())
    for name, mode in (("restrict_w2", api.W2_FULL), ("restrict_w2h", api.W2_H),
                       ("restrict_w2v", api.W2_V)):
        k = g[name]
        nx, ny = k["nx"], k["ny"]
        cm = np.array([[[x + y * nx for x in range(nx)] for y in range(ny)]], dtype=np.int32)
        ig = api.Intergrid(ctx, cm, nx * ny)
        mf = np.array(k["map_f"]) - 1
        mc = np.array([k["map_c"]]) - 1
        sel = None if mode == api.W2_V else [k["face_selector"]]
        W = api.W2Map(ig, k["nlayers"], mc, len(k["answer"]), mf, len(k["fine"]), sel, sel)
        Cf = Field(ctx, R_DOUBLE, len(k["answer"]), 1)
        Cf.set_scalar(0.0)
        W.restrict(mode, Cf, field_from(ctx, np.array(k["fine"]), len(k["fine"]), 1))
        assert np.allclose(Cf.export(), k["answer"], rtol=0, atol=g["tol"]), name
    k = g["prolong_w2"]
    nx, ny = k["nx"], k["ny"]
    cm = np.array([[[x + y * nx for x in range(nx)] for y in range(ny)]], dtype=np.int32)
    ig = api.Intergrid(ctx, cm, nx * ny)
    W = api.W2Map(ig, k["nlayers"], np.array([k["map_c"]]) - 1, len(k["coarse"]),
                  np.array(k["map_f"]) - 1, len(k["answer"]), [2], [2])
    Wt = Field(ctx, R_DOUBLE, len(k["answer"]), 1)
    Wt.set_scalar(0.0)
    W.prolong_weights(Wt)
    assert np.allclose(Wt.export(), g["weights_prolong_w2"]["answer"], rtol=0, atol=g["tol"])
    Fo = Field(ctx, R_DOUBLE, len(k["answer"]), 1)
    Fo.set_scalar(0.0)
    W.prolong(Fo, field_from(ctx, np.array(k["coarse"]), len(k["coarse"]), 1), Wt)
    assert np.allclose(Fo.export(), k["answer"], rtol=0, atol=g["tol"])

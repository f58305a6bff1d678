"""Cubed-sphere generator against the reference's UGRID test meshes (CPU)."""
import json

import numpy as np
import pytest

from tests.conftest import GOLDEN
from lfric_core_b200.mesh import cubed_sphere, coarsen_map, extrusion, extruded_mesh
from lfric_core_b200.problems import helmholtz_problem

MESH = json.loads((GOLDEN / "mesh_mg_kat.json").read_text())


@pytest.mark.parametrize("name,n", [("C4", 4), ("C8", 8)])
def test_links_and_corners_match_reference(name, n):
    ref = MESH["meshes"][name]
    cs = cubed_sphere(n)
    assert np.array_equal(cs.face_links, np.array(ref["face_links_WSEN"]))
    lon = np.array(ref["corner_lon_SW_SE_NE_NW"])
    lat = np.array(ref["corner_lat_SW_SE_NE_NW"])
    xyz = np.stack([np.cos(np.radians(lat)) * np.cos(np.radians(lon)),
                    np.cos(np.radians(lat)) * np.sin(np.radians(lon)),
                    np.sin(np.radians(lat))], axis=-1)
    assert np.abs(cs.vertex_xyz[cs.cell_vertices] - xyz).max() < 1e-10
    c = cs.cell_centre_xyz()
    flon = np.degrees(np.arctan2(c[:, 1], c[:, 0]))
    flat = np.degrees(np.arcsin(c[:, 2]))
    assert np.abs(flat - np.array(ref["face_lat"])).max() < 1e-9
    dl = np.abs(flon - np.array(ref["face_lon"])) % 360
    assert np.minimum(dl, 360 - dl).max() < 1e-9


@pytest.mark.parametrize("pair,nf", [("C4_C8", 8), ("C8_C16", 16)])
def test_coarsening_maps_match_reference(pair, nf):
    assert np.array_equal(coarsen_map(nf), np.array(MESH["maps"][pair]))


@pytest.mark.parametrize("n", [2, 4, 6, 24])
def test_topology(n):
    cs = cubed_sphere(n)
    assert cs.ncell == 6 * n * n and cs.nvert == 6 * n * n + 2
    L = cs.face_links
    # symmetric adjacency: every neighbour points back
    for f in range(4):
        assert np.all((L[L[:, f]] == np.arange(cs.ncell)[:, None]).any(axis=1))
    assert np.all(L != np.arange(cs.ncell)[:, None])


@pytest.mark.parametrize("n", [4, 8, 24])
def test_children_share_the_coarse_frame(n):
    """A child's neighbour across side f is outside its coarse cell exactly
    when the child sits on side f, and is then a child of the coarse
    neighbour across f (what the Galerkin coarsening relies on)."""
    fine, coarse = cubed_sphere(n), cubed_sphere(n // 2)
    ch = coarsen_map(n)
    parent = np.empty(fine.ncell, dtype=int)
    for C in range(coarse.ncell):
        parent[ch[C].ravel()] = C
    side_slots = {0: [(0, 0), (1, 0)], 1: [(1, 0), (1, 1)], 2: [(0, 1), (1, 1)], 3: [(0, 0), (0, 1)]}
    for C in range(coarse.ncell):
        for f in range(4):
            on_side = set(side_slots[f])
            for y in range(2):
                for x in range(2):
                    nb = fine.face_links[ch[C, y, x], f]
                    if (y, x) in on_side:
                        assert parent[nb] == coarse.face_links[C, f]
                    else:
                        assert parent[nb] == C


def test_extrusions():
    z = extrusion(70, 80e3, "quadratic")
    assert z[0] == 0 and abs(z[-1] - 80e3) < 1e-9 and np.all(np.diff(z) > 0)
    assert np.allclose(np.diff(extrusion(20, 20e3, "uniform")), 1000.0)
    m = extruded_mesh(4, 3, 3e3)
    d = m.w0_dofmap()
    assert d.shape == (96, 8) and np.all(d[:, 4:] == d[:, :4] + 1)


def test_helmholtz_operator_is_spd_and_symmetric():
    prob = helmholtz_problem(2, 5, seed=7, mg_levels=2)
    n, nl = prob.ncol, prob.nlayers
    cm = prob.cm.reshape(n, nl, 3)
    hf = prob.hf.reshape(n, nl, 4)
    A = np.zeros((n * nl, n * nl))
    for c in range(n):
        for k in range(nl):
            i = c * nl + k
            A[i, i] = cm[c, k, 1]
            if k > 0:
                A[i, i - 1] = cm[c, k, 0]
            if k < nl - 1:
                A[i, i + 1] = cm[c, k, 2]
            for f in range(4):
                A[i, prob.links[c, f] * nl + k] -= hf[c, k, f]
    assert np.allclose(A, A.T, atol=1e-12)
    assert np.linalg.eigvalsh(A).min() > 0

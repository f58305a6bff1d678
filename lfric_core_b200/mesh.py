"""Equiangular cubed-sphere meshes, extrusions, dofmaps and multigrid maps.

Host-side set-up for the solver hot path (numpy, run once per mesh).  The
conventions follow the reference mesh generator and infrastructure:

* panels 1-4 form the equatorial belt (panel 1 centred on lon 0, lat 0),
  panel 5 is the north cap and panel 6 the south cap, with panel-to-panel
  links W,S,E,N = [4,6,2,5], [1,6,3,5], [2,6,4,5], [3,6,1,5], [1,2,3,4],
  [1,4,3,2] (mesh_tools/source/support/gencube_ps_mod.F90:378-385);
* cells in a panel are numbered row-major from the panel's NW corner
  (gencube_ps_mod.F90:364-374);
* cell neighbours are stored W,S,E,N and cell corners SW,SE,NE,NW, the
  order of the reference element constants SWB=1, SEB=2, NEB=3, NWB=4
  (infrastructure/source/mesh/reference_element_mod.F90:346-349);
* equiangular gnomonic coordinates (gencube_ps_mod.F90:887-1113);
* a multigrid cell map stores, for each coarse cell, the fine cells as
  cell_map(x, y) with x running W->E and y running N->S (row 1 is north),
  as in the mesh_C32_MG.nc maps and the diagram in
  components/science/source/kernel/inter_mesh/sci_prolong_w0_kernel_mod.F90:112-124.

All indices returned here are 0-based.  The C-ABI takes 0-based indices; the
Fortran shim adds or removes the offset of one at the boundary.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

EARTH_RADIUS = 6.371e6

# (centre, east, north) unit vectors of each panel's local frame.
_PANEL_FRAMES = {
    1: ((1, 0, 0), (0, 1, 0), (0, 0, 1)),
    2: ((0, 1, 0), (-1, 0, 0), (0, 0, 1)),
    3: ((-1, 0, 0), (0, -1, 0), (0, 0, 1)),
    4: ((0, -1, 0), (1, 0, 0), (0, 0, 1)),
    5: ((0, 0, 1), (-1, 0, 0), (0, -1, 0)),
    6: ((0, 0, -1), (-1, 0, 0), (0, 1, 0)),
}

W, S, E, N = 0, 1, 2, 3
SWB, SEB, NEB, NWB = 0, 1, 2, 3

# The reference orients cells on panels 3, 4 and 5 with their local frame
# turned by a quarter turn relative to the panel's own (east, north) frame:
# neighbour and corner lists start one (panels 3, 4) or three (panel 5)
# entries later, and the 2x2 cell maps are turned to match (checked against
# the reference meshes in infrastructure/unit-test/data/mesh_C32_MG.nc).
_PANEL_ROLL = {1: 0, 2: 0, 3: 1, 4: 1, 5: 3, 6: 0}


@dataclass
class CubedSphere:
    """A C_n cubed-sphere surface mesh."""

    n: int
    face_links: np.ndarray      # (ncell, 4) int32 neighbours W,S,E,N
    cell_vertices: np.ndarray   # (ncell, 4) int32 corners SW,SE,NE,NW
    vertex_xyz: np.ndarray      # (nvert, 3) float64 on the unit sphere
    panel: np.ndarray           # (ncell,) int32 panel number 1..6

    @property
    def ncell(self) -> int:
        return int(self.face_links.shape[0])

    @property
    def nvert(self) -> int:
        return int(self.vertex_xyz.shape[0])

    def vertex_lonlat(self) -> np.ndarray:
        x, y, z = self.vertex_xyz.T
        return np.stack([np.degrees(np.arctan2(y, x)),
                         np.degrees(np.arcsin(np.clip(z, -1, 1)))], axis=1)

    def cell_centre_xyz(self) -> np.ndarray:
        c = self.vertex_xyz[self.cell_vertices].mean(axis=1)
        return c / np.linalg.norm(c, axis=1, keepdims=True)


def cubed_sphere(n: int) -> CubedSphere:
    """Build the equiangular C_n mesh (6 n^2 cells, 6 n^2 + 2 vertices)."""
    if n < 1:
        raise ValueError("cubed_sphere: n must be >= 1")
    ncell = 6 * n * n
    # Integer lattice position of every (panel, i, j) vertex on the cube
    # surface: n*centre + (2i-n)*east + (n-2j)*north.  Shared edge vertices
    # coincide exactly, which gives an exact de-duplication.
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="xy")
    keys = []
    for p in range(1, 7):
        c, e, nn = (np.array(v, dtype=np.int64) for v in _PANEL_FRAMES[p])
        lat = (n * c[None, None, :] + (2 * ii - n)[..., None] * e
               + (n - 2 * jj)[..., None] * nn)
        keys.append(lat)
    keys = np.stack(keys)                       # (6, n+1, n+1, 3)
    flat = keys.reshape(-1, 3)
    code = ((flat[:, 0] + n) * (2 * n + 1) + (flat[:, 1] + n)) * (2 * n + 1) + (flat[:, 2] + n)
    # Number vertices by first appearance in (panel, row, column) order.
    _, first, inverse = np.unique(code, return_index=True, return_inverse=True)
    order = np.argsort(first)
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    vid = rank[inverse].reshape(6, n + 1, n + 1)   # vid[p, j, i]
    nvert = order.size
    assert nvert == ncell + 2, (nvert, ncell)

    # Equiangular coordinates of each lattice point.
    xyz = np.empty((nvert, 3))
    ang = -math.pi / 4 + (math.pi / 2) * np.arange(n + 1) / n
    t = np.tan(ang)
    for p in range(1, 7):
        c, e, nn = (np.array(v, dtype=np.float64) for v in _PANEL_FRAMES[p])
        te = t[ii]          # east coordinate, i = 0 is west
        tn = t[::-1][jj]    # north coordinate, j = 0 is north
        pts = c[None, None, :] + te[..., None] * e + tn[..., None] * nn
        pts /= np.linalg.norm(pts, axis=-1, keepdims=True)
        xyz[vid[p - 1].ravel()] = pts.reshape(-1, 3)

    cj, ci = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    cell_vertices = np.empty((ncell, 4), dtype=np.int32)
    panel = np.empty(ncell, dtype=np.int32)
    for p in range(6):
        sl = slice(p * n * n, (p + 1) * n * n)
        cell_vertices[sl, SWB] = vid[p, cj + 1, ci].ravel()
        cell_vertices[sl, SEB] = vid[p, cj + 1, ci + 1].ravel()
        cell_vertices[sl, NEB] = vid[p, cj, ci + 1].ravel()
        cell_vertices[sl, NWB] = vid[p, cj, ci].ravel()
        panel[sl] = p + 1

    # Neighbours across each edge: W=(SW,NW), S=(SW,SE), E=(SE,NE), N=(NW,NE).
    edge_corners = {W: (SWB, NWB), S: (SWB, SEB), E: (SEB, NEB), N: (NWB, NEB)}
    ekeys = []
    for side in (W, S, E, N):
        a, b = edge_corners[side]
        va = cell_vertices[:, a].astype(np.int64)
        vb = cell_vertices[:, b].astype(np.int64)
        ekeys.append(np.minimum(va, vb) * nvert + np.maximum(va, vb))
    ekeys = np.stack(ekeys, axis=1)           # (ncell, 4)
    flat_keys = ekeys.ravel()
    owner = np.repeat(np.arange(ncell), 4)
    srt = np.argsort(flat_keys, kind="stable")
    sk = flat_keys[srt]
    if not np.all(sk[0::2] == sk[1::2]):
        raise RuntimeError("cubed_sphere: every edge must be shared by exactly two cells")
    a_idx, b_idx = srt[0::2], srt[1::2]
    links = np.empty(ncell * 4, dtype=np.int32)
    links[a_idx] = owner[b_idx]
    links[b_idx] = owner[a_idx]
    links = links.reshape(ncell, 4)
    for p in range(1, 7):
        r = _PANEL_ROLL[p]
        if r:
            sl = slice((p - 1) * n * n, p * n * n)
            links[sl] = np.roll(links[sl], -r, axis=1)
            cell_vertices[sl] = np.roll(cell_vertices[sl], -r, axis=1)
    return CubedSphere(n=n, face_links=links,
                       cell_vertices=cell_vertices, vertex_xyz=xyz, panel=panel)


def coarsen_map(n_fine: int) -> np.ndarray:
    """Fine cells of each coarse cell of C_{n/2} inside C_n.

    Returns an int32 array (ncoarse, 2, 2) indexed [coarse, y, x]; y runs
    N->S and x runs W->E, matching the C16_C32-style maps in the reference's
    multigrid mesh files (Fortran cell_map(x, y)).
    """
    if n_fine % 2:
        raise ValueError("coarsen_map: n_fine must be even")
    nc = n_fine // 2
    out = np.empty((6 * nc * nc, 2, 2), dtype=np.int32)
    J, I = np.meshgrid(np.arange(nc), np.arange(nc), indexing="ij")
    for p in range(6):
        base = p * n_fine * n_fine
        for y in range(2):
            for x in range(2):
                out[p * nc * nc:(p + 1) * nc * nc, y, x] = (
                    base + (2 * J + y) * n_fine + (2 * I + x)).ravel()
        r = _PANEL_ROLL[p + 1]
        if r:
            sl = slice(p * nc * nc, (p + 1) * nc * nc)
            out[sl] = np.rot90(out[sl], 4 - r, axes=(1, 2))
    return out


def extrusion(nlayers: int, domain_top: float, kind: str = "uniform") -> np.ndarray:
    """Level heights (nlayers+1) above the surface.

    uniform: eta_k = k/n; quadratic: eta_k = (k/n)^2
    (infrastructure/source/mesh/extrusion_mod.f90:292-305, 341-354).
    """
    k = np.arange(nlayers + 1, dtype=np.float64) / nlayers
    if kind == "uniform":
        eta = k
    elif kind == "quadratic":
        eta = k * k
    else:
        raise ValueError(f"extrusion: unknown kind {kind!r}")
    return domain_top * eta


@dataclass
class ExtrudedMesh:
    """A cubed sphere extruded over nlayers levels with W3 and W0 dofmaps."""

    surface: CubedSphere
    nlayers: int
    heights: np.ndarray = field(repr=False)
    radius: float = EARTH_RADIUS

    @property
    def ncell(self) -> int:
        return self.surface.ncell

    def w3_dofmap(self) -> np.ndarray:
        """First W3 dof of each column (column-contiguous levels), (ncell,)."""
        return (np.arange(self.ncell, dtype=np.int64) * self.nlayers).astype(np.int64)

    def w0_dofmap(self) -> np.ndarray:
        """W0 dofmap (ncell, 8): bottom corners SW,SE,NE,NW then top corners.

        A vertex column holds nlayers+1 contiguous dofs; dof of level k of
        vertex v is v*(nlayers+1)+k, so the top-corner entry is the bottom
        entry plus one, as in the reference's column-contiguous dofmaps
        (function_space_constructor_helper_functions_mod.F90:1940-2160).
        """
        base = self.surface.cell_vertices.astype(np.int64) * (self.nlayers + 1)
        return np.concatenate([base, base + 1], axis=1)

    def w0_ndof(self) -> int:
        return self.surface.nvert * (self.nlayers + 1)

    def w2_dofmap(self) -> tuple[np.ndarray, int]:
        """Lowest-order W2 dofmap, (ncell, 6) for the faces W, S, E, N, B, T,
        and the number of dofs.

        Numbered as dofmap_setup numbers one partition
        (infrastructure/source/function_space/
        function_space_constructor_helper_functions_mod.F90:1890-2020):
        cells in order; each side face W, S, E, N not numbered yet gets a
        column of nlayers dofs (the neighbour across it shares the column);
        then the cell's vertical faces get one column of nlayers+1 dofs,
        the bottom face at its start and the top face one further, so that
        map(df) + k is the dof of layer k of face df.  0-based.
        """
        links = self.surface.face_links
        ncell, nl = self.ncell, self.nlayers
        m = np.full((ncell, 6), -1, dtype=np.int64)
        nxt = 0
        for c in range(ncell):
            for f in range(4):
                if m[c, f] < 0:
                    m[c, f] = nxt
                    nb = links[c, f]
                    back = [g for g in range(4) if links[nb, g] == c and m[nb, g] < 0]
                    if nb != c and back:
                        m[nb, back[0]] = nxt
                    nxt += nl
            m[c, 4] = nxt
            m[c, 5] = nxt + 1
            nxt += nl + 1
        return m, nxt

    def w2_face_selectors(self) -> tuple[np.ndarray, np.ndarray]:
        """Face selectors (ew, ns) of a W2 restriction onto this mesh: every
        cell writes its W and S faces, and also its E (N) face when the
        neighbour across it does not reach that face as its own W or S
        (ew, ns = 2), so every face is written by at least one of its two
        cells (restrict_w2's loop over face_selector_ew + face_selector_ns
        faces, components/science/source/kernel/inter_mesh/
        sci_restrict_w2_kernel_mod.F90:212-215).  A face that both cells
        reach writes the same value from each: the same fine faces summed."""
        links = self.surface.face_links
        ncell = self.ncell
        ew = np.ones(ncell, dtype=np.int32)
        ns = np.ones(ncell, dtype=np.int32)
        for c in range(ncell):
            for f, sel in ((E, ew), (N, ns)):
                nb = links[c, f]
                back = [g for g in range(4) if links[nb, g] == c]
                if not any(g in (W, S) for g in back):
                    sel[c] = 2
        return ew, ns

    def w0_coords(self) -> np.ndarray:
        """Cartesian coordinates of every W0 dof, (nvert*(nlayers+1), 3)."""
        r = self.radius + self.heights                  # (nl+1,)
        xyz = self.surface.vertex_xyz[:, None, :] * r[None, :, None]
        return xyz.reshape(-1, 3)


def extruded_mesh(n: int, nlayers: int, domain_top: float,
                  kind: str = "uniform", radius: float = EARTH_RADIUS) -> ExtrudedMesh:
    return ExtrudedMesh(surface=cubed_sphere(n), nlayers=nlayers,
                        heights=extrusion(nlayers, domain_top, kind), radius=radius)


def mg_hierarchy(n_fine: int, nlevels: int):
    """Meshes C_n, C_{n/2}, ... and the cell maps between consecutive levels."""
    meshes, maps = [cubed_sphere(n_fine)], []
    n = n_fine
    for _ in range(nlevels - 1):
        maps.append(coarsen_map(n))
        n //= 2
        meshes.append(cubed_sphere(n))
    return meshes, maps

"""Seeded synthetic problems on the extruded cubed sphere (host-side set-up).

The reference's own Helmholtz operator lives outside lfric_core, so the W3
Helmholtz problem solved here is defined by this project, from the
reference's building blocks:

  A = T' - H_off
    T'    : a columnwise-assembled (CMA) tridiagonal operator per column,
            stored as columnwise_matrix(3, nlayers, ncol) (bandwidth 3, the
            W3->W3 layout of infrastructure/source/operator/
            columnwise_operator_mod.f90:401-413), whose diagonal already holds
            the sum of the horizontal face couplings;
    H_off : the symmetric coupling of every cell to its four face neighbours
            on the same level, stored as hface(4, nlayers, ncol) in the
            neighbour order W,S,E,N.

so (A x)(c,k) = sum_j T'(j,k,c) x(c,k-2+j) - sum_f hface(f,k,c) x(nbr_f(c),k).
A is symmetric positive definite: T (the vertical part) is symmetric and
strictly diagonally dominant and the horizontal part is a weighted graph
Laplacian.

Vertical coefficients (one value per interface, shared by the two rows so T
is symmetric): off-diagonal = -u * g_k with u ~ U(0,1) and g_k the mean layer
spacing over the spacing between the centres of layers k and k+1 (the
quadratic extrusion of extrusion_mod.f90:341-354 makes the bottom layers
thin, so their vertical coupling is strong).  T's diagonal is ratio * (|sub|
+ |super|), ratio ~ U(1.5, 3).  Horizontal couplings: h = s * U(0.5, 1.5) *
dz_k / mean(dz) per unique face and level (thick layers couple strongly in the
horizontal).  Right-hand sides are N(0,1).  All draws use numpy's PCG64 from
the given seed.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mesh import EARTH_RADIUS as EARTH_RADIUS_DEFAULT
from .mesh import CubedSphere, coarsen_map, cubed_sphere, extrusion

DEFAULT_TOP = 80.0e3
DEFAULT_H_SCALE = 4.0


@dataclass
class HelmholtzProblem:
    """A W3 Helmholtz operator, right-hand side and multigrid hierarchy.

    Arrays are in the reference layout: column-contiguous fields
    (index c*nlayers + k), cm = columnwise_matrix(3, nlayers, ncol) flattened
    in Fortran order (band fastest), hf = hface(4, nlayers, ncol) flattened in
    Fortran order, links = (ncol, 4) 0-based W,S,E,N neighbours.
    """

    n: int
    nlayers: int
    cm: np.ndarray
    hf: np.ndarray
    links: np.ndarray
    rhs: np.ndarray
    mg_links: list          # links of levels 1.. (coarser meshes)
    mg_child: list          # child[l]: (ncol_{l+1}, 2, 2) cells of level l

    @property
    def ncol(self) -> int:
        return int(self.links.shape[0])

    @property
    def ndof(self) -> int:
        return self.ncol * self.nlayers

    @property
    def nlevels(self) -> int:
        return 1 + len(self.mg_child)


def _unique_faces(links: np.ndarray):
    """(cell, side) pairs of every face once, plus the matching far side."""
    ncol = links.shape[0]
    cells = np.repeat(np.arange(ncol), 4)
    sides = np.tile(np.arange(4), ncol)
    nbrs = links.ravel()
    # side of the neighbour that points back at the cell
    back = np.empty_like(sides)
    lk = links[nbrs]                                  # (4*ncol, 4)
    back[:] = np.argmax(lk == cells[:, None], axis=1)
    own = cells < nbrs
    return cells[own], sides[own], nbrs[own], back[own]


def helmholtz_operator(surface: CubedSphere, nlayers: int, seed: int,
                       top: float = DEFAULT_TOP, stretching: str = "quadratic",
                       h_scale: float = DEFAULT_H_SCALE):
    """Bands cm (3*nl*ncol), couplings hf (4*nl*ncol) and links of A."""
    rng = np.random.default_rng(seed)
    ncol, nl = surface.ncell, nlayers
    z = extrusion(nl, top, stretching)
    dz = np.diff(z)                                    # layer depths (nl,)
    mean_dz = top / nl
    zc = 0.5 * (z[1:] + z[:-1])
    g = mean_dz / np.diff(zc) if nl > 1 else np.zeros(0)   # (nl-1,)
    # Vertical interfaces: one coefficient per (column, interface k|k+1).
    off = -rng.uniform(0.0, 1.0, size=(ncol, nl - 1)) * g[None, :]
    sub = np.zeros((ncol, nl))
    sup = np.zeros((ncol, nl))
    sup[:, :-1] = off
    sub[:, 1:] = off
    ratio = rng.uniform(1.5, 3.0, size=(ncol, nl))
    diag = ratio * (np.abs(sub) + np.abs(sup))
    # A column with a single level has no vertical neighbours.
    diag = np.where(diag == 0.0, ratio, diag)
    # Horizontal couplings, symmetric: draw per unique face.
    links = surface.face_links.astype(np.int32)
    c, s, nb, bk = _unique_faces(links)
    hval = h_scale * rng.uniform(0.5, 1.5, size=(c.size, nl)) * (dz / mean_dz)[None, :]
    hf = np.zeros((ncol, nl, 4))
    hf[c, :, s] = hval
    hf[nb, :, bk] = hval
    diag = diag + hf.sum(axis=2)
    cm = np.stack([sub, diag, sup], axis=2)            # (ncol, nl, 3)
    return (np.ascontiguousarray(cm).ravel(), np.ascontiguousarray(hf).ravel(), links)


def helmholtz_problem(n: int, nlayers: int, seed: int, mg_levels: int = 4,
                      top: float = DEFAULT_TOP, stretching: str = "quadratic",
                      h_scale: float = DEFAULT_H_SCALE, rhs_seed: int | None = None
                      ) -> HelmholtzProblem:
    """Helmholtz operator on C_n x nlayers with a mg_levels-deep hierarchy."""
    surface = cubed_sphere(n)
    cm, hf, links = helmholtz_operator(surface, nlayers, seed, top, stretching, h_scale)
    rng = np.random.default_rng(seed + 1000003 if rhs_seed is None else rhs_seed)
    rhs = rng.standard_normal(surface.ncell * nlayers)
    mg_links, mg_child = [], []
    m = n
    for _ in range(mg_levels - 1):
        if m % 2:
            raise ValueError("helmholtz_problem: n must be divisible by 2^(mg_levels-1)")
        mg_child.append(coarsen_map(m))
        m //= 2
        mg_links.append(cubed_sphere(m).face_links.astype(np.int32))
    return HelmholtzProblem(n=n, nlayers=nlayers, cm=cm, hf=hf, links=links, rhs=rhs,
                            mg_links=mg_links, mg_child=mg_child)


@dataclass
class BatchWorkload:
    """Independent W3 Helmholtz problems: operators[j] and, per problem i,
    the index of its operator and its right-hand side (reference layout)."""

    operators: list
    problem_op: list
    rhs: list

    @property
    def ndof(self) -> int:
        return sum(self.operators[j].ncol * self.operators[j].nlayers for j in self.problem_op)


def batch_workload(seed: int = 5, n_rhs: int = 64, n_shared: int = 48, l_shared: int = 30,
                   n_uneven: int = 32, n_range=(12, 96), l_range=(10, 70)) -> BatchWorkload:
    """n_rhs seeded right-hand sides (seeds seed+i) on one C_{n_shared} x
    l_shared operator, plus n_uneven independent problems with n and L drawn
    uniformly from n_range and l_range (operator and rhs seeds seed+n_rhs+j)."""
    ops = [helmholtz_problem(n_shared, l_shared, seed=seed, mg_levels=1)]
    problem_op, rhs = [], []
    nd = ops[0].ncol * l_shared
    for i in range(n_rhs):
        problem_op.append(0)
        rhs.append(np.random.default_rng(seed + i).standard_normal(nd))
    draw = np.random.default_rng(seed)
    for j in range(n_uneven):
        n = int(draw.integers(n_range[0], n_range[1] + 1))
        nl = int(draw.integers(l_range[0], l_range[1] + 1))
        s = seed + n_rhs + j
        p = helmholtz_problem(n, nl, seed=s, mg_levels=1)
        ops.append(p)
        problem_op.append(len(ops) - 1)
        rhs.append(p.rhs)
    return BatchWorkload(ops, problem_op, rhs)


def to_level_major(v: np.ndarray, ncol: int, nlayers: int) -> np.ndarray:
    """Reference column-contiguous field -> (level, column) layout."""
    return np.ascontiguousarray(np.asarray(v).reshape(ncol, nlayers).T).ravel()


def from_level_major(v: np.ndarray, ncol: int, nlayers: int) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v).reshape(nlayers, ncol).T).ravel()


# --------------------------------------------------------------------- W0 LMA
# Reference hexahedron vertex order: bottom SW, SE, NE, NW then top (the
# W0 dofmap order of ExtrudedMesh.w0_dofmap).
_HEX = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                 [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.float64)


def _q1(xi):
    """Trilinear basis (8,) and its reference gradient (8, 3) at xi (3,)."""
    s = _HEX * xi + (1 - _HEX) * (1 - xi)                   # (8, 3) factor per axis
    sgn = 2 * _HEX - 1
    phi = s.prod(axis=1)
    grad = np.stack([sgn[:, 0] * s[:, 1] * s[:, 2], s[:, 0] * sgn[:, 1] * s[:, 2],
                     s[:, 0] * s[:, 1] * sgn[:, 2]], axis=1)
    return phi, grad


@dataclass
class W0Problem:
    """Lowest-order W0 (Q1) mass + kappa * stiffness on an extruded cubed sphere.

    matrix is local_stencil(ncell*nlayers, 8, 8) flattened in Fortran order
    (operator_mod.t90:113-119, ik = cell*nlayers + layer), map the W0 dofmap
    (ncell, 8) of first dofs, column-contiguous (vertex*(nlayers+1) + level).
    mass / stiff are the two parts with unit coefficient, same layout."""

    ncell: int
    nlayers: int
    nvert: int
    map: np.ndarray
    mass: np.ndarray
    stiff: np.ndarray
    kappa: np.ndarray          # (ncell, nlayers) coefficient per 3D cell
    rhs: np.ndarray

    @property
    def ndof(self) -> int:
        return self.nvert * (self.nlayers + 1)

    def matrix(self, kappa=None) -> np.ndarray:
        kap = self.kappa if kappa is None else kappa
        n3 = self.ncell * self.nlayers
        k_ik = np.asarray(kap).reshape(n3)                  # ik = cell*nl + layer
        m = self.mass.reshape(64, n3)
        s = self.stiff.reshape(64, n3)
        return (m + s * k_ik[None, :]).ravel()


def w0_element_matrices(mesh) -> tuple[np.ndarray, np.ndarray]:
    """Q1 mass and unit-coefficient stiffness of every hexahedron, 2x2x2 Gauss,
    in local_stencil layout (Fortran (ncell*nl, 8, 8) flattened)."""
    surf, nl = mesh.surface, mesh.nlayers
    ncell = surf.ncell
    r = mesh.radius + mesh.heights                           # (nl+1,)
    base = surf.vertex_xyz[surf.cell_vertices]                # (ncell, 4, 3)
    # vertices of every hex: (ncell, nl, 8, 3)
    bot = base[:, None, :, :] * r[None, :-1, None, None]
    top = base[:, None, :, :] * r[None, 1:, None, None]
    X = np.concatenate([bot, top], axis=2)
    n3 = ncell * nl
    X = X.reshape(n3, 8, 3)
    g = np.array([0.5 - 0.5 / np.sqrt(3.0), 0.5 + 0.5 / np.sqrt(3.0)])
    M = np.zeros((n3, 8, 8))
    K = np.zeros((n3, 8, 8))
    for a in g:
        for b in g:
            for c in g:
                phi, dphi = _q1(np.array([a, b, c]))
                J = np.einsum("nia,ib->nab", X, dphi)          # (n3, 3, 3): dx_a/dxi_b
                detJ = np.linalg.det(J)
                Jinv = np.linalg.inv(J)                        # dxi/dx
                gphys = np.einsum("ib,nba->nia", dphi, Jinv)   # (n3, 8, 3)
                w = 0.125 * np.abs(detJ)
                M += w[:, None, None] * phi[None, :, None] * phi[None, None, :]
                K += w[:, None, None] * np.einsum("nia,nja->nij", gphys, gphys)
    # local_stencil(ik, df, df2): Fortran order, ik fastest
    to_f = lambda A: np.ascontiguousarray(A.transpose(1, 2, 0)).reshape(8, 8, n3).transpose(1, 0, 2).ravel()
    return to_f(M), to_f(K)


def w0_problem(n: int, nlayers: int, seed: int, top: float, kappa_sigma: float = 0.0,
               stretching: str = "uniform", radius: float = EARTH_RADIUS_DEFAULT,
               kappa_scale: float = 1.0) -> W0Problem:
    """W0 diffusion problem: A = M + kappa K; kappa = kappa_scale exp(sigma g),
    g ~ N(0,1) per 3D cell (kappa = kappa_scale when sigma = 0); right-hand
    side N(0,1).  kappa_scale = dz^2 makes the diffusion across one layer
    comparable to the mass term."""
    from .mesh import extruded_mesh
    mesh = extruded_mesh(n, nlayers, top, stretching, radius=radius)
    mass, stiff = w0_element_matrices(mesh)
    rng = np.random.default_rng(seed)
    ncell = mesh.ncell
    kappa = kappa_scale * (np.exp(kappa_sigma * rng.standard_normal((ncell, nlayers)))
                           if kappa_sigma > 0 else np.ones((ncell, nlayers)))
    rhs = rng.standard_normal(mesh.w0_ndof())
    return W0Problem(ncell=ncell, nlayers=nlayers, nvert=mesh.surface.nvert,
                     map=mesh.w0_dofmap(), mass=mass, stiff=stiff, kappa=kappa, rhs=rhs)


# ------------------------------------------------------------------ W2 LMA
# Lowest-order Raviart-Thomas (W2) basis on the unit cube, one function per
# face W, S, E, N, B, T with unit flux through its own face in the positive
# direction of its axis (as the W2 transfers assume: a coarse cell's W and E
# values are fluxes in the same direction): phi_W = (1 - xi1, 0, 0),
# phi_E = (xi1, 0, 0), and likewise in xi2 (S, N) and xi3 (B, T); the
# reference divergences are -1 (W, S, B) and +1 (E, N, T).
_RT_AXIS = (0, 1, 0, 1, 2, 2)
_RT_UP = (False, False, True, True, False, True)     # xi or 1 - xi
_RT_DIV = np.array([-1.0, -1.0, 1.0, 1.0, -1.0, 1.0])


def w2_element_matrices(mesh, tau: float) -> np.ndarray:
    """Per cell-layer 6x6 matrices of M + tau D on the extruded mesh, with
    M the W2 mass matrix and D the divergence-divergence form, both through
    the contravariant Piola map of the trilinear hexahedron (2x2x2 Gauss),
    in the cell's local positive directions.  Returns (ncell*nl, 6, 6)."""
    surf, nl = mesh.surface, mesh.nlayers
    ncell = surf.ncell
    r = mesh.radius + mesh.heights
    base = surf.vertex_xyz[surf.cell_vertices]
    bot = base[:, None, :, :] * r[None, :-1, None, None]
    top = base[:, None, :, :] * r[None, 1:, None, None]
    X = np.concatenate([bot, top], axis=2).reshape(ncell * nl, 8, 3)
    g = np.array([0.5 - 0.5 / np.sqrt(3.0), 0.5 + 0.5 / np.sqrt(3.0)])
    dd = np.outer(_RT_DIV, _RT_DIV)
    A = np.zeros((ncell * nl, 6, 6))
    for a in g:
        for b in g:
            for c in g:
                xi = np.array([a, b, c])
                _, dphi = _q1(xi)
                J = np.einsum("nia,ib->nab", X, dphi)           # dx_a / dxi_b
                detJ = np.abs(np.linalg.det(J))
                ref = np.zeros((6, 3))
                for f in range(6):
                    t = xi[_RT_AXIS[f]]
                    ref[f, _RT_AXIS[f]] = t if _RT_UP[f] else 1.0 - t
                Jphi = np.einsum("nab,fb->nfa", J, ref)          # J phi_hat
                w = 0.125
                A += (w / detJ)[:, None, None] * np.einsum("nfa,nga->nfg", Jphi, Jphi)
                A += (tau * w / detJ)[:, None, None] * dd[None, :, :]
    return A


@dataclass
class W2Level:
    """One level of a W2 multigrid hierarchy in the device layout the
    library's LMA operators use: entities are the side-face columns
    (nlayers dofs) followed by one vertical column per cell (nlayers+1 dofs,
    B at offset 0 and T at offset 1); a field is (nent, nlayers+1) columns,
    the top level of every side face unused (zero).

    ent / off (ncell, 6): entity and level offset of each cell dof W, S, E,
    N, B, T.  matrix: local_stencil (ncell*nl, 6, 6) in Fortran order with
    the global orientation signs applied.  A field on the host is
    column-contiguous, column e holding its nlayers+1 levels (to_columns /
    from_columns convert from / to the flat order).  flat_map (ncell, 6) and
    flat_ndof: the same space in the reference's flat dof order
    (ExtrudedMesh.w2_dofmap).  ew / ns: face selectors of restrictions onto
    this level."""

    n: int
    nlayers: int
    ncell: int
    nent: int
    ent: np.ndarray
    off: np.ndarray
    matrix: np.ndarray
    flat_map: np.ndarray
    flat_ndof: int
    links: np.ndarray
    ew: np.ndarray
    ns: np.ndarray

    @property
    def nlev(self) -> int:
        return self.nlayers + 1

    def to_columns(self, v: np.ndarray) -> np.ndarray:
        """Flat reference-order W2 vector -> (nent, nlev) column-contiguous
        (the order Field.import_ takes; padding levels zero)."""
        out = np.zeros((self.nent, self.nlev))
        for df in range(5):
            ncol = self.nlayers + (1 if df == 4 else 0)
            for k in range(ncol):
                out[self.ent[:, df], k] = v[self.flat_map[:, df] + k]
        return out.ravel()

    def from_columns(self, d: np.ndarray) -> np.ndarray:
        d = np.asarray(d).reshape(self.nent, self.nlev)
        v = np.zeros(self.flat_ndof)
        for df in range(5):
            ncol = self.nlayers + (1 if df == 4 else 0)
            for k in range(ncol):
                v[self.flat_map[:, df] + k] = d[self.ent[:, df], k]
        return v


def w2_level(n: int, nlayers: int, top: float, tau: float,
             radius: float = EARTH_RADIUS_DEFAULT) -> W2Level:
    from .mesh import extruded_mesh
    mesh = extruded_mesh(n, nlayers, top, radius=radius)
    fmap, ndof = mesh.w2_dofmap()
    ncell = mesh.ncell
    # entities: side-face columns in dof order, then one vertical column per cell
    side = np.unique(fmap[:, :4])
    nside = side.size
    face_ent = {int(d): i for i, d in enumerate(side)}
    ent = np.zeros((ncell, 6), dtype=np.int32)
    off = np.zeros((ncell, 6), dtype=np.int32)
    for c in range(ncell):
        for df in range(4):
            ent[c, df] = face_ent[int(fmap[c, df])]
        ent[c, 4] = ent[c, 5] = nside + c
        off[c, 5] = 1
    # global orientation: the two cells of a face agree on its direction
    # when one reaches it as E or N and the other as W or S (inside a panel
    # always); where a panel edge pairs E/N with E/N or W/S with W/S, the
    # cell that did not number the face (the later one) flips its function
    links = mesh.surface.face_links
    sign = np.ones((ncell, 6))
    for c in range(ncell):
        for df in range(4):
            nb = int(links[c, df])
            g = [q for q in range(4) if links[nb, q] == c][0]
            if (df >= 2) != (g < 2) and c > nb:
                sign[c, df] = -1.0
    Ae = w2_element_matrices(mesh, tau)
    nl = nlayers
    s = np.repeat(sign, nl, axis=0)                     # (ncell*nl, 6), ik = c*nl + layer
    Ae = Ae * s[:, :, None] * s[:, None, :]
    # local_stencil(ik, df, df2) in Fortran order: ik fastest, then df, then df2
    matrix = np.ascontiguousarray(Ae.transpose(2, 1, 0)).ravel()
    ew, ns = mesh.w2_face_selectors()
    return W2Level(n=n, nlayers=nlayers, ncell=ncell, nent=nside + ncell, ent=ent, off=off,
                   matrix=matrix, flat_map=fmap.astype(np.int32), flat_ndof=int(ndof),
                   links=mesh.surface.face_links, ew=ew, ns=ns)


@dataclass
class W2Hierarchy:
    """W2 operators A = M + tau D on C_n, C_{n/2}, ... (rediscretised on every
    level) with the 2x2 cell maps between consecutive levels and a seeded
    right-hand side on the finest level (flat reference order)."""

    levels: list
    cell_maps: list
    rhs: np.ndarray


def w2_hierarchy(n: int, nlayers: int, nlevels: int, seed: int, top: float = 10e3,
                 tau: float = 1.0, radius: float = EARTH_RADIUS_DEFAULT) -> W2Hierarchy:
    from .mesh import coarsen_map
    levels, maps = [], []
    m = n
    for l in range(nlevels):
        levels.append(w2_level(m, nlayers, top, tau, radius))
        if l + 1 < nlevels:
            maps.append(coarsen_map(m))
            m //= 2
    rhs = np.random.default_rng(seed).standard_normal(levels[0].flat_ndof)
    return W2Hierarchy(levels=levels, cell_maps=maps, rhs=rhs)


# ------------------------------------------------------------ CMA shapes
def cma_size(nlayers, ndf_to, ndf_from, nface_to, nint_to, nface_from, nint_from):
    """The columnwise-operator parameters of a to-space / from-space pair
    (rows, columns, alpha, beta, gamma-, gamma+, bandwidth), as get_cma_size
    computes them (components/science/unit-test/support/
    get_unit_test_m3x3_cma_data_mod.f90:130-159); nface / nint are a space's
    dofs per cell on layer faces / inside the cell."""
    nrow = nlayers * nint_to + (nlayers + 1) * nface_to
    ncol = nlayers * nint_from + (nlayers + 1) * nface_from
    alpha = nface_from + nint_from
    beta = nface_to + nint_to
    g_m = (ndf_from - 1) * (nint_to + nface_to)
    g_p = (ndf_to - 1) * (nint_from + nface_from)
    bw = 1 + int(np.ceil((g_m + g_p) / beta))
    return dict(alpha=alpha, beta=beta, gm=g_m, gp=g_p, bw=bw, ncol=ncol, nrow=nrow)


def cma_prod_size(a, b):
    """Parameters of the product A B (get_cma_prod_size, same file)."""
    alpha, beta = a["alpha"] * b["alpha"], a["beta"] * b["beta"]
    gm = b["alpha"] * a["gm"] + a["beta"] * b["gm"]
    gp = b["alpha"] * a["gp"] + a["beta"] * b["gp"]
    bw = 1 + int(np.ceil((gm + gp) / beta))
    return dict(alpha=alpha, beta=beta, gm=gm, gp=gp, bw=bw, ncol=b["ncol"], nrow=a["nrow"])


def banded_dofmap(nlayers, ndf, nint, nface):
    """column_banded_dofmap(ndf, nlayers), 1-based
    (infrastructure/source/operator/columnwise_operator_mod.f90:377-393)."""
    k = np.arange(nlayers)[None, :]
    df = np.arange(1, ndf + 1)[:, None]
    return np.asfortranarray(k * (nint + nface) + df, dtype=np.int32)


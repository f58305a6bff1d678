"""The W2 function space on the cubed sphere and its multigrid hierarchy
(host set-up and the oracle; no GPU): the dofmap numbering of
dofmap_setup, face selectors that reach every coarse face, SPD element
matrices, and the oracle's W2 V-cycle as a preconditioner."""
import numpy as np

from lfric_core_b200.mesh import extruded_mesh, W, S, E, N
from lfric_core_b200.problems import w2_hierarchy


def test_w2_dofmap_numbering_and_sharing():
    nl = 3
    m = extruded_mesh(4, nl, 3e3)
    fmap, ndof = m.w2_dofmap()
    ncell = m.ncell
    assert ndof == 2 * ncell * nl + ncell * (nl + 1)
    # the first cell numbers its four side faces, then its vertical column
    assert list(fmap[0]) == [0, nl, 2 * nl, 3 * nl, 4 * nl, 4 * nl + 1]
    links = m.surface.face_links
    seen = {}
    for c in range(ncell):
        for f in range(4):
            nb = links[c, f]
            g = [q for q in range(4) if links[nb, q] == c][0]
            assert fmap[c, f] == fmap[nb, g]           # a face column is shared
            seen.setdefault(int(fmap[c, f]), set()).add(c)
        assert fmap[c, 5] == fmap[c, 4] + 1            # T = B + 1
    assert all(len(v) == 2 for v in seen.values())
    # every dof in exactly one column
    cover = np.zeros(ndof, int)
    for d in seen:
        cover[d:d + nl] += 1
    for c in range(ncell):
        cover[fmap[c, 4]:fmap[c, 4] + nl + 1] += 1
    assert cover.min() == 1 and cover.max() == 1


def test_w2_face_selectors_reach_every_face():
    """restrict_w2 writes W and S always, E when ew = 2 and N when ns = 2:
    every face of the coarse mesh must be written by one of its cells."""
    m = extruded_mesh(6, 2, 2e3)
    ew, ns = m.w2_face_selectors()
    fmap, _ = m.w2_dofmap()
    written = set()
    for c in range(m.ncell):
        faces = [W, S] + ([E] if ew[c] == 2 else []) + ([N] if ns[c] == 2 else [])
        written.update(int(fmap[c, f]) for f in faces)
    assert written == set(int(v) for v in np.unique(fmap[:, :4]))


def test_w2_element_matrices_spd():
    H = w2_hierarchy(6, 3, 2, seed=1, top=3e5, tau=1e9, radius=6.371e5)
    A = H.levels[0].matrix.reshape(6, 6, -1).transpose(2, 1, 0)
    assert np.allclose(A, A.transpose(0, 2, 1), rtol=0, atol=1e-12 * np.abs(A).max())
    assert np.linalg.eigvalsh(A).min() > 0


def test_oracle_w2_multigrid_beats_the_diagonal():
    """GCR(10) with the W2 V-cycle needs fewer iterations than with the
    diagonal on C24 x 4 (C24/C12/C6), and both reach the tolerance."""
    from oracle.oracle import W2Multigrid
    H = w2_hierarchy(24, 4, 3, seed=1, top=4e5, tau=1e9, radius=6.371e5)
    o = W2Multigrid(H, omega=0.6)
    x, st, info = o.gcr_solve(H.rhs, multigrid=True)
    xd, std, infod = o.gcr_solve(H.rhs, multigrid=False, max_iter=400)
    assert st == 0 and std == 0
    assert info.iterations < infod.iterations
    r = H.rhs - o.apply(x)
    assert np.linalg.norm(r) / np.linalg.norm(H.rhs) <= 1e-8
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-6

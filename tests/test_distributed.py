"""The column-partitioned solve on CPU ranks (gloo, world size 2 and 3).

lfric_core_b200.distributed plans the partition and the depth-1 halo,
exchanges halo columns point to point, all-reduces inner products and runs
the reference's gcr_solve over a `space`.  Here each rank's compute is the
oracle's on its local mesh (owned columns plus halo, halo rows the identity)
with numpy fields, so the partition, the halo plan, the exchange and the
global sums are checked without a GPU: the partitioned GCR must take the
single-domain oracle GCR's iteration count and reach its solution."""
import ctypes as C
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]

from lfric_core_b200.distributed import (halo_plan, local_operator, mg_owners,  # noqa: E402
                                         mg_plans, partition)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_and_halo_plan_are_consistent():
    from lfric_core_b200.mesh import cubed_sphere
    links = cubed_sphere(6).face_links
    ncol, world = links.shape[0], 3
    blocks = partition(ncol, world)
    assert blocks[0][0] == 0 and blocks[-1][1] == ncol
    plans = [halo_plan(links, r, world) for r in range(world)]
    for p in plans:
        # every owned column's neighbours are local, in the same order
        for i, g in enumerate(p.owned):
            glob = np.concatenate([p.owned, p.halo])[p.local_links[i]]
            assert np.array_equal(glob, links[g])
        # what q sends to p is exactly what p receives from q, in order
        for q, cols in p.recv.items():
            sent = plans[q].send[p.rank]
            assert np.array_equal(plans[q].owned[sent], p.halo[cols - p.nowned])


class OracleSpace:
    """One rank's compute done by the oracle on numpy fields (test only)."""

    def __init__(self, prob, rank, world):
        from lfric_core_b200.distributed import HaloExchange, global_sum
        from oracle.oracle import HelmOp, lib, ptr
        import torch
        self.L, self.ptr = lib(), ptr
        self.plan = halo_plan(prob.links, rank, world)
        self.nl = prob.nlayers
        lcm, lhf = local_operator(self.plan, prob.cm, prob.hf, prob.nlayers)
        self.cm, self.hf = np.ascontiguousarray(lcm), np.ascontiguousarray(lhf)
        self.links = np.ascontiguousarray(self.plan.local_links, dtype=np.int32)
        self.op = HelmOp(self.plan.nlocal, self.nl, self.cm.ctypes.data, self.hf.ctypes.data,
                         self.links.ctypes.data)
        self.n = self.plan.nlocal * self.nl
        nl = self.nl

        def cols_idx(c):
            return (np.asarray(c)[:, None] * nl + np.arange(nl)[None, :]).ravel()

        def pack(f, c):
            return torch.from_numpy(f[cols_idx(c)].copy())

        def unpack(f, c, buf):
            f[cols_idx(c)] = buf.numpy()

        def new_buffer(f, c):
            return torch.empty(len(c) * nl, dtype=torch.float64)

        self.exchange = HaloExchange(self.plan, pack, unpack, new_buffer)
        self.gsum = global_sum
        self.halo_slice = slice(self.plan.nowned * nl, self.n)

    def new(self):
        return np.zeros(self.n)

    def set(self, v, a):
        v[:] = a

    def copy(self, d, s):
        d[:] = s

    def axpy(self, y, a, x):
        y += a * x

    def scale(self, v, a):
        v *= a

    def dot(self, u, v):
        return self.gsum(float(np.dot(u, v)))

    def norm(self, v):
        return float(np.sqrt(self.gsum(float(np.dot(v, v)))))

    def apply(self, x, y):
        self.exchange(x)
        self.L.ora_helm_apply_d(C.byref(self.op), self.ptr(x), self.ptr(y))
        x[self.halo_slice] = 0.0
        y[self.halo_slice] = 0.0

    def prec(self, x, y):
        work = np.zeros(self.n + 2 * self.nl)
        self.L.ora_helm_smooth_d(C.byref(self.op), C.c_double(1.0), None, self.ptr(x),
                                 self.ptr(y), self.ptr(work))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    from lfric_core_b200.distributed import gcr_solve
    from lfric_core_b200.problems import helmholtz_problem
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = helmholtz_problem(8, 6, seed=21, mg_levels=1)
        sp = OracleSpace(p, rank, world)
        b = sp.new()
        b[:sp.plan.nowned * sp.nl] = p.rhs.reshape(-1, p.nlayers)[sp.plan.owned].ravel()
        x = sp.new()
        res = gcr_solve(sp, x, b, gcrk=10, r_tol=1e-9, max_iter=40)
        out.put((rank, res.status, res.iterations, sp.plan.owned, x[:sp.plan.nowned * sp.nl]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_gcr_matches_the_single_domain_oracle(world):
    from lfric_core_b200.problems import helmholtz_problem
    from oracle.oracle import Helmholtz as OraHelm, SolveInfo, ptr
    p = helmholtz_problem(8, 6, seed=21, mg_levels=1)
    # single domain: the oracle's gcr_solve with the column preconditioner
    ora = OraHelm(p)
    L = ora.L
    op = ora.op(0)
    mg = ora.mg(np.float64, n_pre=0, n_post=0, n_coarse=1, omega=1.0, nlevels=1)
    n = p.ndof
    x1 = np.zeros(n)
    work = np.zeros(23 * n)
    info = SolveInfo()
    st1 = L.ora_gcr_solve_d(C.c_long(n), C.cast(L.ora_helm_apply_cb_d, C.c_void_p), C.byref(op),
                            C.cast(L.ora_mg_apply_cb_d, C.c_void_p), C.byref(mg), 10,
                            C.c_double(1e-9), C.c_double(0.0), 40, 1, ptr(x1),
                            ptr(np.ascontiguousarray(p.rhs)), ptr(work), C.byref(info))
    assert st1 == 0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    x = np.zeros((p.ncol, p.nlayers))
    for rank, st, iters, owned, xo in got:
        assert st == 0
        assert iters == info.iterations
        x[owned] = xo.reshape(-1, p.nlayers)
    x = x.ravel()
    assert np.linalg.norm(x - x1) / np.linalg.norm(x1) < 1e-10


@pytest.mark.parametrize("world", [1, 2, 3])
def test_nested_plans_keep_the_transfers_on_the_rank(world):
    """mg_plans: every finer column is owned by its parent's owner, each
    level's local cell map is one-to-one onto the finer level's local
    columns, and an owned coarse column keeps its own children."""
    from lfric_core_b200.problems import helmholtz_problem
    p = helmholtz_problem(8, 2, seed=21, mg_levels=3)
    links = [p.links] + p.mg_links
    owners = mg_owners(p.mg_child, links[-1].shape[0], world)
    for l, ch in enumerate(p.mg_child):
        ch = ch.reshape(-1, 4)
        assert np.array_equal(owners[l][ch], np.repeat(owners[l + 1][:, None], 4, axis=1))
    seen = [np.zeros(lk.shape[0], dtype=int) for lk in links]
    for r in range(world):
        plans, lch = mg_plans(links, p.mg_child, r, world)
        for l, pl in enumerate(plans):
            seen[l][pl.owned] += 1
            for i, g in enumerate(pl.owned):
                glob = np.concatenate([pl.owned, pl.halo])[pl.local_links[i]]
                assert np.array_equal(glob, links[l][g])
            pad = np.arange(pl.nowned + pl.halo.size, pl.nlocal)
            assert np.array_equal(pl.local_links[pad], np.repeat(pad[:, None], 4, axis=1))
            if world == 1:
                assert pl.halo.size == 0 and pl.npad == 0
        for l, m in enumerate(lch):
            pf, pc = plans[l], plans[l + 1]
            assert m.shape == (pc.nlocal, 2, 2)
            assert np.array_equal(np.sort(m.ravel()), np.arange(pf.nlocal))
            own = m[:pc.nowned].reshape(-1, 4)
            assert np.array_equal(pf.owned[own], p.mg_child[l].reshape(-1, 4)[pc.owned])
    for sn in seen:
        assert (sn == 1).all()


class OracleLevels:
    """mg_vcycle's level interface on one rank, computed by the oracle on
    numpy fields (column-contiguous), with halo exchanges over gloo; the
    coarse operators are the oracle's Galerkin coarsening of the local
    operators (test only)."""

    def __init__(self, prob, rank, world, nlevels):
        from lfric_core_b200.distributed import HaloExchange
        from oracle.oracle import HelmOp, lib, ptr
        import torch
        L = lib()
        self.L, self.ptr, self.nl, self.nlevels = L, ptr, prob.nlayers, nlevels
        links = [prob.links] + list(prob.mg_links[:nlevels - 1])
        self.plans, lch = mg_plans(links, prob.mg_child[:nlevels - 1], rank, world)
        self.child = [np.ascontiguousarray(m.reshape(-1), dtype=np.int32) for m in lch]
        self.links = [np.ascontiguousarray(pl.local_links, dtype=np.int32) for pl in self.plans]
        cm, hf = local_operator(self.plans[0], prob.cm, prob.hf, prob.nlayers)
        self.cm, self.hf = [np.ascontiguousarray(cm)], [np.ascontiguousarray(hf)]
        self.ops = [HelmOp(self.plans[0].nlocal, self.nl, self.cm[0].ctypes.data,
                           self.hf[0].ctypes.data, self.links[0].ctypes.data)]
        for l in range(nlevels - 1):
            nc = self.plans[l + 1].nlocal
            cmc, hfc = np.zeros(3 * self.nl * nc), np.zeros(4 * self.nl * nc)
            L.ora_galerkin_coarsen(C.byref(self.ops[l]), nc, ptr(self.child[l]),
                                   ptr(self.links[l + 1]), ptr(cmc), ptr(hfc))
            self.cm.append(cmc)
            self.hf.append(hfc)
            self.ops.append(HelmOp(nc, self.nl, cmc.ctypes.data, hfc.ctypes.data,
                                   self.links[l + 1].ctypes.data))
        nl = self.nl

        def cols_idx(c):
            return (np.asarray(c)[:, None] * nl + np.arange(nl)[None, :]).ravel()

        def pack(f, c):
            return torch.from_numpy(f[cols_idx(c)].copy())

        def unpack(f, c, buf):
            f[cols_idx(c)] = buf.numpy()

        def new_buffer(f, c):
            return torch.empty(len(c) * nl, dtype=torch.float64)

        self.exch = [HaloExchange(pl, pack, unpack, new_buffer) for pl in self.plans]
        n = [pl.nlocal * nl for pl in self.plans]
        self._work = [(np.zeros(n[l]), np.zeros(n[l + 1]) if l + 1 < nlevels else None,
                       np.zeros(n[l + 1]) if l + 1 < nlevels else None) for l in range(nlevels)]
        self._sw = [np.zeros(n[l] + 2 * nl) for l in range(nlevels)]
        self._r = [np.zeros(n[l]) for l in range(nlevels)]

    def smooth(self, l, omega, x_in, b, x_out):
        p = self.ptr
        self.L.ora_helm_smooth_d(C.byref(self.ops[l]), C.c_double(omega),
                                 None if x_in is None else p(x_in), p(b), p(x_out), p(self._sw[l]))

    def copy(self, l, dst, src):
        dst[:] = src

    def set0(self, l, f):
        f[:] = 0.0

    def exchange(self, l, f):
        self.exch[l](f)

    def resid_restrict(self, l, x, b, bc):
        p, r = self.ptr, self._r[l]
        self.L.ora_helm_residual_d(C.byref(self.ops[l]), p(x), p(b), p(r))
        self.L.ora_restrict_sum_d(self.plans[l + 1].nlocal, self.nl, p(self.child[l]), p(r),
                                  p(bc))

    def prolong_add(self, l, fine, coarse):
        p = self.ptr
        self.L.ora_prolong_add_d(self.plans[l + 1].nlocal, self.nl, p(self.child[l]),
                                 p(coarse), p(fine))

    def work(self, l):
        return self._work[l]


class OracleMgSpace(OracleSpace):
    """OracleSpace with the partitioned V-cycle as the preconditioner."""

    def __init__(self, prob, rank, world, nlevels, mg):
        from lfric_core_b200.distributed import global_sum
        self.levels = OracleLevels(prob, rank, world, nlevels)
        lv = self.levels
        self.L, self.ptr, self.nl = lv.L, lv.ptr, lv.nl
        self.plan, self.op = lv.plans[0], lv.ops[0]
        self.n = self.plan.nlocal * self.nl
        self.exchange = lv.exch[0]
        self.gsum = global_sum
        self.halo_slice = slice(self.plan.nowned * self.nl, self.n)
        self.mg = mg

    def prec(self, x, y):
        from lfric_core_b200.distributed import mg_vcycle
        mg_vcycle(self.levels, x, y, **self.mg)
        y[self.halo_slice] = 0.0


MG_CASE = dict(n=8, nlayers=6, seed=21, nlevels=3,
               mg=dict(n_pre=2, n_post=2, n_coarse=8, omega=0.8))


def _mg_rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    from lfric_core_b200.distributed import gcr_solve
    from lfric_core_b200.problems import helmholtz_problem
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = MG_CASE
        p = helmholtz_problem(c["n"], c["nlayers"], seed=c["seed"], mg_levels=c["nlevels"])
        sp = OracleMgSpace(p, rank, world, c["nlevels"], c["mg"])
        b = sp.new()
        b[:sp.plan.nowned * sp.nl] = p.rhs.reshape(-1, p.nlayers)[sp.plan.owned].ravel()
        x = sp.new()
        res = gcr_solve(sp, x, b, gcrk=10, r_tol=1e-9, max_iter=40)
        out.put((rank, res.status, res.iterations, sp.plan.owned, x[:sp.plan.nowned * sp.nl]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_multigrid_gcr_matches_the_single_domain_oracle(world):
    """GCR(10) with the partitioned V-cycle (3 levels, C8 -> C4 -> C2, nested
    ownership, halo exchanges inside the V-cycle) on gloo ranks takes the
    single-domain oracle GCR + multigrid's iteration count and reaches its
    solution."""
    from lfric_core_b200.problems import helmholtz_problem
    from oracle.oracle import Helmholtz as OraHelm
    c = MG_CASE
    p = helmholtz_problem(c["n"], c["nlayers"], seed=c["seed"], mg_levels=c["nlevels"])
    x1, st1, info = OraHelm(p).gcr_mg_solve(p.rhs, gcrk=10, r_tol=1e-9, max_iter=40, **c["mg"])
    assert st1 == 0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_mg_rank, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    x = np.zeros((p.ncol, p.nlayers))
    for rank, st, iters, owned, xo in got:
        assert st == 0
        assert iters == info.iterations
        x[owned] = xo.reshape(-1, p.nlayers)
    x = x.ravel()
    assert np.linalg.norm(x - x1) / np.linalg.norm(x1) < 1e-10


def test_partition_helpers_reject_bad_input():
    """partition needs 1 <= world <= columns; halo_plan needs a rank for
    every column; mg_owners needs every fine column to have a parent."""
    from lfric_core_b200.mesh import cubed_sphere
    from lfric_core_b200.problems import coarsen_map
    links = cubed_sphere(4).face_links
    with pytest.raises(ValueError):
        partition(10, 0)
    with pytest.raises(ValueError):
        partition(3, 4)
    bad = np.zeros(links.shape[0], dtype=np.int64)
    bad[5] = 2
    with pytest.raises(ValueError):
        halo_plan(links, 0, 2, owner=bad)
    child = coarsen_map(4).copy()
    child.reshape(-1)[0] = child.reshape(-1)[1]      # one fine column lost its parent
    with pytest.raises(ValueError):
        mg_owners([child], 24, 2)
    with pytest.raises(ValueError):                  # more ranks than coarsest columns
        mg_owners([coarsen_map(4)], 24, 25)

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

from lfric_core_b200.distributed import halo_plan, local_operator, partition  # noqa: E402


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

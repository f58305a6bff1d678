"""Column-partitioned Helmholtz solves over several GPUs (one process each).

The reference partitions the mesh over MPI ranks, exchanges a depth-1 halo
before every operator apply (infrastructure/source/utilities/
halo_comms_mod.F90:18-34, 365-420, through YAXT) and sums every inner
product over the ranks (global_sum, infrastructure/source/utilities/
lfric_mpi_mod.F90:362-394).  Here:

* partition: rank r owns one contiguous block of the global column
  numbering (panel by panel, row by row);
* local columns: the owned ones, then the halo -- the columns of other
  ranks that an owned column is linked to -- in (owner, global id) order;
  a halo column links to itself and carries the identity column operator
  and no couplings, so its rows of A x and T'^{-1} r are x and r;
* halo exchange: every rank packs, for each neighbouring rank, the owned
  columns that rank needs (all levels, one contiguous buffer), sends it
  with torch.distributed point-to-point (NCCL between GPUs, gloo between
  CPU processes) and unpacks what it receives into its halo columns;
* Krylov vectors keep their halo columns at zero, so an inner product over
  a rank's whole local field is its share of the global one, and one
  all-reduce per inner product completes it.

The solver is the reference's gcr_solve (components/science/source/solver/
sci_iterative_solver_mod.f90:1288-1408) with the column (block-Jacobi)
preconditioner T'^{-1}, written once over a `space` that supplies the
vector operations, the distributed apply and the preconditioner;
`LibrarySpace` runs them on the GPU through the C ABI.  Nothing crosses
ranks except halo columns and inner products.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def partition(ncol: int, world: int) -> list[tuple[int, int]]:
    """Contiguous column blocks [start, end) of the global numbering, one
    per rank, sizes differing by at most one."""
    if world < 1 or ncol < world:
        raise ValueError("partition: need 1 <= world <= ncol")
    base, extra = divmod(ncol, world)
    out, s = [], 0
    for r in range(world):
        e = s + base + (1 if r < extra else 0)
        out.append((s, e))
        s = e
    return out


@dataclass
class HaloPlan:
    """One rank's view of a column partition.

    owned: global ids of the owned columns (local ids 0 .. nowned-1);
    halo: global ids of the halo columns (local ids nowned ..);
    local_links (nlocal, 4): neighbours W, S, E, N of every local column in
    local ids (a halo column links to itself);
    send[q]: local ids of the owned columns rank q needs, in q's halo order;
    recv[q]: local ids of the halo columns rank q fills."""

    rank: int
    world: int
    owned: np.ndarray
    halo: np.ndarray
    local_links: np.ndarray
    send: dict = field(default_factory=dict)
    recv: dict = field(default_factory=dict)

    @property
    def nowned(self) -> int:
        return int(self.owned.size)

    @property
    def nlocal(self) -> int:
        return int(self.owned.size + self.halo.size)


def halo_plan(links: np.ndarray, rank: int, world: int) -> HaloPlan:
    """The depth-1 halo plan of `rank` for the mesh links (ncol, 4)."""
    links = np.asarray(links)
    ncol = links.shape[0]
    blocks = partition(ncol, world)
    owner = np.empty(ncol, dtype=np.int64)
    for r, (s, e) in enumerate(blocks):
        owner[s:e] = r

    def halo_of(r):
        s, e = blocks[r]
        nb = np.unique(links[s:e].ravel())
        nb = nb[(nb < s) | (nb >= e)]
        return nb[np.lexsort((nb, owner[nb]))]          # by owner, then id

    s, e = blocks[rank]
    owned = np.arange(s, e)
    halo = halo_of(rank)
    local_id = {int(g): i for i, g in enumerate(owned)}
    local_id.update({int(g): owned.size + i for i, g in enumerate(halo)})
    ll = np.empty((owned.size + halo.size, 4), dtype=np.int32)
    for i, g in enumerate(owned):
        ll[i] = [local_id[int(v)] for v in links[g]]
    for i in range(halo.size):
        ll[owned.size + i] = owned.size + i
    plan = HaloPlan(rank=rank, world=world, owned=owned, halo=halo, local_links=ll)
    for q in range(world):
        if q == rank:
            continue
        hq = halo_of(q)
        need = hq[owner[hq] == rank]                       # my columns in q's halo
        if need.size:
            plan.send[q] = np.array([local_id[int(g)] for g in need], dtype=np.int32)
        mine = halo[owner[halo] == q]
        if mine.size:
            plan.recv[q] = np.array([local_id[int(g)] for g in mine], dtype=np.int32)
    return plan


def local_operator(plan: HaloPlan, cm: np.ndarray, hf: np.ndarray, nlayers: int):
    """The rank's local Helmholtz data (column-contiguous, the layout of
    HelmholtzProblem.cm / .hf): the owned columns' rows, and for every halo
    column the identity column operator without couplings."""
    cm = np.asarray(cm).reshape(-1, nlayers, 3)
    hf = np.asarray(hf).reshape(-1, nlayers, 4)
    n = plan.nlocal
    lcm = np.zeros((n, nlayers, 3))
    lhf = np.zeros((n, nlayers, 4))
    lcm[:plan.nowned] = cm[plan.owned]
    lhf[:plan.nowned] = hf[plan.owned]
    lcm[plan.nowned:, :, 1] = 1.0
    return lcm.ravel(), lhf.ravel()


class HaloExchange:
    """Fills the halo columns of a rank's local field from their owners.

    pack(field, cols) -> buffer and unpack(field, cols, buffer) move the
    given local columns (all levels) through a contiguous 1-D torch tensor;
    the buffers travel with torch.distributed isend / irecv (every rank
    posts all its receives and sends, then waits for them)."""

    def __init__(self, plan: HaloPlan, pack, unpack, new_buffer, group=None):
        self.plan, self.pack, self.unpack, self.new_buffer = plan, pack, unpack, new_buffer
        self.group = group

    def __call__(self, f) -> None:
        import torch.distributed as dist
        if self.plan.world == 1 or (not self.plan.send and not self.plan.recv):
            return
        reqs, inbox = [], {}
        for q, cols in sorted(self.plan.recv.items()):
            inbox[q] = self.new_buffer(f, cols)
            reqs.append(dist.irecv(inbox[q], src=q, group=self.group))
        for q, cols in sorted(self.plan.send.items()):
            reqs.append(dist.isend(self.pack(f, cols), dst=q, group=self.group))
        for r in reqs:
            r.wait()
        for q, cols in sorted(self.plan.recv.items()):
            self.unpack(f, cols, inbox[q])


def global_sum(value: float, group=None, device="cpu") -> float:
    """Sum of a scalar over the ranks (global_sum of lfric_mpi_mod)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(value)
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())


@dataclass
class GcrResult:
    status: int            # 0 ok, 1 not converged, 2 NaN
    iterations: int
    final_err: float


def gcr_solve(space, x, b, gcrk: int = 10, r_tol: float = 1e-8, a_tol: float = 0.0,
              max_iter: int = 20) -> GcrResult:
    """Right-preconditioned restarted GCR(k) with modified Gram-Schmidt
    (gcr_solve, sci_iterative_solver_mod.f90:1288-1408; convergence
    monitored): dx = P^{-1} b, res = b - A dx, then restarts of gcrk steps
    until ||res|| / ||b|| < r_tol; x += dx.  `space` provides new(), set(v,
    a), copy(dst, src), axpy(y, a, x) (y += a x), scale(v, a), dot(u, v) and
    norm(v) (global), apply(x, y) (y = A x) and prec(x, y) (y = P^{-1} x)."""
    sp = space
    dx, res, ax = sp.new(), sp.new(), sp.new()
    v = [sp.new() for _ in range(gcrk)]
    pv = [sp.new() for _ in range(gcrk)]
    sp.set(dx, 0.0)
    sp.prec(b, dx)
    sp.apply(dx, ax)
    sp.copy(res, b)
    sp.axpy(res, -1.0, ax)
    sc_err = sp.norm(b)
    if sc_err < np.finfo(np.float64).eps:
        return GcrResult(0, 0, 0.0)
    sc_err = max(sc_err, a_tol)
    err, steps, it = float("nan"), 0, 0
    for it in range(1, max_iter + 1):
        for iv in range(gcrk):
            sp.prec(res, pv[iv])
            sp.apply(pv[iv], v[iv])
            for j in range(iv):
                alpha = sp.dot(v[iv], v[j])
                sp.axpy(v[iv], -alpha, v[j])
                sp.axpy(pv[iv], -alpha, pv[j])
            alpha = sp.norm(v[iv])
            beta = 1.0 / alpha
            sp.scale(v[iv], beta)
            sp.scale(pv[iv], beta)
            alpha = sp.dot(res, v[iv])
            sp.axpy(dx, alpha, pv[iv])
            sp.axpy(res, -alpha, v[iv])
            steps += 1
            err = sp.norm(res) / sc_err
            if err < r_tol:
                break
        if err < r_tol:
            break
    status = 0
    if np.isnan(err):
        status = 2
    elif it >= max_iter and err > r_tol:
        status = 1
    sp.axpy(x, 1.0, dx)
    return GcrResult(status, steps, err)


class LibrarySpace:
    """The GPU side of one rank: the local Helmholtz operator and fields
    through the C ABI, NCCL halo exchanges and all-reduced inner products.
    Fields are the library's (nlocal, nlayers) W3 fields; halo columns of
    Krylov vectors are kept at zero."""

    def __init__(self, ctx, prob, rank: int, world: int, group=None):
        import torch
        from . import api
        self.api, self.ctx, self.group = api, ctx, group
        self.plan = halo_plan(prob.links, rank, world)
        self.nl = prob.nlayers
        lcm, lhf = local_operator(self.plan, prob.cm, prob.hf, prob.nlayers)
        self.mesh = api.Mesh(ctx, self.plan.local_links)
        self.op = api.Helmholtz(ctx, api.R_DOUBLE, self.mesh, prob.nlayers, lcm, lhf)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self._devcols = {}

        def pack(f, c):
            buf = torch.empty(len(c) * self.nl, dtype=torch.float64, device=dev)
            ctx.check(ctx.lib.lfg_field_pack_columns(
                f.h, self._cols_ptr(c), len(c), api.C.c_void_p(buf.data_ptr())), "pack_columns")
            return buf

        def unpack(f, c, buf):
            ctx.check(ctx.lib.lfg_field_unpack_columns(
                f.h, self._cols_ptr(c), len(c), api.C.c_void_p(buf.data_ptr())),
                "unpack_columns")

        def new_buffer(f, c):
            return torch.empty(len(c) * self.nl, dtype=torch.float64, device=dev)

        self.exchange = HaloExchange(self.plan, pack, unpack, new_buffer, group)

    def _cols_ptr(self, c):
        """The plan's column list c on the device (made once per list), as
        the int pointer the C ABI takes."""
        import torch
        key = c.ctypes.data
        if key not in self._devcols:
            self._devcols[key] = torch.tensor(c, dtype=torch.int32, device=self.device)
        C = self.api.C
        return C.cast(self._devcols[key].data_ptr(), C.POINTER(C.c_int))

    # vector space ---------------------------------------------------------
    def new(self):
        return self.op.field()

    def set(self, v, a):
        v.set_scalar(a)

    def copy(self, dst, src):
        dst.copy(src)

    def axpy(self, y, a, x):
        y.axpy(a, x)

    def scale(self, v, a):
        v.scale(a)

    def dot(self, u, v) -> float:
        return global_sum(u.dot(v), self.group, self.device)

    def norm(self, v) -> float:
        return float(np.sqrt(global_sum(v.dot(v), self.group, self.device)))

    def apply(self, x, y):
        """y = A x over the partition: halo exchange of x, the local apply,
        then the halo columns of x and y back to zero."""
        self.exchange(x)
        self.op.apply(y, x)
        n0, nh = self.plan.nowned, self.plan.nlocal - self.plan.nowned
        for f in (x, y):
            self.ctx.check(self.ctx.lib.lfg_field_zero_columns(f.h, n0, nh), "zero_columns")

    def prec(self, x, y):
        """y = T'^{-1} x, column by column (no communication)."""
        self.op.smooth(1.0, None, x, y)

    # host transfer of the owned part ------------------------------------
    def field_from_global(self, v_global: np.ndarray):
        g = np.asarray(v_global).reshape(-1, self.nl)
        local = np.zeros((self.plan.nlocal, self.nl))
        local[:self.plan.nowned] = g[self.plan.owned]
        return self.op.field(local.ravel())

    def owned_values(self, f) -> np.ndarray:
        return f.export().reshape(-1, self.nl)[:self.plan.nowned]

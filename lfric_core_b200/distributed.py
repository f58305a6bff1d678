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
sci_iterative_solver_mod.f90:1288-1408), written once over a `space` that
supplies the vector operations, the distributed apply and the
preconditioner: the column (block-Jacobi) preconditioner T'^{-1}
(`LibrarySpace`) or the multigrid V-cycle (`LibraryMgSpace`), on the GPU
through the C ABI.  Nothing crosses ranks except halo columns and inner
products.

The partitioned multigrid nests the ownership: the coarsest mesh's columns
are split into contiguous blocks and every finer column belongs to its
parent's owner (`mg_owners`), so the restriction and the prolongation only
move data between a rank's own columns.  Each level's local columns are
the owned ones, the halo, and padding columns (self-linked, identity rows)
that make the local intergrid map a one-to-one 2 x 2 map: the coarse halo
and padding columns take the fine halo and padding columns as children.
Their values are never read by an owned column: every sweep and every
residual first refills the halo from the owners.
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
    npad: int = 0          # padding columns after the halo (self-linked)

    @property
    def nowned(self) -> int:
        return int(self.owned.size)

    @property
    def nlocal(self) -> int:
        return int(self.owned.size + self.halo.size + self.npad)


def block_owner(ncol: int, world: int) -> np.ndarray:
    """owner[c] of every column under `partition`."""
    owner = np.empty(ncol, dtype=np.int64)
    for r, (s, e) in enumerate(partition(ncol, world)):
        owner[s:e] = r
    return owner


def halo_plan(links: np.ndarray, rank: int, world: int, owner: np.ndarray | None = None,
              npad: int = 0) -> HaloPlan:
    """The depth-1 halo plan of `rank` for the mesh links (ncol, 4).
    owner[c] is the rank of column c (default: the contiguous blocks of
    `partition`); a rank owns its columns in ascending global order.  npad
    padding columns follow the halo."""
    links = np.asarray(links)
    ncol = links.shape[0]
    owner = block_owner(ncol, world) if owner is None else np.asarray(owner, dtype=np.int64)
    if owner.shape != (ncol,) or owner.min() < 0 or owner.max() >= world:
        raise ValueError("halo_plan: owner must give every column a rank in [0, world)")

    def halo_of(r):
        nb = np.unique(links[owner == r].ravel())
        nb = nb[owner[nb] != r]
        return nb[np.lexsort((nb, owner[nb]))]          # by owner, then id

    owned = np.flatnonzero(owner == rank)
    halo = halo_of(rank)
    local_id = np.full(ncol, -1, dtype=np.int64)
    local_id[owned] = np.arange(owned.size)
    local_id[halo] = owned.size + np.arange(halo.size)
    n = owned.size + halo.size + npad
    ll = np.empty((n, 4), dtype=np.int32)
    ll[:owned.size] = local_id[links[owned]]
    ll[owned.size:] = np.arange(owned.size, n)[:, None]
    plan = HaloPlan(rank=rank, world=world, owned=owned, halo=halo, local_links=ll, npad=npad)
    for q in range(world):
        if q == rank:
            continue
        hq = halo_of(q)
        need = hq[owner[hq] == rank]                       # my columns in q's halo
        if need.size:
            plan.send[q] = local_id[need].astype(np.int32)
        mine = halo[owner[halo] == q]
        if mine.size:
            plan.recv[q] = local_id[mine].astype(np.int32)
    return plan


def mg_owners(child: list, ncoarsest: int, world: int) -> list[np.ndarray]:
    """Nested ownership of a multigrid hierarchy: the coarsest level's
    columns in the contiguous blocks of `partition`, every finer column
    owned by its parent's owner.  child[l] is the (ncol_{l+1}, 2, 2) cell
    map of level l+1 onto level l; returns owner[l] for every level."""
    owners = [block_owner(ncoarsest, world)]
    for ch in reversed(child):
        ch = np.asarray(ch).reshape(owners[0].size, -1)
        o = np.full(ch.size, -1, dtype=np.int64)
        o[ch] = owners[0][:, None]
        if (o < 0).any():
            raise ValueError("mg_owners: a fine column has no parent")
        owners.insert(0, o)
    return owners


def mg_plans(links: list, child: list, rank: int, world: int) -> tuple[list, list]:
    """The halo plans of every level of a nested partition (links[l]: the
    (ncol_l, 4) links of level l) and the local cell maps joining them:
    local_child[l] (nlocal_{l+1}, 2, 2) holds local column ids of level l.
    An owned coarse column keeps its own children; the coarse halo and
    padding columns take the fine halo and padding columns, four by four,
    and each level is padded so that it has four columns per coarse one."""
    L = len(links)
    owners = mg_owners(child, np.asarray(links[-1]).shape[0], world)
    plans = [None] * L
    plans[L - 1] = halo_plan(links[L - 1], rank, world, owners[L - 1])
    for l in range(L - 2, -1, -1):
        p = halo_plan(links[l], rank, world, owners[l])
        npad = 4 * plans[l + 1].nlocal - p.nowned - p.halo.size
        if npad < 0:
            raise ValueError("mg_plans: the fine halo outgrows the coarse one")
        plans[l] = halo_plan(links[l], rank, world, owners[l], npad=npad)
    local_child = []
    for l in range(L - 1):
        pf, pc = plans[l], plans[l + 1]
        lid = np.full(np.asarray(links[l]).shape[0], -1, dtype=np.int64)
        lid[pf.owned] = np.arange(pf.nowned)
        ch = np.asarray(child[l]).reshape(-1, 4)[pc.owned]
        own = lid[ch]
        if (own < 0).any():
            raise ValueError("mg_plans: an owned coarse column has a child owned elsewhere")
        rest = np.arange(pf.nowned, pf.nlocal).reshape(-1, 4)
        local_child.append(np.concatenate([own, rest]).reshape(-1, 2, 2).astype(np.int32))
    return plans, local_child


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


def mg_vcycle(lv, b, x, n_pre: int = 2, n_post: int = 2, n_coarse: int = 8,
              omega: float = 0.8) -> None:
    """x = one multigrid V-cycle applied to b over a partitioned hierarchy
    (x's initial value is not used).  The sequence is the library's
    V-cycle (lfg_prec_multigrid): on each level n_pre block-Jacobi column
    sweeps from zero, the residual restricted to the next level, the
    coarse correction prolonged and added, n_post sweeps; n_coarse sweeps
    from zero on the coarsest level.  Before every sweep from a guess and
    before the residual the guess's halo columns are refilled.

    lv supplies, per level l: smooth(l, omega, x_in or None, b, x_out),
    copy(l, dst, src), set0(l, f), exchange(l, f), resid_restrict(l, x, b,
    coarse_b), prolong_add(l, fine, coarse) and work(l) -> (tmp, coarse_b,
    coarse_x)."""
    last = lv.nlevels - 1

    def sweeps(l, n, x, b, from_zero):
        tmp = lv.work(l)[0]
        for s in range(n):
            if s == 0 and from_zero:
                lv.smooth(l, omega, None, b, x)
            else:
                lv.exchange(l, x)
                lv.smooth(l, omega, x, b, tmp)
                lv.copy(l, x, tmp)

    def cycle(l, b, x):
        if l == last:
            if n_coarse > 0:
                sweeps(l, n_coarse, x, b, True)
            else:
                lv.set0(l, x)
            return
        _, bc, xc = lv.work(l)
        if n_pre > 0:
            sweeps(l, n_pre, x, b, True)
        else:
            lv.set0(l, x)
        lv.exchange(l, x)
        lv.resid_restrict(l, x, b, bc)
        cycle(l + 1, bc, xc)
        lv.prolong_add(l, x, xc)
        sweeps(l, n_post, x, b, False)

    cycle(0, b, x)


class _DeviceColumns:
    """Halo columns of library fields through torch buffers on the device
    (lfg_field_pack_columns / unpack_columns); column lists are copied to
    the device once each."""

    def __init__(self, ctx, nl: int, device):
        self.ctx, self.nl, self.device = ctx, nl, device
        self._lists = {}

    def _ptr(self, c):
        import ctypes as C
        import torch
        key = id(c)
        if key not in self._lists:
            self._lists[key] = (c, torch.tensor(c, dtype=torch.int32, device=self.device))
        return C.cast(self._lists[key][1].data_ptr(), C.POINTER(C.c_int))

    def new_buffer(self, f, c):
        import torch
        return torch.empty(len(c) * self.nl, dtype=torch.float64, device=self.device)

    def pack(self, f, c):
        import ctypes as C
        buf = self.new_buffer(f, c)
        self.ctx.check(self.ctx.lib.lfg_field_pack_columns(
            f.h, self._ptr(c), len(c), C.c_void_p(buf.data_ptr())), "pack_columns")
        return buf

    def unpack(self, f, c, buf):
        import ctypes as C
        self.ctx.check(self.ctx.lib.lfg_field_unpack_columns(
            f.h, self._ptr(c), len(c), C.c_void_p(buf.data_ptr())), "unpack_columns")


class LibraryLevels:
    """One rank's multigrid hierarchy on the GPU through the C ABI: per
    level the local mesh and FP64 Helmholtz operator (level 0 the owned
    rows of the problem's operator, coarser levels the library's Galerkin
    coarsening of the local operator, which gives an owned coarse column
    the global operator's row and the halo and padding columns 4 I), the
    local intergrid map, the halo exchange and work fields.  The methods
    are mg_vcycle's level interface."""

    def __init__(self, ctx, prob, rank: int, world: int, nlevels: int | None = None,
                 group=None, exchange: bool = True):
        import torch
        from . import api
        L = prob.nlevels if nlevels is None else nlevels
        if not 1 <= L <= prob.nlevels:
            raise ValueError("LibraryLevels: bad number of levels")
        links = [prob.links] + list(prob.mg_links[:L - 1])
        self.plans, self.local_child = mg_plans(links, prob.mg_child[:L - 1], rank, world)
        self.nlevels, self.nl = L, prob.nlayers
        lcm, lhf = local_operator(self.plans[0], prob.cm, prob.hf, prob.nlayers)
        self.meshes = [api.Mesh(ctx, p.local_links) for p in self.plans]
        self.ops = [api.Helmholtz(ctx, api.R_DOUBLE, self.meshes[0], prob.nlayers, lcm, lhf)]
        self.maps = []
        for l in range(L - 1):
            ig = api.Intergrid(ctx, self.local_child[l], self.plans[l].nlocal)
            self.maps.append(ig)
            self.ops.append(self.ops[l].coarsen(ig, self.meshes[l + 1], api.R_DOUBLE))
        self._work = [(op.field(),
                       self.ops[l + 1].field() if l + 1 < L else None,
                       self.ops[l + 1].field() if l + 1 < L else None)
                      for l, op in enumerate(self.ops)]
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.columns = _DeviceColumns(ctx, prob.nlayers, self.device)
        cols = self.columns
        self.exch = [HaloExchange(p, cols.pack, cols.unpack, cols.new_buffer, group)
                     if exchange else (lambda f: None) for p in self.plans]

    def smooth(self, l, omega, x_in, b, x_out):
        self.ops[l].smooth(omega, x_in, b, x_out)

    def copy(self, l, dst, src):
        dst.copy(src)

    def set0(self, l, f):
        f.set_scalar(0.0)

    def exchange(self, l, f):
        self.exch[l](f)

    def resid_restrict(self, l, x, b, bc):
        self.ops[l].residual_restrict(self.maps[l], x, b, bc)

    def prolong_add(self, l, fine, coarse):
        self.maps[l].prolong(fine, coarse)

    def work(self, l):
        return self._work[l]


class LibrarySpace:
    """The GPU side of one rank: the local Helmholtz operator and fields
    through the C ABI, NCCL halo exchanges and all-reduced inner products.
    Fields are the library's (nlocal, nlayers) W3 fields; halo columns of
    Krylov vectors are kept at zero."""

    def __init__(self, ctx, prob, rank: int, world: int, group=None, exchange: bool = True):
        import torch
        from . import api
        self.api, self.ctx, self.group = api, ctx, group
        self.plan = halo_plan(prob.links, rank, world)
        self.nl = prob.nlayers
        lcm, lhf = local_operator(self.plan, prob.cm, prob.hf, prob.nlayers)
        self.mesh = api.Mesh(ctx, self.plan.local_links)
        self.op = api.Helmholtz(ctx, api.R_DOUBLE, self.mesh, prob.nlayers, lcm, lhf)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.columns = _DeviceColumns(ctx, self.nl, self.device)
        cols = self.columns
        self.exchange = (HaloExchange(self.plan, cols.pack, cols.unpack, cols.new_buffer, group)
                         if exchange else (lambda f: None))

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

    def zero_halo(self, f):
        """The halo (and padding) columns of f set to zero."""
        n0, nh = self.plan.nowned, self.plan.nlocal - self.plan.nowned
        if nh:
            self.ctx.check(self.ctx.lib.lfg_field_zero_columns(f.h, n0, nh), "zero_columns")

    def apply(self, x, y):
        """y = A x over the partition: halo exchange of x, the local apply,
        then the halo columns of x and y back to zero."""
        self.exchange(x)
        self.op.apply(y, x)
        self.zero_halo(x)
        self.zero_halo(y)

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


class LibraryMgSpace(LibrarySpace):
    """LibrarySpace with the partitioned multigrid V-cycle (mg_vcycle over
    LibraryLevels) as the preconditioner; the finest level's plan (nested
    ownership, padding) replaces the contiguous column blocks."""

    def __init__(self, ctx, prob, rank: int, world: int, group=None, nlevels: int | None = None,
                 n_pre: int = 2, n_post: int = 2, n_coarse: int = 8, omega: float = 0.8,
                 exchange: bool = True):
        from . import api
        self.api, self.ctx, self.group = api, ctx, group
        self.levels = LibraryLevels(ctx, prob, rank, world, nlevels, group, exchange)
        self.plan, self.nl = self.levels.plans[0], prob.nlayers
        self.mesh, self.op = self.levels.meshes[0], self.levels.ops[0]
        self.device, self.columns = self.levels.device, self.levels.columns
        self.exchange = self.levels.exch[0]
        self.mg = dict(n_pre=n_pre, n_post=n_post, n_coarse=n_coarse, omega=omega)

    def prec(self, x, y):
        """y = V-cycle(x); the halo and padding columns of y back to zero."""
        mg_vcycle(self.levels, x, y, **self.mg)
        self.zero_halo(y)

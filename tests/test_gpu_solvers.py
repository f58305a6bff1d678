"""Solvers through the C ABI against the oracle (FP64 parity 1e-12) and
size-independent properties at the full C192 x 70 size."""
import os

import numpy as np
import pytest

from lfric_core_b200 import api
from lfric_core_b200.api import R_DOUBLE, R_SINGLE, Field, field_from
from lfric_core_b200.problems import helmholtz_problem, w0_problem
from oracle.oracle import Helmholtz as OraHelm
from tests import ora_helpers as oh

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.fixture(scope="module")
def helm24():
    return helmholtz_problem(24, 20, seed=3, mg_levels=4)


def test_gcr_multigrid_fp64_parity(ctx, helm24):
    p = helm24
    ora = OraHelm(p)
    x_ref, st_ref, info = ora.gcr_mg_solve(p.rhs, gcrk=10, r_tol=1e-8, max_iter=20)
    S = api.HelmholtzSystem(ctx, p, mixed=False)
    res = S.solve_fp64(p.rhs)
    assert res.status == st_ref == 0
    assert res.iterations == info.iterations
    assert rel(S.solution(), x_ref) < 1e-12
    assert abs(res.final_err - info.final_err) / info.final_err < 1e-6


def test_gcr_repeated_solves_give_the_same_bits(ctx, helm24):
    """Monitored GCR with the multigrid preconditioner (whose V-cycles are
    replayed from captured graphs from their second use on): every solve
    takes the oracle's iteration count and gives the first solve's bits,
    with convergence inside a restart, at the last step the iteration
    limit allows, and a limit that stops it before convergence
    (NOT_CONVERGED after exactly that many steps)."""
    p = helm24
    x_ref, st_ref, info = OraHelm(p).gcr_mg_solve(p.rhs, gcrk=10, r_tol=1e-8, max_iter=20)
    S = api.HelmholtzSystem(ctx, p, mixed=False)
    outs = []
    for _ in range(3):
        res = S.solve_fp64(p.rhs)
        outs.append((res.status, res.iterations, res.final_err, S.solution()))
    assert outs[0][:2] == (st_ref, info.iterations)
    for o in outs[1:]:
        assert o[:3] == outs[0][:3]
        assert np.array_equal(o[3], outs[0][3])
    assert rel(outs[-1][3], x_ref) < 1e-12
    K = info.iterations
    B = S.op64.field(p.rhs)
    for gcrk, max_iter in ((3, 20), (K, 1), (3, 1)):
        sol = api.IterativeSolver(api.LinearOperator.from_helmholtz(S.op64), S.mg64, S.x64,
                                  "gcr", r_tol=1e-8, max_iter=max_iter, gcrk=gcrk)
        runs = []
        for _ in range(3):
            X = S.op64.field()
            out = sol.apply(X, B)
            runs.append((out.status, out.iterations, out.final_err, X.export()))
        for r in runs[1:]:
            assert r[:3] == runs[0][:3]
            assert np.array_equal(r[3], runs[0][3])
        if gcrk * max_iter < K:
            assert runs[0][0] == api.NOT_CONVERGED and runs[0][1] == gcrk * max_iter
        else:
            assert runs[0][0] == 0


def test_mixed_refinement_parity(ctx, helm24):
    p = helm24
    ora = OraHelm(p)
    x_ref, st_ref, mi = ora.mixed_solve(p.rhs, tol=1e-8, inner_tol=1e-4, inner_max_iter=2)
    S = api.HelmholtzSystem(ctx, p, fp64=False)
    res = S.solve_mixed(p.rhs)
    assert res.status == st_ref == 0
    assert res.rel_residual <= 1e-8
    # FP32 inner arithmetic differs in rounding from the oracle's FP32
    # arithmetic; both reach 1e-8 in FP64 and agree far below the exact
    # solution's distance from either.
    assert res.outer_iterations == mi.outer_iterations
    assert rel(S.solution(), x_ref) < 1e-7
    # true FP64 residual checked independently by the oracle
    r = p.rhs - ora.apply(S.solution())
    assert np.linalg.norm(r) / np.linalg.norm(p.rhs) <= 1e-8


@pytest.mark.parametrize("method", ["jacobi", "chebyshev", "precondition_only"])
def test_relaxation_solvers_parity(ctx, helm24, method):
    import ctypes as C
    from oracle.oracle import lib, ptr, SolveInfo
    p = helm24
    ora = OraHelm(p)
    S = api.HelmholtzSystem(ctx, p, mixed=False)
    kw = dict(jacobi=dict(max_iter=15, rho_relax=0.9), chebyshev=dict(max_iter=10, lmin=0.2, lmax=1.2),
              precondition_only=dict())[method]
    sol = api.IterativeSolver(api.LinearOperator.from_helmholtz(S.op64), S.mg64, S.x64, method,
                              r_tol=1e-30, fail_on_non_converged=False, **kw)
    B = S.op64.field(p.rhs)
    X = S.op64.field()
    out = sol.apply(X, B)
    L = lib()
    op, mg = ora.op(0), ora.mg()
    n = p.ndof
    x = np.zeros(n)
    info = SolveInfo()
    cb_a = C.cast(L.ora_helm_apply_cb_d, C.c_void_p)
    cb_p = C.cast(L.ora_mg_apply_cb_d, C.c_void_p)
    b = np.ascontiguousarray(p.rhs)
    if method == "jacobi":
        work = np.zeros(2 * n)
        L.ora_jacobi_solve_d(C.c_long(n), cb_a, C.byref(op), cb_p, C.byref(mg), C.c_double(1e-30),
                             C.c_double(0.0), 15, 1, C.c_double(0.9), ptr(x), ptr(b), ptr(work),
                             C.byref(info))
    elif method == "chebyshev":
        work = np.zeros(4 * n)
        L.ora_chebyshev_solve_d(C.c_long(n), cb_a, C.byref(op), cb_p, C.byref(mg), C.c_double(0.2),
                                C.c_double(1.2), 10, 1, ptr(x), ptr(b), ptr(work), C.byref(info))
    else:
        work = np.zeros(2 * n)
        L.ora_precondition_only_solve_d(C.c_long(n), cb_a, C.byref(op), cb_p, C.byref(mg), 1,
                                        ptr(x), ptr(b), ptr(work), C.byref(info))
    assert rel(X.export(), x) < 1e-12
    assert out.iterations == info.iterations


@pytest.mark.parametrize("n,nl", [(6, 5), (24, 20)])
def test_cg_jacobi_w0_parity(ctx, n, nl):
    """W0 mass + stiffness with a constant coefficient 1.0, uniform 1 km
    layers, Jacobi-preconditioned CG to 1e-8; (24, 20) is the full C24 x 20
    plain-method workload."""
    from oracle.oracle import W0 as OraW0
    p = w0_problem(n, nl, seed=1, top=nl * 1e3)
    A = p.matrix()
    nent, nlev = p.nvert, p.nlayers + 1
    lma = api.LocalOperator(ctx, R_DOUBLE, p.ncell, p.nlayers, A, p.map, nent, nlev)
    diag = Field(ctx, R_DOUBLE, nent, nlev)
    lma.diagonal(diag)
    sol = api.IterativeSolver(api.LinearOperator.from_lma(lma), api.Preconditioner.diagonal(diag),
                              diag, "cg", r_tol=1e-8, max_iter=2000)
    B, X = field_from(ctx, p.rhs, nent, nlev), Field(ctx, R_DOUBLE, nent, nlev)
    out = sol.apply(X, B)
    x, st, info = OraW0(p, A).cg_solve(p.rhs, r_tol=1e-8, max_iter=2000)
    assert out.status == st == 0
    assert out.iterations == info.iterations
    assert rel(X.export(), x) < 1e-12


def test_cg_convergence_found_inside_a_read_batch(ctx):
    """On small meshes monitored CG reads its residual norms once per batch
    of iterations and rolls x back to the iteration that converged: a solve
    stopped at that iteration by max_iter gives the same bits, and an
    iteration limit inside a batch reports that many iterations and the
    oracle's x after them."""
    from oracle.oracle import W0 as OraW0
    p = w0_problem(6, 5, seed=1, top=5e3)
    A = p.matrix()
    nent, nlev = p.nvert, p.nlayers + 1
    lma = api.LocalOperator(ctx, R_DOUBLE, p.ncell, p.nlayers, A, p.map, nent, nlev)
    diag = Field(ctx, R_DOUBLE, nent, nlev)
    lma.diagonal(diag)
    B = field_from(ctx, p.rhs, nent, nlev)

    def solve(max_iter):
        sol = api.IterativeSolver(api.LinearOperator.from_lma(lma),
                                  api.Preconditioner.diagonal(diag), diag, "cg", r_tol=1e-8,
                                  max_iter=max_iter)
        X = Field(ctx, R_DOUBLE, nent, nlev)
        return sol.apply(X, B), X.export()

    out, x = solve(2000)
    k = out.iterations
    assert out.status == 0 and k > 8
    out_k, x_k = solve(k)
    assert out_k.status == 0 and out_k.iterations == k
    assert np.array_equal(x, x_k)
    assert out_k.final_err == out.final_err
    out_s, x_s = solve(k - 3)
    assert out_s.status == api.NOT_CONVERGED and out_s.iterations == k - 3
    x_ref, st, info = OraW0(p, A).cg_solve(p.rhs, r_tol=1e-8, max_iter=k - 3)
    assert info.iterations == k - 3
    assert rel(x_s, x_ref) < 1e-12


def test_graph_replay_after_the_scratch_buffer_grows():
    """Monitored CG replays its full batches from a captured graph whose LMA
    applies hold the context's scratch buffer.  When a larger operator then
    grows that buffer (freeing the old one), the next solve captures again
    instead of replaying the freed address: every solve of the same system
    into the same x gives the same bits."""
    c = api.Context(int(os.environ.get("LFG_DEVICE", "0")))
    try:
        p = w0_problem(6, 5, seed=1, top=5e3)
        A = p.matrix()
        nent, nlev = p.nvert, p.nlayers + 1
        lma = api.LocalOperator(c, R_DOUBLE, p.ncell, p.nlayers, A, p.map, nent, nlev)
        diag = Field(c, R_DOUBLE, nent, nlev)
        lma.diagonal(diag)
        B, X = field_from(c, p.rhs, nent, nlev), Field(c, R_DOUBLE, nent, nlev)
        sol = api.IterativeSolver(api.LinearOperator.from_lma(lma),
                                  api.Preconditioner.diagonal(diag), diag, "cg", r_tol=1e-8,
                                  max_iter=2000)

        def solve():
            X.set_scalar(0.0)
            out = sol.apply(X, B)
            assert out.status == 0 and out.iterations > 8
            return out.iterations, X.export()

        k0, x0 = solve()           # eager
        for _ in range(2):         # captured, then replayed
            k, x = solve()
            assert k == k0 and np.array_equal(x, x0)
        big = w0_problem(24, 20, seed=2, top=2e4)
        lb = api.LocalOperator(c, R_DOUBLE, big.ncell, big.nlayers, big.matrix(), big.map,
                               big.nvert, big.nlayers + 1)
        yb = Field(c, R_DOUBLE, big.nvert, big.nlayers + 1)
        lb.apply(api.LMA_WRITE, yb, field_from(c, big.rhs, big.nvert, big.nlayers + 1))
        for _ in range(3):         # eager after the growth, captured, replayed
            k, x = solve()
            assert k == k0 and np.array_equal(x, x0)
    finally:
        c.close()


@pytest.mark.parametrize("method,iters", [("bicgstab", 6), ("gmres", 2), ("fgmres", 2)])
def test_krylov_variants_parity(ctx, helm24, method, iters):
    """bicgstab / gmres / fgmres with the multigrid preconditioner against the
    oracle's restatement, a fixed number of iterations (gcrk = 8)."""
    import ctypes as C
    from oracle.oracle import lib, ptr, SolveInfo
    p = helm24
    ora = OraHelm(p)
    S = api.HelmholtzSystem(ctx, p, mixed=False)
    k = 8
    sol = api.IterativeSolver(api.LinearOperator.from_helmholtz(S.op64), S.mg64, S.x64, method,
                              r_tol=1e-30, max_iter=iters, gcrk=k, fail_on_non_converged=False)
    x0 = np.random.default_rng(11).standard_normal(p.ndof) * 1e-3   # non-zero first guess
    B, X = S.op64.field(p.rhs), S.op64.field(x0)
    out = sol.apply(X, B)
    L = lib()
    op, mg = ora.op(0), ora.mg()
    n = p.ndof
    x = x0.copy()
    info = SolveInfo()
    cb_a = C.cast(L.ora_helm_apply_cb_d, C.c_void_p)
    cb_p = C.cast(L.ora_mg_apply_cb_d, C.c_void_p)
    b = np.ascontiguousarray(p.rhs)
    if method == "bicgstab":
        work = np.zeros(8 * n)
        L.ora_bicgstab_solve_d(n, cb_a, C.byref(op), cb_p, C.byref(mg), 1e-30, 0.0, iters, 1,
                               ptr(x), ptr(b), ptr(work), C.byref(info))
    else:
        work = np.zeros((5 + 2 * k) * n)
        getattr(L, f"ora_{method}_solve_d")(n, cb_a, C.byref(op), cb_p, C.byref(mg), k, 1e-30,
                                            0.0, iters, 1, ptr(x), ptr(b), ptr(work),
                                            C.byref(info))
    assert out.iterations == info.iterations
    assert rel(X.export(), x) < 1e-12
    assert abs(out.final_err - info.final_err) <= 1e-6 * abs(info.final_err) + 1e-15


@pytest.mark.parametrize("nf", [1, 2, 3])
def test_block_gcr_parity(ctx, helm24, nf):
    """block_gcr_solve with the multigrid preconditioner against the
    oracle; the vector is split into nf fields by level ranges (the device
    vector is level-major, so a level range is one segment)."""
    import ctypes as C
    from oracle.oracle import lib, ptr, SolveInfo
    p = helm24
    ora = OraHelm(p)
    S = api.HelmholtzSystem(ctx, p, mixed=False)
    sol = api.IterativeSolver(api.LinearOperator.from_helmholtz(S.op64), S.mg64, S.x64,
                              "block_gcr", r_tol=1e-8, max_iter=20, gcrk=6)
    nl, ncol = p.nlayers, p.ncol
    cuts = [0] + [round(nl * (i + 1) / nf) for i in range(nf)]
    sol.set_fields([c * ncol for c in cuts])
    B, X = S.op64.field(p.rhs), S.op64.field()
    out = sol.apply(X, B)
    # the oracle works in the column-contiguous layout: dof c*nl + k
    level = np.tile(np.arange(nl), ncol)
    field_of = np.searchsorted(np.array(cuts[1:]), level, side="right").astype(np.int32)
    L = lib()
    n = p.ndof
    x = np.zeros(n)
    info = SolveInfo()
    work = np.zeros((2 + 2 * 6) * n)
    op, mg = ora.op(0), ora.mg()
    st = L.ora_block_gcr_solve_d(n, C.cast(L.ora_helm_apply_cb_d, C.c_void_p), C.byref(op),
                                 C.cast(L.ora_mg_apply_cb_d, C.c_void_p), C.byref(mg), 6, 1e-8,
                                 0.0, 20, 1, nf, field_of.ctypes.data_as(C.POINTER(C.c_int)),
                                 ptr(x), ptr(np.ascontiguousarray(p.rhs)), ptr(work),
                                 C.byref(info))
    assert out.status == st == 0
    assert out.iterations == info.iterations
    assert rel(X.export(), x) < 1e-12
    assert abs(out.final_err - info.final_err) <= 1e-6 * info.final_err


@pytest.mark.parametrize("method", ["bicgstab", "gmres", "fgmres", "cg"])
def test_krylov_variants_converge(ctx, method):
    p = helmholtz_problem(8, 10, seed=5, mg_levels=2)
    S = api.HelmholtzSystem(ctx, p, mixed=False)
    sol = api.IterativeSolver(api.LinearOperator.from_helmholtz(S.op64), S.mg64, S.x64, method,
                              r_tol=1e-9, max_iter=40, gcrk=8)
    B, X = S.op64.field(p.rhs), S.op64.field()
    out = sol.apply(X, B)
    assert out.status == 0, out
    ora = OraHelm(p)
    r = p.rhs - ora.apply(X.export())
    assert np.linalg.norm(r) / np.linalg.norm(p.rhs) < 1e-7


def test_solver_status_codes(ctx, helm24):
    S = api.HelmholtzSystem(ctx, helm24, mixed=False)
    sol = api.IterativeSolver(api.LinearOperator.from_helmholtz(S.op64), S.mg64, S.x64, "gcr",
                              r_tol=1e-14, max_iter=1, gcrk=2)
    B, X = S.op64.field(helm24.rhs), S.op64.field()
    assert sol.apply(X, B).status == api.NOT_CONVERGED
    bad = helm24.rhs.copy()
    bad[17] = np.nan
    assert sol.apply(X, S.op64.field(bad)).status in (api.NAN_STATUS, api.NOT_CONVERGED)
    with pytest.raises(api.LfgError):
        sol.apply(X, Field(ctx, R_DOUBLE, 3, 3))


# --------------------------------------------------------------- full size
@pytest.fixture(scope="module")
def helm192():
    return helmholtz_problem(192, 70, seed=3, mg_levels=4)


def test_mixed_parity_c96(ctx):
    """The mixed solve on C96 x 70 (multigrid C96/48/24/12): the fine level
    runs the TMA-staged substitutions (zero start and from x_in; the
    prolongation-corrected post-smoother per column), the coarse levels the
    segmented sweep; against the oracle's mixed solve."""
    p = helmholtz_problem(96, 70, seed=3, mg_levels=4)
    ora = OraHelm(p)
    x_ref, st_ref, mi = ora.mixed_solve(p.rhs, tol=1e-8, inner_tol=1e-4, inner_max_iter=2)
    S = api.HelmholtzSystem(ctx, p, fp64=True)
    res = S.solve_mixed(p.rhs)
    assert res.status == st_ref == 0
    assert res.outer_iterations == mi.outer_iterations
    assert rel(S.solution(), x_ref) < 1e-7
    r = p.rhs - ora.apply(S.solution())
    assert np.linalg.norm(r) / np.linalg.norm(p.rhs) <= 1e-8
    # FP64 GCR + MG at the same size against the oracle (per-column FP64 kernels)
    x64, st64, info = ora.gcr_mg_solve(p.rhs, gcrk=10, r_tol=1e-8, max_iter=20)
    r64 = S.solve_fp64(p.rhs)
    assert r64.status == st64 == 0 and r64.iterations == info.iterations
    assert rel(S.solution(), x64) < 1e-12
    ctx.synchronize()


def test_full_size_parity_c192(ctx, helm192):
    """The headline workload, C192 x 70 with multigrid C192/96/48/24, against
    the oracle: the FP64 GCR(10) + multigrid solve takes the oracle's
    iteration count and agrees to 1e-12; the mixed solve takes the oracle's
    outer iteration count, agrees with the oracle's mixed solve to 1e-7 and
    reaches 1e-8 in the true FP64 residual, computed by the oracle's apply.
    Repeated solves are bit-identical (deterministic reductions)."""
    p = helm192
    ora = OraHelm(p)
    S = api.HelmholtzSystem(ctx, p)
    # FP64 GCR(10) + MG
    x64, st64, info = ora.gcr_mg_solve(p.rhs, gcrk=10, r_tol=1e-8, max_iter=20)
    r1 = S.solve_fp64(p.rhs)
    assert r1.status == st64 == 0
    assert r1.iterations == info.iterations
    x1 = S.solution()
    assert rel(x1, x64) < 1e-12
    r = p.rhs - ora.apply(x1)
    assert np.linalg.norm(r) / np.linalg.norm(p.rhs) <= 1e-8 * (1 + 1e-6)
    S.solve_fp64()
    assert np.array_equal(S.solution(), x1)
    # mixed: FP32 inner GCR(10) + MG, FP64 refinement
    xm, stm, mi = ora.mixed_solve(p.rhs, tol=1e-8, inner_tol=1e-4, inner_max_iter=2)
    m = S.solve_mixed()
    assert m.status == stm == 0
    assert m.outer_iterations == mi.outer_iterations
    xg = S.solution()
    assert rel(xg, xm) < 1e-7
    r = p.rhs - ora.apply(xg)
    assert np.linalg.norm(r) / np.linalg.norm(p.rhs) <= 1e-8
    S.solve_mixed()
    assert np.array_equal(S.solution(), xg)
    ctx.synchronize()


def test_cma_line_solve_c96(ctx):
    """Config-2: C96 x 70 tridiagonal line solve, FP64 against the oracle,
    FP32 solve + FP64 refinement reaching FP64 accuracy."""
    p = helmholtz_problem(96, 70, seed=2, mg_levels=1)
    ncol, nl = p.ncol, p.nlayers
    ind = np.arange(1, nl + 1, dtype=np.int32)
    A64 = api.ColumnwiseOperator(ctx, R_DOUBLE, ncol, nl, nl, 3, 1, 1, 1, 1, ind, ind, p.cm)
    A32 = api.ColumnwiseOperator(ctx, R_SINGLE, ncol, nl, nl, 3, 1, 1, 1, 1, ind, ind, p.cm)
    B = field_from(ctx, p.rhs, ncol, nl)
    X = Field(ctx, R_DOUBLE, ncol, nl)
    A64.apply_inverse(X, B)
    ref = oh.cma_appinv(p.cm, ncol, nl, ind, p.rhs, nl)
    assert rel(X.export(), ref) < 1e-12
    # FP32 Thomas + FP64 refinement
    X2, R, R32, E32 = Field(ctx, R_DOUBLE, ncol, nl), Field(ctx, R_DOUBLE, ncol, nl), \
        Field(ctx, R_SINGLE, ncol, nl), Field(ctx, R_SINGLE, ncol, nl)
    R.copy(B)
    for _ in range(4):
        R32.copy(R)
        A32.apply_inverse(E32, R32)
        X2.axpy(1.0, E32)
        R.copy(B)
        R.scale(-1.0)
        A64.apply(R, X2)          # R = -b + A x
        R.scale(-1.0)             # R = b - A x
    assert rel(X2.export(), ref) < 1e-12

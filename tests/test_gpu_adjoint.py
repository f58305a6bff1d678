"""Hand-written adjoints: dot-product tests of the transposed applies, and
gradients of J = 0.5 ||u - u_obs||^2 through the W0 diffusion solve against
central finite differences (h = 1e-6) and the FP64 tangent-linear model."""
import numpy as np
import pytest

from lfric_core_b200 import api
from lfric_core_b200.api import R_DOUBLE, R_SINGLE, Field, field_from
from lfric_core_b200.problems import w0_problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def actx():
    c = api.Context(0)
    yield c
    c.close()


def test_lma_transpose_dot_product(ctx):
    p = w0_problem(8, 6, seed=2, top=6e3, kappa_sigma=0.5)
    rng = np.random.default_rng(1)
    # a non-symmetric element matrix exercises the transpose
    A = p.matrix() * (1.0 + 0.3 * rng.standard_normal(p.mass.size))
    lma = api.LocalOperator(ctx, R_DOUBLE, p.ncell, p.nlayers, A, p.map, p.nvert, p.nlayers + 1)
    x, y = rng.standard_normal(p.ndof), rng.standard_normal(p.ndof)
    X, Y = field_from(ctx, x, p.nvert, p.nlayers + 1), field_from(ctx, y, p.nvert, p.nlayers + 1)
    AX, ATY = Field(ctx, R_DOUBLE, p.nvert, p.nlayers + 1), Field(ctx, R_DOUBLE, p.nvert, p.nlayers + 1)
    lma.apply(api.LMA_INC, AX, X)
    lma.apply(api.LMA_TRANSPOSE, ATY, Y)
    lhs, rhs = np.dot(AX.export(), y), np.dot(x, ATY.export())
    assert abs(lhs - rhs) / abs(lhs) < 1e-13


@pytest.mark.parametrize("kind,tol", [(R_DOUBLE, 1e-13), (R_SINGLE, 1e-5)])
def test_cma_transpose_dot_product(ctx, kind, tol):
    # Wtheta (nl+1 rows) -> W3 (nl columns): alpha=1, beta=1, gamma_m=0, gamma_p=1, bw=2
    ncol, nl = 500, 12
    nrow, ncolumn = nl + 1, nl
    rng = np.random.default_rng(3)
    cm = rng.standard_normal((ncol, nrow, 2))
    it = np.arange(1, nrow + 1, dtype=np.int32)
    iff = np.arange(1, ncolumn + 1, dtype=np.int32)
    A = api.ColumnwiseOperator(ctx, kind, ncol, nrow, ncolumn, 2, 1, 1, 0, 1, it, iff, cm)
    x, y = rng.standard_normal(ncol * ncolumn), rng.standard_normal(ncol * nrow)
    AX = Field(ctx, kind, ncol, nrow)
    ATY = Field(ctx, kind, ncol, ncolumn)
    X = field_from(ctx, x, ncol, ncolumn, kind=kind)
    Y = field_from(ctx, y, ncol, nrow, kind=kind)
    A.apply(AX, X)
    ctx.check(ctx.lib.lfg_cma_apply_transpose(A.h, ATY.h, Y.h))
    lhs, rhs = np.dot(AX.export(np.float64), y), np.dot(x, ATY.export(np.float64))
    assert abs(lhs - rhs) / abs(lhs) < tol


def _config4(n=48, nl=30):
    # 1 km layers; kappa = (1 km)^2 exp(0.5 g): diffusion across a layer is
    # comparable to the mass term
    return w0_problem(n, nl, seed=4, top=nl * 1e3, kappa_sigma=0.5, kappa_scale=1e6)


@pytest.mark.parametrize("n,nl", [(8, 10), (48, 30)])
def test_gradients_against_fd_and_tlm(actx, n, nl):
    """Config-4 check: 16 random directions in (f, kappa); central FD with
    h = 1e-6 and the tangent-linear model against the adjoint gradient."""
    import torch
    from lfric_core_b200.autograd import DiffusionSolve, W0Diffusion
    p = _config4(n, nl)
    sysm = W0Diffusion(actx, p, r_tol=1e-13, max_iter=5000)
    dev = torch.device("cuda")
    lm = lambda a, ncol, nlev: torch.tensor(np.ascontiguousarray(
        np.asarray(a).reshape(ncol, nlev).T), dtype=torch.float64, device=dev).reshape(-1)
    f = lm(p.rhs, p.nvert, nl + 1).requires_grad_(True)
    kap = lm(p.kappa.ravel(), p.ncell, nl).requires_grad_(True)
    rng = np.random.default_rng(7)
    with torch.no_grad():                 # observations near the forward solution
        u_nom = DiffusionSolve.apply(f.detach(), kap.detach(), sysm)
        uobs = u_nom + 0.1 * u_nom.std() * torch.tensor(rng.standard_normal(p.ndof),
                                                        dtype=torch.float64, device=dev)

    def J(ff, kk):
        u = DiffusionSolve.apply(ff, kk, sysm)
        return 0.5 * torch.sum((u - uobs) ** 2), u

    j0, u0 = J(f, kap)
    j0.backward()
    gf, gk = f.grad.detach().clone(), kap.grad.detach().clone()
    h = 1e-6
    worst_fd, worst_tlm = 0.0, 0.0
    for d in range(16):
        df = torch.tensor(rng.standard_normal(p.ndof), dtype=torch.float64, device=dev)
        # kappa directions are relative (a perturbation of log kappa)
        dk = kap.detach() * torch.tensor(rng.standard_normal(p.ncell * nl), dtype=torch.float64,
                                         device=dev)
        if d % 2:                       # alternate: f-only and kappa-only directions
            df = df * 0
        else:
            dk = dk * 0
        adj = float(torch.dot(gf, df) + torch.dot(gk, dk))
        with torch.no_grad():
            jp, _ = J(f + h * df, kap + h * dk)
            jm, _ = J(f - h * df, kap - h * dk)
        fd = float(jp - jm) / (2 * h)
        # tangent-linear: du from A du = df - (dk K) u, dJ = <u - uobs, du>
        with torch.no_grad():
            sysm.begin(u0, df, dk)
            du = torch.empty_like(u0)
            with torch.cuda.stream(sysm.stream):
                sysm.assemble(kap.detach())
                sysm.tangent(u0.detach(), df, dk, du)
            sysm.end()
            tlm = float(torch.dot(u0.detach() - uobs, du))
        scale = max(abs(adj), 1e-300)
        worst_fd = max(worst_fd, abs(fd - adj) / scale)
        worst_tlm = max(worst_tlm, abs(tlm - adj) / scale)
    assert worst_tlm < 1e-8, worst_tlm
    assert worst_fd < 1e-4, worst_fd

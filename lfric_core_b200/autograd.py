"""Differentiable W0 diffusion solve on the device (PyTorch autograd).

A(kappa) = M + kappa K is the lowest-order W0 mass + diffusion operator held
as LMA element matrices (operator_type, infrastructure/source/operator/
operator_mod.t90), kappa one coefficient per 3D cell.  The forward solve is
the reference's Jacobi-preconditioned conjugate gradient (cg_solve,
components/science/source/solver/sci_iterative_solver_mod.f90:495-592) on
the GPU.  The backward pass is written by hand:

  lambda = A^{-T} dJ/du                (a transpose solve: CG on the
                                        transpose_matrix_vector operator)
  dJ/df  = lambda
  dJ/dkappa_e = - lambda_e^T K_e u_e   (per-cell bilinear form)

The operator is re-assembled from kappa in the backward pass (recomputation)
rather than keeping the forward solve's Krylov vectors.

Tensors are float64 CUDA tensors in the device layout of the library:
W0 fields (nlayers+1, nvert) level-major, kappa (nlayers, ncell).  All
library work runs on a private stream ordered against PyTorch's current
stream.
"""
from __future__ import annotations

import numpy as np
import torch

from . import api
from .api import R_DOUBLE, Field, LocalOperator
from .problems import W0Problem


class W0Diffusion:
    """Device-resident A(kappa) = M + kappa K with forward and adjoint solves."""

    def __init__(self, ctx: api.Context, prob: W0Problem, r_tol: float = 1e-8,
                 max_iter: int = 2000):
        self.ctx, self.prob = ctx, prob
        self.ncell, self.nl = prob.ncell, prob.nlayers
        self.nent, self.nlev = prob.nvert, prob.nlayers + 1
        mk = dict(ncell=prob.ncell, nlayers=prob.nlayers, map_to=prob.map,
                  nent_to=self.nent, nlev_to=self.nlev)
        self.M = LocalOperator(ctx, R_DOUBLE, local_stencil=prob.mass, **mk)
        self.K = LocalOperator(ctx, R_DOUBLE, local_stencil=prob.stiff, **mk)
        self.A = LocalOperator(ctx, R_DOUBLE, local_stencil=prob.matrix(), **mk)
        self.zero = LocalOperator(ctx, R_DOUBLE, local_stencil=np.zeros_like(prob.mass), **mk)
        self.diag = Field(ctx, R_DOUBLE, self.nent, self.nlev)
        self.kappa = Field(ctx, R_DOUBLE, self.ncell, self.nl)
        prec = api.Preconditioner.diagonal(self.diag)
        self.cg = api.IterativeSolver(api.LinearOperator.from_lma(self.A), prec, self.diag, "cg",
                                      r_tol=r_tol, max_iter=max_iter)
        self.lin_t = api.LinearOperator(ctx, _linop_transpose(ctx, self.A), [self.A])
        self.cg_t = api.IterativeSolver(self.lin_t, prec, self.diag, "cg", r_tol=r_tol,
                                        max_iter=max_iter)
        self.stream = torch.cuda.Stream()
        ctx.set_stream(self.stream.cuda_stream)

    # -- helpers ------------------------------------------------------------
    def wrap(self, t: torch.Tensor, ncol: int, nlev: int) -> Field:
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
            raise TypeError("expected a contiguous float64 CUDA tensor")
        if t.numel() != ncol * nlev:
            raise ValueError(f"tensor of {t.numel()} values for a field of {ncol * nlev}")
        return Field(self.ctx, R_DOUBLE, ncol, nlev, device_ptr=t.data_ptr())

    def w0_field(self, t):
        return self.wrap(t, self.nent, self.nlev)

    def begin(self, *tensors):
        self.stream.wait_stream(torch.cuda.current_stream())
        for t in tensors:
            t.record_stream(self.stream)

    def end(self):
        torch.cuda.current_stream().wait_stream(self.stream)

    # -- operator and solves -------------------------------------------------
    def assemble(self, kappa: torch.Tensor):
        """A = M + kappa K on the device; Jacobi diagonal of A."""
        kf = self.wrap(kappa, self.ncell, self.nl)
        self.A.combine(self.M, self.K, kf)
        self.diag.set_scalar(0.0)
        self.A.diagonal(self.diag)

    def solve(self, f: torch.Tensor, u: torch.Tensor, transpose: bool = False):
        u.zero_()
        res = (self.cg_t if transpose else self.cg).apply(self.w0_field(u), self.w0_field(f))
        if res.status != api.OK:
            raise api.LfgError(res.status, f"{'adjoint' if transpose else 'forward'} CG "
                                           f"failed after {res.iterations} iterations")
        return res

    def apply(self, x: torch.Tensor, y: torch.Tensor, transpose: bool = False):
        y.zero_()
        mode = api.LMA_TRANSPOSE if transpose else api.LMA_INC
        self.A.apply(mode, self.w0_field(y), self.w0_field(x))

    def kappa_gradient(self, lam: torch.Tensor, u: torch.Tensor, g: torch.Tensor):
        """g(cell, layer) = - lambda_e^T K_e u_e."""
        self.K.bilinear(self.w0_field(lam), self.w0_field(u), -1.0,
                        self.wrap(g, self.ncell, self.nl))

    def tangent(self, u: torch.Tensor, df: torch.Tensor, dkappa: torch.Tensor,
                du: torch.Tensor):
        """Tangent-linear model: A du = df - (dkappa K) u."""
        tmp = torch.empty_like(u)
        self.zero_k = getattr(self, "zero_k", None) or LocalOperator(
            self.ctx, R_DOUBLE, self.ncell, self.nl, np.zeros_like(self.prob.mass), self.prob.map,
            self.nent, self.nlev)
        self.zero_k.combine(self.zero, self.K, self.wrap(dkappa, self.ncell, self.nl))
        tmp.zero_()
        self.zero_k.apply(api.LMA_INC, self.w0_field(tmp), self.w0_field(u))
        rhs = df - tmp
        self.solve(rhs, du)


def _linop_transpose(ctx, lma: LocalOperator):
    import ctypes as C
    h = C.c_void_p()
    ctx.check(ctx.lib.lfg_linop_from_lma_transpose(lma.h, C.byref(h)), "linop_from_lma_transpose")
    return h


class DiffusionSolve(torch.autograd.Function):
    """u = A(kappa)^{-1} f with the hand-written adjoint as its backward."""

    @staticmethod
    def forward(ctx, f, kappa, system: W0Diffusion):
        system.begin(f, kappa)
        u = torch.empty_like(f)
        with torch.cuda.stream(system.stream):
            system.assemble(kappa)
            system.solve(f, u)
        system.end()
        ctx.save_for_backward(kappa, u)
        ctx.system = system
        return u

    @staticmethod
    def backward(ctx, grad_u):
        system = ctx.system
        kappa, u = ctx.saved_tensors
        grad_u = grad_u.contiguous()
        system.begin(kappa, u, grad_u)
        lam = torch.empty_like(u)
        gk = torch.empty_like(kappa)
        with torch.cuda.stream(system.stream):
            system.assemble(kappa)                       # recompute, no stored bases
            system.solve(grad_u, lam, transpose=True)    # lambda = A^{-T} grad_u
            system.kappa_gradient(lam, u, gk)
        system.end()
        return lam, gk, None


class LmaApply(torch.autograd.Function):
    """y = A x for a fixed assembled operator; backward y -> A^T grad."""

    @staticmethod
    def forward(ctx, x, system: W0Diffusion):
        system.begin(x)
        y = torch.empty_like(x)
        with torch.cuda.stream(system.stream):
            system.apply(x, y)
        system.end()
        ctx.system = system
        return y

    @staticmethod
    def backward(ctx, gy):
        system = ctx.system
        gy = gy.contiguous()
        system.begin(gy)
        gx = torch.empty_like(gy)
        with torch.cuda.stream(system.stream):
            system.apply(gy, gx, transpose=True)
        system.end()
        return gx, None

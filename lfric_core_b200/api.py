"""Python front end of the C ABI (include/lfg.h).

Each class owns one ABI handle and mirrors a reference type:

  Field              field_type data + abstract_vector_type algebra
                     (infrastructure/source/field/vector_mod.F90:17-189)
  ColumnwiseOperator columnwise_operator_type (operator/columnwise_operator_mod.f90)
  LocalOperator      operator_type LMA (operator/operator_mod.t90)
  Helmholtz          the project-defined W3 Helmholtz operator
  LinearOperator     abstract_linear_operator_type (solver/sci_linear_operator_mod.f90)
  Preconditioner     abstract_preconditioner_type (solver/sci_preconditioner_mod.f90)
  IterativeSolver    abstract_iterative_solver_type and its solvers
                     (solver/sci_iterative_solver_mod.f90)
  BatchedHelmholtz   many independent Helmholtz solves in one persistent launch

Errors come back as LfgError carrying the ABI status; the solver's
NOT_CONVERGED / NAN statuses are returned, not raised, as the reference's
fail_on_non_converged decides what is fatal.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import lfg_batch_cfg, lfg_solver_cfg

R_SINGLE, R_DOUBLE = 4, 8
OK, NOT_CONVERGED, NAN_STATUS = 0, 1, 2
LMA_INC, LMA_WRITE, LMA_TRANSPOSE = 0, 1, 2
RESTRICT_UNWEIGHTED, RESTRICT_WEIGHTED, RESTRICT_MASS_W3 = 0, 1, 2
SOLVERS = {"cg": 0, "gcr": 1, "jacobi": 2, "chebyshev": 3, "precondition_only": 4,
           "bicgstab": 5, "gmres": 6, "fgmres": 7, "block_gcr": 8}


class LfgError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[status {status}] {message}")
        self.status = status


def _kind_of(dtype) -> int:
    dt = np.dtype(dtype)
    if dt == np.float64:
        return R_DOUBLE
    if dt == np.float32:
        return R_SINGLE
    raise TypeError(f"unsupported dtype {dt}")


def _dtype_of(kind: int):
    return np.float64 if kind == R_DOUBLE else np.float32


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Context:
    """One CUDA device and stream; owns every device buffer made through it."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        st = self.lib.lfg_ctx_create(device, C.byref(h))
        if st != OK:
            raise LfgError(st, "lfg_ctx_create failed (is a CUDA device present?)")
        self.h = h

    def check(self, status: int, what: str = "") -> int:
        if status not in (OK,):
            msg = self.lib.lfg_last_error(self.h).decode()
            raise LfgError(status, f"{what}: {msg}" if what else msg)
        return status

    def synchronize(self):
        self.check(self.lib.lfg_ctx_synchronize(self.h), "synchronize")

    def set_stream(self, stream_ptr: int | None):
        self.check(self.lib.lfg_ctx_set_stream(self.h, C.c_void_p(stream_ptr or 0)), "set_stream")

    def test_tma_spin_limit(self, spins: int):
        """Test hook: TMA stage waits give up after `spins` polls (< 0: the
        built-in limit)."""
        self.check(self.lib.lfg_ctx_test_tma_spin_limit(self.h, C.c_longlong(spins)),
                   "test_tma_spin_limit")

    def kernel_launches(self) -> int:
        n = C.c_uint64()
        self.check(self.lib.lfg_ctx_kernel_launches(self.h, C.byref(n)))
        return n.value

    def algorithmic_bytes(self) -> int:
        """Bytes the launched kernels must move at least: each array a kernel
        reads or writes counted once, at its stored precision."""
        n = C.c_uint64()
        self.check(self.lib.lfg_ctx_algorithmic_bytes(self.h, C.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.lfg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Handle:
    _destroy = None

    def __init__(self, ctx: Context, h, keep=()):
        self.ctx, self.h, self._keep = ctx, h, list(keep)

    def close(self):
        # after the context is gone its objects may not be touched (their
        # memory went with the device context); drop the handle only
        if getattr(self, "h", None) and self._destroy and getattr(self.ctx, "h", None):
            getattr(self.ctx.lib, self._destroy)(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Field(_Handle):
    """A column field: ncol entities x nlev levels, level-major on the device."""

    _destroy = "lfg_field_destroy"

    def __init__(self, ctx: Context, kind: int, ncol: int, nlev: int, device_ptr: int | None = None,
                 keep=()):
        h = C.c_void_p()
        if device_ptr is None:
            ctx.check(ctx.lib.lfg_field_create(ctx.h, kind, ncol, nlev, C.byref(h)), "field_create")
        else:
            ctx.check(ctx.lib.lfg_field_wrap(ctx.h, kind, ncol, nlev, C.c_void_p(device_ptr),
                                             C.byref(h)), "field_wrap")
        super().__init__(ctx, h, keep)
        self.kind, self.ncol, self.nlev = kind, ncol, nlev

    @property
    def size(self) -> int:
        return self.ncol * self.nlev

    def device_ptr(self) -> int:
        p = C.c_void_p()
        self.ctx.check(self.ctx.lib.lfg_field_device_ptr(self.h, C.byref(p)))
        return p.value

    def import_(self, data: np.ndarray) -> "Field":
        """Copy a host array in the reference's column-contiguous order in."""
        a = np.ascontiguousarray(data)
        if a.size != self.size:
            raise ValueError(f"import: {a.size} values for a field of {self.size}")
        self.ctx.check(self.ctx.lib.lfg_field_import(self.h, a.ctypes.data_as(C.c_void_p),
                                                     _kind_of(a.dtype)), "field_import")
        return self

    def export(self, dtype=None) -> np.ndarray:
        dt = np.dtype(dtype or _dtype_of(self.kind))
        out = np.empty(self.size, dtype=dt)
        self.ctx.check(self.ctx.lib.lfg_field_export(self.h, out.ctypes.data_as(C.c_void_p),
                                                     _kind_of(dt)), "field_export")
        return out

    def export_into(self, out: np.ndarray) -> np.ndarray:
        self.ctx.check(self.ctx.lib.lfg_field_export(self.h, out.ctypes.data_as(C.c_void_p),
                                                     _kind_of(out.dtype)), "field_export")
        return out

    # abstract_vector_type bindings (vector_mod.F90:17-59)
    def set_scalar(self, a: float):
        self.ctx.check(self.ctx.lib.lfg_setval_c(self.h, a), "setval_c")

    def copy(self, src: "Field"):
        self.ctx.check(self.ctx.lib.lfg_setval_X(self.h, src.h), "setval_X")

    def axpy(self, alpha: float, x: "Field"):      # self = self + alpha x
        self.ctx.check(self.ctx.lib.lfg_inc_X_plus_bY(self.h, alpha, x.h), "inc_X_plus_bY")

    def aypx(self, alpha: float, x: "Field"):      # self = alpha self + x
        self.ctx.check(self.ctx.lib.lfg_inc_aX_plus_Y(alpha, self.h, x.h), "inc_aX_plus_Y")

    def axpby(self, a: float, x: "Field", b: float, y: "Field"):  # self = a x + b y
        self.ctx.check(self.ctx.lib.lfg_aX_plus_bY(self.h, a, x.h, b, y.h), "aX_plus_bY")

    def scale(self, a: float):
        self.ctx.check(self.ctx.lib.lfg_inc_a_times_X(a, self.h), "inc_a_times_X")

    def divide(self, x: "Field", y: "Field"):      # self = x / y
        self.ctx.check(self.ctx.lib.lfg_X_divideby_Y(self.h, x.h, y.h), "X_divideby_Y")

    def dot(self, x: "Field") -> float:
        r = C.c_double()
        self.ctx.check(self.ctx.lib.lfg_X_innerproduct_Y(self.h, x.h, C.byref(r)), "innerproduct")
        return r.value

    def dot_into(self, x: "Field", device_ptr: int):
        """<self, x> written to the double at device_ptr in stream order
        (no host synchronisation)."""
        self.ctx.check(self.ctx.lib.lfg_X_innerproduct_Y_device(self.h, x.h,
                                                                C.c_void_p(device_ptr)),
                       "innerproduct_device")

    def norm(self) -> float:
        r = C.c_double()
        self.ctx.check(self.ctx.lib.lfg_X_innerproduct_X(self.h, C.byref(r)), "innerproduct")
        return float(np.sqrt(r.value))

    def duplicate(self) -> "Field":
        return Field(self.ctx, self.kind, self.ncol, self.nlev)


def field_from(ctx: Context, data: np.ndarray, ncol: int, nlev: int, kind: int | None = None) -> Field:
    kind = kind or _kind_of(np.asarray(data).dtype)
    return Field(ctx, kind, ncol, nlev).import_(data)


class Mesh(_Handle):
    _destroy = "lfg_mesh_destroy"

    def __init__(self, ctx: Context, links: np.ndarray):
        links = np.ascontiguousarray(links, dtype=np.int32)
        h = C.c_void_p()
        ctx.check(ctx.lib.lfg_mesh_create(ctx.h, links.shape[0], _iptr(links), C.byref(h)),
                  "mesh_create")
        super().__init__(ctx, h)
        self.ncol = links.shape[0]


class Intergrid(_Handle):
    """cell_map: (ncoarse, ny, nx) fine cells of each coarse cell (0-based)."""

    _destroy = "lfg_intergrid_destroy"

    def __init__(self, ctx: Context, cell_map: np.ndarray, nfine: int,
                 coarse_corners: np.ndarray | None = None, fine_corners: np.ndarray | None = None):
        cm = np.ascontiguousarray(cell_map, dtype=np.int32)
        ncoarse, ny, nx = cm.shape
        cc = None if coarse_corners is None else np.ascontiguousarray(coarse_corners, dtype=np.int32)
        fc = None if fine_corners is None else np.ascontiguousarray(fine_corners, dtype=np.int32)
        h = C.c_void_p()
        ctx.check(ctx.lib.lfg_intergrid_create(
            ctx.h, ncoarse, nfine, nx, ny, _iptr(cm), None if cc is None else _iptr(cc),
            None if fc is None else _iptr(fc), C.byref(h)), "intergrid_create")
        super().__init__(ctx, h)
        self.ncoarse, self.nfine, self.nx, self.ny = ncoarse, nfine, nx, ny

    def restrict(self, mode: int, coarse: Field, fine: Field, weights: Field | None = None):
        self.ctx.check(self.ctx.lib.lfg_restrict_scalar(self.h, mode, coarse.h, fine.h,
                                                        None if weights is None else weights.h),
                       "restrict_scalar")

    def prolong(self, fine: Field, coarse: Field, weights: Field | None = None):
        self.ctx.check(self.ctx.lib.lfg_prolong_scalar(self.h, fine.h, coarse.h,
                                                       None if weights is None else weights.h),
                       "prolong_scalar")

    def restrict_w0(self, coarse: Field, fine: Field):
        self.ctx.check(self.ctx.lib.lfg_restrict_w0(self.h, coarse.h, fine.h), "restrict_w0")

    def prolong_w0(self, fine: Field, coarse: Field):
        self.ctx.check(self.ctx.lib.lfg_prolong_w0(self.h, fine.h, coarse.h), "prolong_w0")


W2_FULL, W2_H, W2_V = 0, 1, 2


class W2Map(_Handle):
    """W2 intergrid maps for lfg_w2_*: 0-based dofmaps (ncell, ndf) of the
    coarse and fine W2 spaces on an Intergrid's meshes, face selectors per
    coarse cell.  Fields are flat (undf x 1) in the reference's dof order."""

    _destroy = "lfg_w2map_destroy"

    def __init__(self, ig: "Intergrid", nlayers: int, map_coarse, undf_coarse: int, map_fine,
                 undf_fine: int, sel_ew=None, sel_ns=None):
        mc = np.ascontiguousarray(map_coarse, dtype=np.int32)
        mf = np.ascontiguousarray(map_fine, dtype=np.int32)
        ew = None if sel_ew is None else np.ascontiguousarray(sel_ew, dtype=np.int32)
        ns = None if sel_ns is None else np.ascontiguousarray(sel_ns, dtype=np.int32)
        h = C.c_void_p()
        ig.ctx.check(ig.ctx.lib.lfg_w2map_create(
            ig.h, nlayers, mc.shape[1], _iptr(mc), undf_coarse, _iptr(mf), undf_fine,
            None if ew is None else _iptr(ew), None if ns is None else _iptr(ns), C.byref(h)),
            "w2map_create")
        super().__init__(ig.ctx, h, [ig])
        self.undf_coarse, self.undf_fine = undf_coarse, undf_fine

    @classmethod
    def columns(cls, ig: "Intergrid", nlayers: int, col_coarse, ncol_coarse: int, col_fine,
                ncol_fine: int, sel_ew, sel_ns) -> "W2Map":
        """The same transfers on W2 fields held as level-major columns
        (ncol, nlayers+1), the layout of the W2 LMA operators: col_* (ncell,
        ndf) give the column of each cell dof."""
        mc = np.ascontiguousarray(col_coarse, dtype=np.int32)
        mf = np.ascontiguousarray(col_fine, dtype=np.int32)
        ew = np.ascontiguousarray(sel_ew, dtype=np.int32)
        ns = np.ascontiguousarray(sel_ns, dtype=np.int32)
        h = C.c_void_p()
        ig.ctx.check(ig.ctx.lib.lfg_w2map_create_columns(
            ig.h, nlayers, mc.shape[1], _iptr(mc), ncol_coarse, _iptr(mf), ncol_fine, _iptr(ew),
            _iptr(ns), C.byref(h)), "w2map_create_columns")
        self = cls.__new__(cls)
        _Handle.__init__(self, ig.ctx, h, [ig])
        self.undf_coarse = ncol_coarse * (nlayers + 1)
        self.undf_fine = ncol_fine * (nlayers + 1)
        return self

    def restrict(self, mode: int, coarse: "Field", fine: "Field"):
        self.ctx.check(self.ctx.lib.lfg_w2_restrict(self.h, mode, coarse.h, fine.h), "w2_restrict")

    def prolong_weights(self, weights: "Field"):
        self.ctx.check(self.ctx.lib.lfg_w2_prolong_weights(self.h, weights.h), "w2_weights")

    def prolong(self, fine: "Field", coarse: "Field", weights: "Field"):
        self.ctx.check(self.ctx.lib.lfg_w2_prolong(self.h, fine.h, coarse.h, weights.h),
                       "w2_prolong")


class ColumnwiseOperator(_Handle):
    """columnwise_operator_type: columnwise_matrix(bw, nrow, ncol) Fortran order."""

    _destroy = "lfg_cma_destroy"

    def __init__(self, ctx: Context, kind: int, ncol: int, nrow: int, ncolumn: int, bandwidth: int,
                 alpha: int, beta: int, gamma_m: int, gamma_p: int, ind_to, ind_from,
                 columnwise_matrix: np.ndarray | None = None):
        it = np.ascontiguousarray(ind_to, dtype=np.int32)
        iff = np.ascontiguousarray(ind_from, dtype=np.int32)
        h = C.c_void_p()
        cm = None
        if columnwise_matrix is not None:
            cm = np.ascontiguousarray(columnwise_matrix, dtype=np.float64).ravel()
        ctx.check(ctx.lib.lfg_cma_create(ctx.h, kind, ncol, nrow, ncolumn, bandwidth, alpha,
                                         beta, gamma_m, gamma_p, _iptr(it), _iptr(iff),
                                         None if cm is None else _dptr(cm), C.byref(h)),
                  "cma_create")
        super().__init__(ctx, h)
        self.kind, self.ncol, self.nrow, self.ncolumn = kind, ncol, nrow, ncolumn
        self.bandwidth = bandwidth
        self.alpha, self.beta, self.gamma_m, self.gamma_p = alpha, beta, gamma_m, gamma_p

    def get(self) -> np.ndarray:
        """columnwise_matrix(bw, nrow, ncol) as a Fortran-ordered array."""
        out = np.empty(self.bandwidth * self.nrow * self.ncol)
        self.ctx.check(self.ctx.lib.lfg_cma_get(self.h, _dptr(out)), "cma_get")
        return out.reshape((self.bandwidth, self.nrow, self.ncol), order="F")

    # CMA assembly and algebra (components/science/source/kernel/columnwise_operators/)
    def assemble(self, lma: "LocalOperator", cb_to, cb_from):
        t = np.asfortranarray(cb_to, dtype=np.int32)
        f = np.asfortranarray(cb_from, dtype=np.int32)
        self.ctx.check(self.ctx.lib.lfg_cma_assemble(self.h, lma.h, _iptr(t.ravel(order="F")),
                                                     _iptr(f.ravel(order="F"))), "cma_assemble")

    def multiply(self, a: "ColumnwiseOperator", b: "ColumnwiseOperator"):     # C += A B
        self.ctx.check(self.ctx.lib.lfg_cma_multiply(self.h, a.h, b.h), "cma_multiply")

    def scaled_add(self, a: "ColumnwiseOperator", b: "ColumnwiseOperator", alpha: float,
                   beta: float):                                                # C = aA + bB
        self.ctx.check(self.ctx.lib.lfg_cma_scaled_add(self.h, a.h, b.h, alpha, beta),
                       "cma_scaled_add")

    def assemble_diag_hmht(self, dh: "LocalOperator", m2h: "LocalOperator", cb):
        t = np.asfortranarray(cb, dtype=np.int32)
        self.ctx.check(self.ctx.lib.lfg_cma_assemble_diag_hmht(self.h, dh.h, m2h.h,
                                                               _iptr(t.ravel(order="F"))),
                       "cma_assemble_diag_hmht")

    def assemble_m2v_lumped_inv(self, m: "LocalOperator", cb):
        t = np.asfortranarray(cb, dtype=np.int32)
        self.ctx.check(self.ctx.lib.lfg_cma_assemble_m2v_lumped_inv(self.h, m.h,
                                                                    _iptr(t.ravel(order="F"))),
                       "cma_assemble_m2v_lumped_inv")

    def apply(self, lhs: Field, x: Field):           # lhs += A x
        self.ctx.check(self.ctx.lib.lfg_cma_apply(self.h, lhs.h, x.h), "cma_apply")

    def apply_inverse(self, lhs: Field, x: Field):   # lhs = A^{-1} x
        self.ctx.check(self.ctx.lib.lfg_cma_apply_inverse(self.h, lhs.h, x.h), "cma_apply_inverse")


def tri_solve(y: Field, x: Field, tri_0: Field, tri_plus: Field, tri_minus: Field):
    y.ctx.check(y.ctx.lib.lfg_tri_solve(y.h, x.h, tri_0.h, tri_plus.h, tri_minus.h), "tri_solve")


class LocalOperator(_Handle):
    """operator_type LMA: local_stencil(ncell*nlayers, ndf_to, ndf_from), Fortran order."""

    _destroy = "lfg_lma_destroy"

    def __init__(self, ctx: Context, kind: int, ncell: int, nlayers: int, local_stencil: np.ndarray,
                 map_to: np.ndarray, nent_to: int, nlev_to: int,
                 map_from: np.ndarray | None = None, nent_from: int | None = None,
                 nlev_from: int | None = None):
        mt = np.ascontiguousarray(map_to, dtype=np.int32)
        mf = mt if map_from is None else np.ascontiguousarray(map_from, dtype=np.int32)
        nent_from = nent_to if nent_from is None else nent_from
        nlev_from = nlev_to if nlev_from is None else nlev_from
        ndf_to, ndf_from = mt.shape[1], mf.shape[1]
        ls = np.ascontiguousarray(local_stencil, dtype=np.float64).ravel()
        h = C.c_void_p()
        ctx.check(ctx.lib.lfg_lma_create(ctx.h, kind, ncell, nlayers, ndf_to, ndf_from, _dptr(ls),
                                         _iptr(mt), nent_to, nlev_to, _iptr(mf), nent_from,
                                         nlev_from, C.byref(h)), "lma_create")
        super().__init__(ctx, h)
        self.kind, self.ncell, self.nlayers = kind, ncell, nlayers
        self.ndf_to, self.ndf_from = ndf_to, ndf_from
        self.nent_to, self.nlev_to, self.nent_from, self.nlev_from = nent_to, nlev_to, nent_from, nlev_from

    def set_values(self, local_stencil: np.ndarray):
        ls = np.ascontiguousarray(local_stencil, dtype=np.float64).ravel()
        self.ctx.check(self.ctx.lib.lfg_lma_set_values(self.h, _dptr(ls)), "lma_set_values")

    def apply(self, mode: int, lhs: Field, x: Field):
        self.ctx.check(self.ctx.lib.lfg_lma_apply(self.h, mode, lhs.h, x.h), "lma_apply")

    def diagonal(self, diag: Field):
        self.ctx.check(self.ctx.lib.lfg_lma_diagonal(self.h, diag.h), "lma_diagonal")

    def operator_tri_solve(self, y: Field, x: Field):
        self.ctx.check(self.ctx.lib.lfg_operator_tri_solve(self.h, y.h, x.h), "operator_tri_solve")

    def combine(self, m: "LocalOperator", k: "LocalOperator", kappa: Field):
        self.ctx.check(self.ctx.lib.lfg_lma_combine(self.h, m.h, k.h, kappa.h), "lma_combine")

    def bilinear(self, u: Field, v: Field, scale: float, g: Field):
        self.ctx.check(self.ctx.lib.lfg_lma_bilinear(self.h, u.h, v.h, scale, g.h), "lma_bilinear")


class Helmholtz(_Handle):
    _destroy = "lfg_helm_destroy"

    def __init__(self, ctx: Context, kind: int, mesh: Mesh, nlayers: int, cm=None, hf=None,
                 handle=None, keep=()):
        if handle is None:
            cm = np.ascontiguousarray(cm, dtype=np.float64).ravel()
            hf = np.ascontiguousarray(hf, dtype=np.float64).ravel()
            handle = C.c_void_p()
            ctx.check(ctx.lib.lfg_helm_create(ctx.h, kind, mesh.h, nlayers, _dptr(cm), _dptr(hf),
                                              C.byref(handle)), "helm_create")
        super().__init__(ctx, handle, [mesh, *keep])
        self.kind, self.mesh, self.nlayers, self.ncol = kind, mesh, nlayers, mesh.ncol

    def apply(self, y: Field, x: Field):
        self.ctx.check(self.ctx.lib.lfg_helm_apply(self.h, y.h, x.h), "helm_apply")

    def smooth(self, omega: float, x_in: Field | None, b: Field, x_out: Field):
        self.ctx.check(self.ctx.lib.lfg_helm_smooth(self.h, omega, None if x_in is None else x_in.h,
                                                    b.h, x_out.h), "helm_smooth")

    def residual_restrict(self, ig: "Intergrid", x: Field, b: Field, coarse_b: Field):
        """coarse_b = restrict_mass_w3(b - A x) in one launch."""
        self.ctx.check(self.ctx.lib.lfg_helm_residual_restrict(self.h, ig.h, x.h, b.h,
                                                               coarse_b.h),
                       "helm_residual_restrict")

    def sweep_rhs(self, x: Field, b: Field, r: Field):
        """r = b + H_off x (the right-hand side of a column sweep)."""
        self.ctx.check(self.ctx.lib.lfg_helm_sweep_rhs(self.h, x.h, b.h, r.h), "helm_sweep_rhs")

    def coarsen(self, ig: Intergrid, coarse_mesh: Mesh, kind: int) -> "Helmholtz":
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.lfg_helm_coarsen(self.h, ig.h, coarse_mesh.h, kind, C.byref(h)),
                       "helm_coarsen")
        return Helmholtz(self.ctx, kind, coarse_mesh, self.nlayers, handle=h)

    def copy_kind(self, kind: int) -> "Helmholtz":
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.lfg_helm_copy_kind(self.h, kind, C.byref(h)), "helm_copy_kind")
        return Helmholtz(self.ctx, kind, self.mesh, self.nlayers, handle=h)

    def field(self, data=None) -> Field:
        f = Field(self.ctx, self.kind, self.ncol, self.nlayers)
        if data is not None:
            f.import_(data)
        return f


class LinearOperator(_Handle):
    _destroy = "lfg_linop_destroy"

    @classmethod
    def from_helmholtz(cls, op: Helmholtz) -> "LinearOperator":
        h = C.c_void_p()
        op.ctx.check(op.ctx.lib.lfg_linop_from_helm(op.h, C.byref(h)), "linop_from_helm")
        return cls(op.ctx, h, [op])

    @classmethod
    def from_lma(cls, op: LocalOperator) -> "LinearOperator":
        h = C.c_void_p()
        op.ctx.check(op.ctx.lib.lfg_linop_from_lma(op.h, C.byref(h)), "linop_from_lma")
        return cls(op.ctx, h, [op])

    def apply(self, x: Field, y: Field):
        self.ctx.check(self.ctx.lib.lfg_linop_apply(self.h, x.h, y.h), "linop_apply")


class Preconditioner(_Handle):
    _destroy = "lfg_prec_destroy"

    @classmethod
    def null(cls, ctx: Context) -> "Preconditioner":
        h = C.c_void_p()
        ctx.check(ctx.lib.lfg_prec_null(ctx.h, C.byref(h)), "prec_null")
        return cls(ctx, h)

    @classmethod
    def diagonal(cls, diag: Field) -> "Preconditioner":
        h = C.c_void_p()
        diag.ctx.check(diag.ctx.lib.lfg_prec_diagonal(diag.h, C.byref(h)), "prec_diagonal")
        return cls(diag.ctx, h, [diag])

    @classmethod
    def multigrid(cls, levels: list, maps: list, n_pre=2, n_post=2, n_coarse=8,
                  omega=0.8) -> "Preconditioner":
        ctx = levels[0].ctx
        lv = (C.c_void_p * len(levels))(*[l.h.value for l in levels])
        mp = (C.c_void_p * max(1, len(maps)))(*[m.h.value for m in maps])
        h = C.c_void_p()
        ctx.check(ctx.lib.lfg_prec_multigrid(len(levels), C.cast(lv, C.POINTER(C.c_void_p)),
                                             C.cast(mp, C.POINTER(C.c_void_p)), n_pre, n_post,
                                             n_coarse, omega, C.byref(h)), "prec_multigrid")
        return cls(ctx, h, [*levels, *maps])

    @classmethod
    def w2_multigrid(cls, levels: list, maps: list, n_pre=2, n_post=2, n_coarse=8,
                     omega=0.6) -> "Preconditioner":
        """V-cycle over W2 LMA operators (finest first) joined by column-layout
        W2Maps: weighted Jacobi smoothing, restrict_w2 / prolong_w2."""
        ctx = levels[0].ctx
        lv = (C.c_void_p * len(levels))(*[l.h.value for l in levels])
        mp = (C.c_void_p * max(1, len(maps)))(*[m.h.value for m in maps])
        h = C.c_void_p()
        ctx.check(ctx.lib.lfg_prec_w2_multigrid(len(levels), C.cast(lv, C.POINTER(C.c_void_p)),
                                                C.cast(mp, C.POINTER(C.c_void_p)), n_pre,
                                                n_post, n_coarse, omega, C.byref(h)),
                  "prec_w2_multigrid")
        return cls(ctx, h, [*levels, *maps])

    def apply(self, x: Field, y: Field):
        self.ctx.check(self.ctx.lib.lfg_prec_apply(self.h, x.h, y.h), "prec_apply")


@dataclass
class SolveResult:
    status: int
    iterations: int
    final_err: float


class IterativeSolver(_Handle):
    """abstract_iterative_solver_type; method one of SOLVERS."""

    _destroy = "lfg_solver_destroy"

    def __init__(self, lin_op: LinearOperator, prec: Preconditioner, like: Field, method: str,
                 r_tol=1e-8, a_tol=0.0, max_iter=100, monitor_convergence=True,
                 fail_on_non_converged=True, gcrk=10, rho_relax=1.0, lmin=0.0, lmax=1.0):
        cfg = lfg_solver_cfg(SOLVERS[method], gcrk, r_tol, a_tol, max_iter,
                             int(monitor_convergence), int(fail_on_non_converged), rho_relax,
                             lmin, lmax)
        h = C.c_void_p()
        ctx = lin_op.ctx
        ctx.check(ctx.lib.lfg_solver_create(lin_op.h, prec.h, C.byref(cfg), like.h, C.byref(h)),
                  "solver_create")
        super().__init__(ctx, h, [lin_op, prec])
        self.method, self.kind = method, like.kind

    def set_fields(self, offsets):
        """Block GCR: field n is elements [offsets[n], offsets[n+1]) of the
        level-major device vector (a field_vector packed by segments)."""
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        self.ctx.check(self.ctx.lib.lfg_solver_set_fields(
            self.h, len(off) - 1, off.ctypes.data_as(C.POINTER(C.c_int64))), "solver_set_fields")

    def apply(self, x: Field, b: Field) -> SolveResult:
        it, err = C.c_int(), C.c_double()
        st = self.ctx.lib.lfg_solver_apply(self.h, x.h, b.h, C.byref(it), C.byref(err))
        if st not in (OK, NOT_CONVERGED, NAN_STATUS):
            self.ctx.check(st, "solver_apply")
        return SolveResult(st, it.value, err.value)


@dataclass
class MixedResult:
    status: int
    outer_iterations: int
    inner_iterations: int
    rel_residual: float


class MixedSolver(_Handle):
    _destroy = "lfg_mixed_destroy"

    def __init__(self, op64: Helmholtz, inner: IterativeSolver, tol=1e-8, max_outer=10):
        h = C.c_void_p()
        op64.ctx.check(op64.ctx.lib.lfg_mixed_create(op64.h, inner.h, tol, max_outer, C.byref(h)),
                       "mixed_create")
        super().__init__(op64.ctx, h, [op64, inner])

    def apply(self, x: Field, b: Field) -> MixedResult:
        o, i, r = C.c_int(), C.c_int(), C.c_double()
        st = self.ctx.lib.lfg_mixed_apply(self.h, x.h, b.h, C.byref(o), C.byref(i), C.byref(r))
        if st not in (OK, NOT_CONVERGED, NAN_STATUS):
            self.ctx.check(st, "mixed_apply")
        return MixedResult(st, o.value, i.value, r.value)


@dataclass
class BatchResult:
    status: int
    outer_iterations: int
    inner_iterations: int
    rel_residual: float


class BatchedHelmholtz(_Handle):
    """Independent problems A_i x_i = b_i (r_double Helmholtz operators,
    shared or not) solved together by lfg_batch_*: one persistent launch,
    mixed refinement with an inner column-preconditioned FP32 CG."""

    _destroy = "lfg_batch_destroy"

    def __init__(self, ctx: Context, ops: list, tol=1e-8, inner_tol=1e-5, max_outer=10,
                 max_inner=200, tile_cols=0, blocks_per_sm=0, use_graph=True, spin_limit=0):
        if not ops or any(o.kind != R_DOUBLE for o in ops):
            raise ValueError("BatchedHelmholtz: needs r_double Helmholtz operators")
        cfg = lfg_batch_cfg(tol, inner_tol, max_outer, max_inner, tile_cols, blocks_per_sm,
                            int(bool(use_graph)), spin_limit)
        arr = (C.c_void_p * len(ops))(*[o.h.value if isinstance(o.h, C.c_void_p) else o.h
                                        for o in ops])
        h = C.c_void_p()
        ctx.check(ctx.lib.lfg_batch_create(ctx.h, len(ops), arr, C.byref(cfg), C.byref(h)),
                  "batch_create")
        super().__init__(ctx, h, list(ops))
        self.ops = list(ops)

    class _Views:
        """Field views of every problem's rhs or solution; each view keeps
        the batch alive (the batch holds no reference back)."""

        def __init__(self, batch, fn):
            self.batch, self.fn = batch, fn

        def __len__(self):
            return len(self.batch.ops)

        def __getitem__(self, i) -> Field:
            B = self.batch
            if not 0 <= i < len(B.ops):
                raise IndexError(i)
            v = C.c_void_p()
            B.ctx.check(getattr(B.ctx.lib, self.fn)(B.h, i, C.byref(v)), self.fn)
            p = C.c_void_p()
            B.ctx.check(B.ctx.lib.lfg_field_device_ptr(v, C.byref(p)))
            o = B.ops[i]
            return Field(B.ctx, R_DOUBLE, o.ncol, o.nlayers, device_ptr=p.value, keep=[B])

    @property
    def rhs(self) -> "_Views":
        return BatchedHelmholtz._Views(self, "lfg_batch_rhs")

    @property
    def sol(self) -> "_Views":
        return BatchedHelmholtz._Views(self, "lfg_batch_solution")

    def __len__(self):
        return len(self.ops)

    def launch(self):
        self.ctx.check(self.ctx.lib.lfg_batch_launch(self.h), "batch_launch")

    def wait(self) -> int:
        nf = C.c_int()
        self.ctx.check(self.ctx.lib.lfg_batch_wait(self.h, C.byref(nf)), "batch_wait")
        return nf.value

    def solve(self) -> int:
        """Solve every problem from x = 0; returns how many did not reach tol."""
        nf = C.c_int()
        self.ctx.check(self.ctx.lib.lfg_batch_solve(self.h, C.byref(nf)), "batch_solve")
        return nf.value

    def result(self, i: int) -> BatchResult:
        st, o, n, r = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        self.ctx.check(self.ctx.lib.lfg_batch_result(self.h, i, C.byref(st), C.byref(o),
                                                     C.byref(n), C.byref(r)), "batch_result")
        return BatchResult(st.value, o.value, n.value, r.value)

    def tuning(self) -> dict:
        v = [C.c_int() for _ in range(4)]
        self.ctx.check(self.ctx.lib.lfg_batch_tuning(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("tile_cols", "blocks_per_sm", "grid_blocks", "phases"),
                        (x.value for x in v)))

    def test_stall(self, extra: int):
        self.ctx.check(self.ctx.lib.lfg_batch_test_stall(self.h, extra), "batch_test_stall")


class HelmholtzSystem:
    """Device-resident Helmholtz problem: operators of every multigrid level
    (Galerkin, built on the device), FP64 and FP32 V-cycles, the FP64
    GCR(k) solver and the mixed-precision refinement solver."""

    def __init__(self, ctx: Context, prob, gcrk=10, tol=1e-8, max_iter=20, n_pre=2, n_post=2,
                 n_coarse=8, omega=0.8, inner_tol=1e-4, inner_max_iter=2, max_outer=10,
                 mixed=True, fp64=True):
        self.ctx, self.prob = ctx, prob
        nl = prob.nlayers
        self.meshes = [Mesh(ctx, prob.links)] + [Mesh(ctx, l) for l in prob.mg_links]
        self.maps = [Intergrid(ctx, ch, self.meshes[i].ncol) for i, ch in enumerate(prob.mg_child)]
        op64 = Helmholtz(ctx, R_DOUBLE, self.meshes[0], nl, prob.cm, prob.hf)
        self.levels64 = [op64]
        for i, ig in enumerate(self.maps):
            self.levels64.append(self.levels64[-1].coarsen(ig, self.meshes[i + 1], R_DOUBLE))
        self.op64 = op64
        mgkw = dict(n_pre=n_pre, n_post=n_post, n_coarse=n_coarse, omega=omega)
        self.b64 = Field(ctx, R_DOUBLE, op64.ncol, nl)
        self.x64 = Field(ctx, R_DOUBLE, op64.ncol, nl)
        if fp64:
            self.mg64 = Preconditioner.multigrid(self.levels64, self.maps, **mgkw)
            self.gcr64 = IterativeSolver(LinearOperator.from_helmholtz(op64), self.mg64, self.x64,
                                         "gcr", r_tol=tol, max_iter=max_iter, gcrk=gcrk)
        if mixed:
            self.levels32 = [l.copy_kind(R_SINGLE) for l in self.levels64]
            self.mg32 = Preconditioner.multigrid(self.levels32, self.maps, **mgkw)
            like32 = Field(ctx, R_SINGLE, op64.ncol, nl)
            self.gcr32 = IterativeSolver(LinearOperator.from_helmholtz(self.levels32[0]), self.mg32,
                                         like32, "gcr", r_tol=inner_tol, max_iter=inner_max_iter,
                                         gcrk=gcrk, fail_on_non_converged=False)
            self.mixed = MixedSolver(op64, self.gcr32, tol=tol, max_outer=max_outer)

    def solve_fp64(self, b: np.ndarray | None = None) -> SolveResult:
        if b is not None:
            self.b64.import_(b)
        self.x64.set_scalar(0.0)
        return self.gcr64.apply(self.x64, self.b64)

    def solve_mixed(self, b: np.ndarray | None = None) -> MixedResult:
        if b is not None:
            self.b64.import_(b)
        return self.mixed.apply(self.x64, self.b64)

    def solution(self) -> np.ndarray:
        return self.x64.export(np.float64)


class W2System:
    """A W2 hierarchy (problems.W2Hierarchy) on the device: each level's LMA
    operator on (columns, nlayers+1) fields, the column-layout W2 maps
    between consecutive levels, and the multigrid preconditioner over them."""

    def __init__(self, ctx: Context, hier, n_pre=2, n_post=2, n_coarse=8, omega=0.6):
        self.ctx, self.hier = ctx, hier
        self.ops, self.maps, self.igs = [], [], []
        for lev in hier.levels:
            nlev = lev.nlayers + 1
            cmap = (lev.ent.astype(np.int64) * nlev + lev.off).astype(np.int32)
            self.ops.append(LocalOperator(ctx, R_DOUBLE, lev.ncell, lev.nlayers, lev.matrix,
                                          cmap, lev.nent, nlev))
        for l, cm in enumerate(hier.cell_maps):
            fine, coarse = hier.levels[l], hier.levels[l + 1]
            ig = Intergrid(ctx, cm, fine.ncell)
            self.igs.append(ig)
            self.maps.append(W2Map.columns(ig, fine.nlayers, coarse.ent, coarse.nent, fine.ent,
                                           fine.nent, coarse.ew, coarse.ns))
        self.prec = Preconditioner.w2_multigrid(self.ops, self.maps, n_pre, n_post, n_coarse,
                                                omega)

    def field(self, flat=None, level: int = 0) -> Field:
        lev = self.hier.levels[level]
        f = Field(self.ctx, R_DOUBLE, lev.nent, lev.nlayers + 1)
        if flat is not None:
            f.import_(lev.to_columns(flat))
        return f

    def flat(self, f: Field, level: int = 0) -> np.ndarray:
        return self.hier.levels[level].from_columns(f.export())

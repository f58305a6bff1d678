/*
 * lfg.h -- C ABI of the B200 LFRic linear-solver hot path.
 *
 * One call per *invoke* (whole mesh), never per cell.  Every entry point
 * returns an int status (LFG_OK = 0).  All handles are opaque; all arrays
 * crossing the ABI are plain host pointers with explicit sizes, except the
 * *_device_ptr / lfg_field_wrap entry points, which exchange raw CUDA device
 * pointers.  Index arrays are 0-based (the Fortran iso_c_binding shim
 * subtracts one), except the CMA's indirection maps and column-banded
 * dofmaps, which keep the reference's 1-based row and column numbers.  A
 * Fortran caller binds these with bind(C) interfaces, wrapped in types that
 * extend the reference's abstract_linear_operator_type,
 * abstract_preconditioner_type, abstract_vector_type and
 * abstract_iterative_solver_type.
 *
 * Field layout.  A field is the set of dofs of one function space on an
 * extruded mesh: ncol horizontal entities (cells for W3/Wtheta, vertices
 * for W0), each owning nlev vertically stacked dofs.  At the ABI the host
 * array uses the reference's column-contiguous ordering (dof of level k of
 * entity e at e*nlev + k: map(df)+k addressing of
 * infrastructure/source/function_space/
 * function_space_constructor_helper_functions_mod.F90:1940-2160).  On the
 * device fields are stored level-major (k*ncol + e), so that one thread per
 * column reads consecutive addresses across a warp.
 */
#ifndef LFG_H
#define LFG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------------- status */
#define LFG_OK 0
#define LFG_NOT_CONVERGED 1   /* iteration limit reached (fail_on_non_converged) */
#define LFG_NAN 2             /* NaN residual (ieee_is_nan in the reference) */
#define LFG_ERR_ARG 3         /* invalid argument; see lfg_last_error */
#define LFG_ERR_CUDA 4        /* CUDA runtime error */
#define LFG_ERR_NOMEM 5       /* device allocation failed */
#define LFG_ERR_STATE 6       /* call made on an object in the wrong state */

/* -------------------------------------------------------------- real kinds */
#define LFG_R_SINGLE 4        /* r_single / r_solver = real32 */
#define LFG_R_DOUBLE 8        /* r_double / r_def = real64 */

typedef struct lfg_ctx_s* lfg_ctx;
typedef struct lfg_field_s* lfg_field;
typedef struct lfg_mesh_s* lfg_mesh;
typedef struct lfg_intergrid_s* lfg_intergrid;
typedef struct lfg_cma_s* lfg_cma;
typedef struct lfg_lma_s* lfg_lma;
typedef struct lfg_helm_s* lfg_helm;
typedef struct lfg_linop_s* lfg_linop;
typedef struct lfg_prec_s* lfg_prec;
typedef struct lfg_solver_s* lfg_solver;

/* ---------------------------------------------------------------- context
 * A context owns one CUDA stream and every device buffer created through
 * it.  Calls on one context are serialised by the caller (the reference runs
 * one solver per MPI rank, not re-entrant). */
int lfg_ctx_create(int device, lfg_ctx* ctx);
int lfg_ctx_destroy(lfg_ctx ctx);
/* Use an external cudaStream_t (passed as void*); NULL restores the own stream. */
int lfg_ctx_set_stream(lfg_ctx ctx, void* stream);
/* Waits for the context's stream; LFG_ERR_STATE when a kernel's bounded
 * wait ran out since the last check (solver applies check the same). */
int lfg_ctx_synchronize(lfg_ctx ctx);
/* Number of kernels this library has launched on the context so far. */
int lfg_ctx_kernel_launches(lfg_ctx ctx, uint64_t* count);
/* Algorithmic bytes of those kernels: every array a kernel reads counted
 * once and every array it writes counted once, at its stored precision
 * (index maps not counted); kernels replayed from a solver's CUDA graphs
 * count each replay.  Divided by a solve's time it gives the solve-level
 * bandwidth.  A diagnostic of this library, with no counterpart in the
 * reference. */
int lfg_ctx_algorithmic_bytes(lfg_ctx ctx, uint64_t* bytes);
/* Test hook, no counterpart in the reference: the TMA column substitutions
 * of kernels launched from now on (lfg_helm_smooth on fine meshes) give up
 * a stage wait after `spins` polls (0: at once), record the failure and
 * return after their issued loads have landed, so the next
 * lfg_ctx_synchronize reports LFG_ERR_STATE.  A negative value restores the
 * built-in limit.  Kernels already captured in a solver's CUDA graphs keep
 * the limit they were captured with. */
int lfg_ctx_test_tma_spin_limit(lfg_ctx ctx, long long spins);
/* Message of the last failed call on this context (never NULL). */
const char* lfg_last_error(lfg_ctx ctx);
/* Library version string and the compute capability it was built for. */
const char* lfg_version(void);

/* ----------------------------------------------------------------- fields
 * Replaces field_type/field_proxy data arrays and the abstract_vector_type
 * storage (infrastructure/source/field/vector_mod.F90:17-59). */
int lfg_field_create(lfg_ctx ctx, int kind, int ncol, int nlev, lfg_field* field);
/* Wrap caller-owned device memory (level-major, nlev*ncol values of kind). */
int lfg_field_wrap(lfg_ctx ctx, int kind, int ncol, int nlev, void* device_ptr,
                   lfg_field* field);
int lfg_field_destroy(lfg_field field);
int lfg_field_device_ptr(lfg_field field, void** device_ptr);
/* Halo plumbing of a column-partitioned field (no counterpart in the
 * reference, whose halo exchange is YAXT's, infrastructure/source/utilities/
 * halo_comms_mod.F90): device_buf[k*ncols + i] = field(device_cols[i], k) for
 * every level (pack), the reverse (unpack), and field columns
 * [first, first+count) set to zero at every level.  device_cols and
 * device_buf are device pointers; the calls run on the context's stream. */
int lfg_field_pack_columns(lfg_field field, const int* device_cols, int ncols,
                           void* device_buf);
int lfg_field_unpack_columns(lfg_field field, const int* device_cols, int ncols,
                             const void* device_buf);
int lfg_field_zero_columns(lfg_field field, int first, int count);
/* Copy a host array in the reference's column-contiguous order into the
 * field (import_field, sci_field_vector_mod.x90:307-331); host_kind may
 * differ from the field's kind (the value is converted). */
int lfg_field_import(lfg_field field, const void* host, int host_kind);
int lfg_field_export(lfg_field field, void* host, int host_kind);

/* ------------------------------------------------- vector algebra built-ins
 * PSyclone built-ins invoked by sci_field_vector_mod.x90:132-286 and
 * sci_r_solver_field_vector_mod.x90:119-296.  Scalars are double and are
 * cast to the field's kind before use, as r_solver_field_vector does. */
int lfg_setval_c(lfg_field x, double c);                                /* X = c        */
int lfg_setval_X(lfg_field dst, lfg_field src);                         /* copy, any kinds */
int lfg_inc_X_plus_bY(lfg_field x, double b, lfg_field y);              /* X = X + bY   */
int lfg_inc_aX_plus_Y(double a, lfg_field x, lfg_field y);              /* X = aX + Y   */
int lfg_aX_plus_bY(lfg_field z, double a, lfg_field x, double b, lfg_field y); /* Z = aX+bY */
int lfg_inc_a_times_X(double a, lfg_field x);                           /* X = aX       */
int lfg_X_divideby_Y(lfg_field z, lfg_field x, lfg_field y);            /* Z = X/Y      */
/* Inner products accumulate in double whatever the kind
 * (sci_psykal_light_mod.f90:72-214); deterministic two-level reduction. */
int lfg_X_innerproduct_Y(lfg_field x, lfg_field y, double* result);
int lfg_X_innerproduct_X(lfg_field x, double* result);
/* The same inner product written to one double of device memory, in the
 * context's stream order, without waiting for it (no counterpart in the
 * reference, whose inner products return to the host): for callers that
 * keep Krylov scalars on the device. */
int lfg_X_innerproduct_Y_device(lfg_field x, lfg_field y, void* device_result);

/* ---------------------------------------------------------------- meshes */
/* Horizontal cubed-sphere connectivity: links[4*c + f] is the neighbour of
 * cell c across face f = W,S,E,N (mesh face_face_connectivity). */
int lfg_mesh_create(lfg_ctx ctx, int ncol, const int* links, lfg_mesh* mesh);
int lfg_mesh_destroy(lfg_mesh mesh);

/* Intergrid map of a coarse mesh onto a fine one: cell_map[(C*ny + y)*nx + x]
 * is the fine cell at position (x, y) of coarse cell C (x W->E, y N->S; the
 * reference's cell_map(x, y)).  Optional W0 corner tables (4 vertex ids per
 * cell, SW,SE,NE,NW; NULL when unused) enable the W0 transfers. */
int lfg_intergrid_create(lfg_ctx ctx, int ncoarse, int nfine, int nx, int ny,
                         const int* cell_map, const int* coarse_corners,
                         const int* fine_corners, lfg_intergrid* ig);
int lfg_intergrid_destroy(lfg_intergrid ig);
#define LFG_RESTRICT_UNWEIGHTED 0   /* sci_restrict_scalar_unweighted_kernel_mod.F90:71-183 */
#define LFG_RESTRICT_WEIGHTED 1     /* sci_restrict_scalar_weighted_kernel_mod.F90:77-196  */
#define LFG_RESTRICT_MASS_W3 2      /* sci_restrict_mass_w3_kernel_mod.F90:70-179          */
/* coarse = restrict(fine); weights is a fine field (WEIGHTED only, else NULL). */
int lfg_restrict_scalar(lfg_intergrid ig, int mode, lfg_field coarse, lfg_field fine,
                        lfg_field weights);
/* fine += coarse (weights NULL: sci_prolong_scalar_unweighted_kernel_mod.F90:74-169)
 * fine += weights*coarse (sci_prolong_scalar_weighted_kernel_mod.F90:77-178). */
int lfg_prolong_scalar(lfg_intergrid ig, lfg_field fine, lfg_field coarse, lfg_field weights);
/* W0 injection (sci_restrict_w0_kernel_mod.F90:75-154) and bilinear
 * prolongation (sci_prolong_w0_kernel_mod.F90:76-194); fields have
 * nlev = nlayers+1 and one column per vertex. */
int lfg_restrict_w0(lfg_intergrid ig, lfg_field coarse, lfg_field fine);
int lfg_prolong_w0(lfg_intergrid ig, lfg_field fine, lfg_field coarse);

/* W2 intergrid transfers (components/science/source/kernel/inter_mesh/) on
 * flat W2 fields (ncol = undf, nlev = 1) in the reference's dof order.
 * map_coarse[C*ndf + df] / map_fine[c*ndf + df]: 0-based dof of level 0 of
 * cell dof df (W, S, E, N, B, T for ndf 6 and W, S, E, N for ndf 4; B, T for
 * ndf 2); face selectors (1 or 2 per coarse cell) say how many of the E-W
 * and N-S faces the cell writes, as the reference's face_selector fields. */
typedef struct lfg_w2map_s* lfg_w2map;
int lfg_w2map_create(lfg_intergrid ig, int nlayers, int ndf, const int* map_coarse,
                     int undf_coarse, const int* map_fine, int undf_fine,
                     const int* face_selector_ew, const int* face_selector_ns, lfg_w2map* map);
/* The same transfers on W2 fields held as level-major columns, the layout
 * the LMA operators use (no counterpart in the reference, whose W2 fields
 * are flat): every side face and every cell's vertical faces form one
 * column of nlayers+1 levels (a side face uses the first nlayers), a field
 * is (ncol, nlayers+1), and col_coarse[C*ndf + df] / col_fine[c*ndf + df]
 * give the column of cell dof df (T is read through B's column). */
int lfg_w2map_create_columns(lfg_intergrid ig, int nlayers, int ndf, const int* col_coarse,
                             int ncol_coarse, const int* col_fine, int ncol_fine,
                             const int* face_selector_ew, const int* face_selector_ns,
                             lfg_w2map* map);
int lfg_w2map_destroy(lfg_w2map map);
#define LFG_W2_FULL 0   /* restrict_w2  (sci_restrict_w2_kernel_mod.F90)  */
#define LFG_W2_H 1      /* restrict_w2h (sci_restrict_w2h_kernel_mod.F90) */
#define LFG_W2_V 2      /* restrict_w2v (sci_restrict_w2v_kernel_mod.F90) */
int lfg_w2_restrict(lfg_w2map map, int mode, lfg_field coarse, lfg_field fine);
/* weights_prolong_w2_kernel_code (sci_weights_prolong_w2_kernel_mod.F90) */
int lfg_w2_prolong_weights(lfg_w2map map, lfg_field weights);
/* prolong_w2_kernel_code (sci_prolong_w2_kernel_mod.F90) */
int lfg_w2_prolong(lfg_w2map map, lfg_field fine, lfg_field coarse, lfg_field weights);

/* ------------------------------------------------------------ CMA operators
 * columnwise_operator_type (infrastructure/source/operator/
 * columnwise_operator_mod.f90:42-114): banded column matrices
 * columnwise_matrix(bandwidth, nrow, ncol) in Fortran order, with the
 * parameters alpha, beta, gamma_m, gamma_p and the indirection maps
 * (1-based, as built by build_dofmaps :350-396). */
int lfg_cma_create(lfg_ctx ctx, int kind, int ncol, int nrow, int ncolumn, int bandwidth,
                   int alpha, int beta, int gamma_m, int gamma_p,
                   const int* indirection_to, const int* indirection_from,
                   const double* columnwise_matrix, lfg_cma* cma);
int lfg_cma_destroy(lfg_cma cma);
/* The bands in the reference layout columnwise_matrix(bandwidth, nrow, ncell)
 * (columnwise_operator_mod.f90:411-413); lfg_cma_create takes the same
 * layout (NULL: all zero). */
int lfg_cma_get(lfg_cma cma, double* columnwise_matrix);
/* lhs += A x (sci_columnwise_op_app_kernel_mod.F90:73-124). */
int lfg_cma_apply(lfg_cma cma, lfg_field lhs, lfg_field x);
/* lhs += A^T x: the adjoint of lfg_cma_apply (lhs on the from-space, x on
 * the to-space); each output row gathers the band entries that reach it. */
int lfg_cma_apply_transpose(lfg_cma cma, lfg_field lhs, lfg_field x);
/* lhs = A^{-1} x for a tridiagonal A (bandwidth 3), Thomas algorithm
 * (sci_columnwise_op_appinv_kernel_mod.F90:77-145). */
int lfg_cma_apply_inverse(lfg_cma cma, lfg_field lhs, lfg_field x);
/* Thomas solve with three W3 band fields (sci_tri_solve_kernel_mod.f90:72-156). */
int lfg_tri_solve(lfg_field y, lfg_field x, lfg_field tri_0, lfg_field tri_plus,
                  lfg_field tri_minus);

/* Thomas solve of the tri_solve kernel for callers that cannot allocate
 * device memory.  No counterpart in the reference: it exists for hosts whose
 * device memory is owned by another allocator (an application that reserves
 * the GPU's memory up front, a caching pool) or that are recovering from an
 * out-of-memory error, and so cannot call cudaMalloc or create a context.
 * The caller passes level-major device arrays (nlev*ncol values of `kind`)
 * on the current device and a cudaStream_t (NULL: the legacy default
 * stream).  Working storage is one file-scope device array of
 * LFG_NOALLOC_SCRATCH_BYTES that every GPU loading the library keeps until
 * exit; a call needs 2*nlev*ncol*kind bytes of it and fails with
 * LFG_ERR_ARG beyond that.
 * Set-up per device: the array's device address is looked up and the
 * library's device code loaded on that device, which may itself need
 * memory.  lfg_ctx_create does this for its device.  On a device where no
 * context was ever created, the first call does it instead: make that first
 * call (or create a context) before memory runs short, and before any
 * stream capture.
 * The status is that of this call's own launch; errors left by the caller's
 * earlier work are neither reported nor cleared.  All calls share the
 * array: calls whose kernels overlap on the GPU (different streams, or
 * other host threads) race on it.  Nothing in it needs clearing; each call
 * writes its part before reading it. */
#define LFG_NOALLOC_SCRATCH_BYTES (32u << 20)
int lfg_tri_solve_noalloc(int kind, int ncol, int nlev, const void* x, const void* tri_0,
                          const void* tri_plus, const void* tri_minus, void* y,
                          void* stream);

/* ------------------------------------------------- CMA assembly
 * column_banded_dofmap(ndf, nlayers) is 1-based, df fastest: the row (or
 * column) of dof df of layer k in the column matrix, (k-1)(ndof_interior +
 * ndof_face) + df as columnwise_operator_type builds it
 * (columnwise_operator_mod.f90:377-393).  The LMA's cells are the CMA's
 * columns. */
/* C = the LMA's element matrices placed in the bands
 * (columnwise_op_asm_kernel_code, sci_columnwise_op_asm_kernel_mod.F90). */
int lfg_cma_assemble(lfg_cma c, lfg_lma a, const int* column_banded_dofmap_to,
                     const int* column_banded_dofmap_from);
/* C += A B (columnwise_op_mul_kernel_code, sci_columnwise_op_mul_kernel_mod.F90). */
int lfg_cma_multiply(lfg_cma c, lfg_cma a, lfg_cma b);
/* C = alpha A + beta B (columnwise_op_scaledadd_kernel_code,
 * sci_columnwise_op_scaledadd_kernel_mod.F90). */
int lfg_cma_scaled_add(lfg_cma c, lfg_cma a, lfg_cma b, double alpha, double beta);
/* C = per-cell Dh M2h^-1 Dh^T with M2h taken diagonal
 * (columnwise_op_asm_diag_hmht_kernel_code,
 * sci_columnwise_op_asm_diag_hmht_kernel_mod.F90); dh maps W2h -> W3. */
int lfg_cma_assemble_diag_hmht(lfg_cma c, lfg_lma dh, lfg_lma m2h,
                               const int* column_banded_dofmap);
/* C = inverse of the lumped diagonal of M (columnwise_op_asm_m2v_lumped_inv_krnl_code,
 * sci_columnwise_op_asm_m2v_lumped_inv_krnl_mod.F90). */
int lfg_cma_assemble_m2v_lumped_inv(lfg_cma c, lfg_lma m, const int* column_banded_dofmap);

/* ------------------------------------------------------------ LMA operators
 * operator_type local_stencil(ncell*nlayers, ndf_to, ndf_from) in Fortran
 * order (infrastructure/source/operator/operator_mod.t90:113-119) with the
 * dofmaps map_to(ndf_to, ncell) and map_from(ndf_from, ncell): 0-based
 * reference dof of level 0 of each cell dof, in the column-contiguous
 * ordering entity*nlev + offset. */
int lfg_lma_create(lfg_ctx ctx, int kind, int ncell, int nlayers, int ndf_to,
                   int ndf_from, const double* local_stencil, const int* map_to,
                   int nent_to, int nlev_to, const int* map_from, int nent_from,
                   int nlev_from, lfg_lma* lma);
int lfg_lma_destroy(lfg_lma lma);
int lfg_lma_set_values(lfg_lma lma, const double* local_stencil);
#define LFG_LMA_INC 0        /* lhs += A x   matrix_vector_kernel_mod.F90:107-140           */
#define LFG_LMA_WRITE 1      /* lhs  = A x   dg_matrix_vector_kernel_mod.F90:113-154        */
#define LFG_LMA_TRANSPOSE 2  /* lhs += A^T x transpose_matrix_vector_kernel_mod.F90:107-144 */
int lfg_lma_apply(lfg_lma lma, int mode, lfg_field lhs, lfg_field x);
/* diag += diag(A) (sci_mm_diagonal_kernel_mod.F90:99-127). */
int lfg_lma_diagonal(lfg_lma lma, lfg_field diag);
/* Tridiagonal solve with the matrix assembled from a 2x2 Wtheta LMA
 * (sci_operator_tri_solve_kernel_mod.f90:69-120): y, x have nlev = nlayers+1. */
int lfg_operator_tri_solve(lfg_lma lma, lfg_field y, lfg_field x);
/* A_out = M + kappa(cell,layer) * K, per cell (for coefficient-dependent
 * assembly, e.g. the adjoint test); kappa is a field with nlev = nlayers. */
int lfg_lma_combine(lfg_lma out, lfg_lma m, lfg_lma k, lfg_field kappa);
/* g(cell,layer) = scale * sum_ij u(i) A_ij v(j) over the cell's dofs. */
int lfg_lma_bilinear(lfg_lma lma, lfg_field u, lfg_field v, double scale, lfg_field g);

/* ----------------------------------------------------- Helmholtz operator
 * W3 operator A = T' - H_off (defined by this project; the reference's
 * Helmholtz operator lives outside lfric_core): columnwise_matrix(3,nl,ncol)
 * tridiagonal T' whose diagonal includes the face couplings, and
 * hface(4,nl,ncol) couplings to the W,S,E,N neighbours. */
int lfg_helm_create(lfg_ctx ctx, int kind, lfg_mesh mesh, int nlayers, const double* cm,
                    const double* hface, lfg_helm* helm);
int lfg_helm_destroy(lfg_helm helm);
int lfg_helm_apply(lfg_helm helm, lfg_field y, lfg_field x);          /* y = A x */
/* One block-Jacobi column sweep x_out = x_in + omega T'^{-1}(b - A x_in);
 * x_in NULL means a zero initial guess. */
int lfg_helm_smooth(lfg_helm helm, double omega, lfg_field x_in, lfg_field b,
                    lfg_field x_out);
/* The multigrid V-cycle's building blocks, one launch each (no counterpart
 * in the reference, whose multigrid lives in the applications):
 * coarse_b = restrict_mass_w3(b - A x), the residual summed over each coarse
 * cell's children in cell_map order
 * (sci_restrict_mass_w3_kernel_mod.F90:126-179 applied to b - A x); */
int lfg_helm_residual_restrict(lfg_helm helm, lfg_intergrid ig, lfg_field x, lfg_field b,
                               lfg_field coarse_b);
/* r = b + H_off x, the right-hand side T' x_out = r of a block-Jacobi
 * column sweep (lfg_helm_smooth's first kernel on fine meshes). */
int lfg_helm_sweep_rhs(lfg_helm helm, lfg_field x, lfg_field b, lfg_field r);
/* Galerkin coarse operator R A P (R = restrict_mass_w3, P = prolong_scalar_unweighted). */
int lfg_helm_coarsen(lfg_helm fine, lfg_intergrid ig, lfg_mesh coarse_mesh, int kind,
                     lfg_helm* coarse);
int lfg_helm_copy_kind(lfg_helm src, int kind, lfg_helm* dst);

/* -------------------------------------------------- abstract solver types
 * abstract_linear_operator_type%apply(x, y)
 *   (components/science/source/solver/sci_linear_operator_mod.f90:18-36),
 * abstract_preconditioner_type%apply(x, y)
 *   (sci_preconditioner_mod.f90:19-38),
 * abstract_iterative_solver_type%apply(x, b)
 *   (sci_iterative_solver_mod.f90:38-57). */
int lfg_linop_from_helm(lfg_helm helm, lfg_linop* op);
int lfg_linop_from_lma(lfg_lma lma, lfg_linop* op);        /* mass_matrix_operator */
/* The transposed operator y = A^T x (transpose_matrix_vector), for adjoint solves. */
int lfg_linop_from_lma_transpose(lfg_lma lma, lfg_linop* op);
int lfg_linop_destroy(lfg_linop op);
int lfg_linop_apply(lfg_linop op, lfg_field x, lfg_field y);          /* y = A x */

int lfg_prec_null(lfg_ctx ctx, lfg_prec* prec);            /* y = x */
int lfg_prec_diagonal(lfg_field diag, lfg_prec* prec);     /* y = x / diag */
/* Multigrid V-cycle over a Helmholtz hierarchy (level 0 finest; the caller
 * keeps the operators and intergrid maps alive).  n_pre/n_post sweeps per
 * level, n_coarse sweeps on the coarsest level, relaxation omega. */
int lfg_prec_multigrid(int nlevels, const lfg_helm* levels, const lfg_intergrid* maps,
                       int n_pre, int n_post, int n_coarse, double omega, lfg_prec* prec);
/* Multigrid V-cycle over W2 LMA operators (abstract_hierarchical_preconditioner_type,
 * components/science/source/solver/sci_hierarchical_preconditioner_mod.f90:22-38):
 * levels[l] is the r_double W2 operator of level l (6 dofs per cell, fields
 * of lfg_w2map_create_columns's layout), maps[l] joins level l to level
 * l+1; weighted Jacobi smoothing (n_pre / n_post sweeps, n_coarse on the
 * coarsest level, relaxation omega), restrict_w2 of the residual and
 * prolong_w2 of the correction. */
int lfg_prec_w2_multigrid(int nlevels, const lfg_lma* levels, const lfg_w2map* maps,
                          int n_pre, int n_post, int n_coarse, double omega, lfg_prec* prec);
int lfg_prec_destroy(lfg_prec prec);
int lfg_prec_apply(lfg_prec prec, lfg_field x, lfg_field y);         /* y = P^{-1} x */

#define LFG_SOLVER_CG 0               /* cg_solve :495-592            */
#define LFG_SOLVER_GCR 1              /* gcr_solve :1288-1408         */
#define LFG_SOLVER_JACOBI 2           /* jacobi_solve :1745-1815      */
#define LFG_SOLVER_CHEBYSHEV 3        /* chebyshev_solve :1868-1940   */
#define LFG_SOLVER_PRECONDITION_ONLY 4 /* precondition_only_solve :1660-1694 */
#define LFG_SOLVER_BICGSTAB 5         /* bicgstab_solve :645-779      */
#define LFG_SOLVER_GMRES 6            /* gmres_solve :830-1003        */
#define LFG_SOLVER_FGMRES 7           /* fgmres_solve :1055-1237      */
#define LFG_SOLVER_BLOCK_GCR 8        /* block_gcr_solve :1461-1628   */
/* Mirrors the constructor arguments of the reference solver types
 * (sci_iterative_solver_mod.f90:100-113, 250-264) and solver_config. */
typedef struct {
  int method;               /* LFG_SOLVER_* */
  int gcrk;                 /* restart length (GCR, GMRES, FGMRES) */
  double r_tol, a_tol;
  int max_iter;
  int monitor_convergence;
  int fail_on_non_converged;
  double rho_relax;         /* Jacobi over-relaxation factor */
  double lmin, lmax;        /* Chebyshev eigenvalue bounds */
} lfg_solver_cfg;
/* All workspace vectors are allocated here, never inside apply. */
int lfg_solver_create(lfg_linop op, lfg_prec prec, const lfg_solver_cfg* cfg,
                      lfg_field like, lfg_solver* solver);
int lfg_solver_destroy(lfg_solver solver);
/* Block GCR only: the vector is a field_vector of n_fields fields stored as
 * consecutive segments of the device field; segment n is elements
 * [offsets[n], offsets[n+1]) of the level-major array (offsets[0] = 0,
 * offsets[n_fields] = ncol*nlev).  Convergence is tested per field
 * (field_norm(n), block_gcr_solve :1509, :1560-1570).  Default: one field. */
int lfg_solver_set_fields(lfg_solver solver, int n_fields, const int64_t* offsets);
/* Solve A x = b.  Returns LFG_OK, or LFG_NOT_CONVERGED / LFG_NAN as the
 * reference would log at LOG_LEVEL_ERROR; iterations and the last monitored
 * relative residual are returned when the pointers are non-NULL. */
int lfg_solver_apply(lfg_solver solver, lfg_field x, lfg_field b, int* iterations,
                     double* final_err);

/* ------------------------------------------------- mixed-precision solve
 * Iterative refinement: FP64 residual b - A x and update x += e, inner
 * FP32 GCR(k) + FP32 multigrid with FP64 inner products, from x = 0 until
 * ||b - A x|| <= tol ||b|| (FP64).  op64 is the FP64 operator, inner the
 * FP32 solver (built over FP32 operators of the same problem). */
typedef struct lfg_mixed_s* lfg_mixed;
int lfg_mixed_create(lfg_helm op64, lfg_solver inner, double tol, int max_outer,
                     lfg_mixed* mixed);
int lfg_mixed_destroy(lfg_mixed mixed);
int lfg_mixed_apply(lfg_mixed mixed, lfg_field x, lfg_field b, int* outer_iterations,
                    int* inner_iterations, double* rel_residual);

/* ------------------------------------------------- batched solves
 * Many independent W3 Helmholtz problems A_i x_i = b_i solved together in
 * one persistent (cooperative) kernel launch, replayed from a CUDA graph.
 * Each problem runs the mixed refinement above with an inner FP32
 * cg_solve (sci_iterative_solver_mod.f90:495-592, monitor on, a_tol 0)
 * preconditioned by the exact column solve T'^{-1} (columnwise_op_appinv,
 * sci_columnwise_op_appinv_kernel_mod.F90:77-145): per outer iteration
 * r = b - A x (FP64), inner CG on A e = float(r) to inner_tol relative or
 * max_inner iterations, x += e (FP64), until ||b - A x|| <= tol ||b||.
 * Problems may share an operator (several right-hand sides).  The batch
 * has no counterpart in the reference, whose solvers handle one problem per
 * call; each problem's arithmetic is that of the single solve. */
typedef struct lfg_batch_s* lfg_batch;
typedef struct {
  double tol;           /* outer FP64 relative residual (1e-8) */
  double inner_tol;     /* inner FP32 CG relative residual (1e-5) */
  int max_outer;        /* refinement steps before LFG_NOT_CONVERGED (10) */
  int max_inner;        /* inner CG iterations per refinement step (200) */
  int tile_cols;        /* columns per tile: 64, 128, 256; 0 = autotune */
  int blocks_per_sm;    /* co-resident CTAs per SM; 0 = autotune */
  int use_graph;        /* 1: replay the launch from a captured CUDA graph */
  long long spin_limit; /* bound on each grid-barrier wait, in spins; 0 = default */
} lfg_batch_cfg;
/* ops[i]: the r_double operator of problem i (borrowed; must outlive the
 * batch).  cfg NULL: the defaults in parentheses above, use_graph 1. */
int lfg_batch_create(lfg_ctx ctx, int nproblems, const lfg_helm* ops, const lfg_batch_cfg* cfg,
                     lfg_batch* batch);
int lfg_batch_destroy(lfg_batch batch);
/* Device views (owned by the batch) of problem i's right-hand side and
 * solution, for lfg_field_import / lfg_field_export. */
int lfg_batch_rhs(lfg_batch batch, int problem, lfg_field* rhs);
int lfg_batch_solution(lfg_batch batch, int problem, lfg_field* x);
/* Enqueue one solve of every problem from x = 0 on the context's stream
 * (the first call autotunes the launch shape and captures the graph). */
int lfg_batch_launch(lfg_batch batch);
/* Wait for it; nfailed = problems that did not reach tol.  LFG_ERR_STATE
 * when a grid-barrier wait ran out or the phase limit was reached. */
int lfg_batch_wait(lfg_batch batch, int* nfailed);
int lfg_batch_solve(lfg_batch batch, int* nfailed);   /* launch + wait */
int lfg_batch_result(lfg_batch batch, int problem, int* status, int* outer_iterations,
                     int* inner_iterations, double* rel_residual);
/* Launch shape in use and the phases (grid barriers) of the last solve. */
int lfg_batch_tuning(lfg_batch batch, int* tile_cols, int* blocks_per_sm, int* grid_blocks,
                     int* phases);
/* Test hook: the grid barrier waits for extra_arrivals CTAs beyond the
 * grid, so every wait runs out after spin_limit spins and the next solve
 * must end with LFG_ERR_STATE.  0 restores normal operation. */
int lfg_batch_test_stall(lfg_batch batch, int extra_arrivals);

#ifdef __cplusplus
}
#endif
#endif /* LFG_H */

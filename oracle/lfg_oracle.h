/*
 * Oracle for the LFRic linear-solver hot path: a plain-C CPU restatement of
 * the reference's kernels and solvers.
 *
 * TEST INFRASTRUCTURE ONLY.  Only the tests, the smoke check and the
 * CPU-baseline leg of the benchmark may load this library; it is the checker,
 * never the thing measured or shipped.  The reference itself is Fortran and
 * no Fortran compiler exists in this image, so this restatement stands in for
 * it; the golden vectors under tests/golden pin it to the reference's own
 * unit tests.
 *
 * Conventions.  Per-cell kernels (ora_*_code_*) keep the reference's Fortran
 * calling convention: 1-based dofmaps and column-major arrays.  Whole-mesh
 * routines (ora_helm_*, ora_mg_*, ora_*_solve_*) use 0-based indices and the
 * reference's column-contiguous field layout: the dof of level k in column c
 * is c*nlayers + k.
 */
#ifndef LFG_ORACLE_H
#define LFG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------- per-cell kernels ----------------------------- */
#define ORA_DECL_LMA(T, SFX)                                                            \
  void ora_matrix_vector_code_##SFX(int cell, int nlayers, T* lhs, const T* x,          \
                                    int ncell_3d, const T* matrix, int ndf1, int undf1, \
                                    const int* map1, int ndf2, int undf2, const int* map2); \
  void ora_dg_matrix_vector_code_##SFX(int cell, int nlayers, T* lhs, const T* x,       \
                                       int ncell_3d, const T* matrix, int ndf1,         \
                                       int undf1, const int* map1, int ndf2, int undf2, \
                                       const int* map2);                                \
  void ora_transpose_matrix_vector_code_##SFX(int cell, int nlayers, T* lhs, const T* x,\
                                              int ncell_3d, const T* matrix, int ndf1,  \
                                              int undf1, const int* map1, int ndf2,     \
                                              int undf2, const int* map2);              \
  void ora_mm_diagonal_code_##SFX(int cell, int nlayers, T* mm_diag, int ncell_3d,      \
                                  const T* mass_matrix, int ndf, int undf, const int* map); \
  void ora_columnwise_op_app_code_##SFX(int cell, int ncell_2d, T* lhs, const T* x,     \
                                        const T* columnwise_matrix, int nrow, int ncol, \
                                        int bandwidth, int alpha, int beta, int gamma_m,\
                                        int gamma_p, int ndf1, int undf1,               \
                                        const int* map1, const int* ind_to, int ndf2,   \
                                        int undf2, const int* map2, const int* ind_from); \
  void ora_columnwise_op_appinv_code_##SFX(int cell, int ncell_2d, T* lhs, const T* x,  \
                                           const T* columnwise_matrix, int nrow,        \
                                           int bandwidth, int alpha, int beta,          \
                                           int gamma_m, int gamma_p, int ndf, int undf, \
                                           const int* map, const int* ind, T* c_prime,  \
                                           T* d_prime);                                 \
  void ora_columnwise_op_asm_code_##SFX(int cell, int nlayers, int ncell_2d, int ncell_3d,\
      const T* local_stencil, T* columnwise_matrix, int nrow, int ncol, int bandwidth,  \
      int alpha, int beta, int gamma_m, int gamma_p, int ndf_to, const int* cbm_to,     \
      int ndf_from, const int* cbm_from);                                               \
  void ora_columnwise_op_mul_code_##SFX(int cell, int ncell_2d, const T* A, int nrow_A,  \
      int ncol_A, int bw_A, int alpha_A, int beta_A, int gm_A, int gp_A, const T* B,    \
      int nrow_B, int ncol_B, int bw_B, int alpha_B, int beta_B, int gm_B, int gp_B,    \
      T* C, int nrow_C, int ncol_C, int bw_C, int alpha_C, int beta_C, int gm_C,        \
      int gp_C);                                                                        \
  void ora_columnwise_op_scaledadd_code_##SFX(int cell, int ncell_2d, const T* A,        \
      int nrow_A, int ncol_A, int bw_A, int alpha_A, int beta_A, int gm_A, int gp_A,    \
      const T* B, int nrow_B, int ncol_B, int bw_B, int alpha_B, int beta_B, int gm_B,  \
      int gp_B, T* C, int nrow_C, int ncol_C, int bw_C, int alpha_C, int beta_C,        \
      int gm_C, int gp_C, T alpha, T beta);                                             \
  void ora_columnwise_op_asm_diag_hmht_code_##SFX(int cell, int nlayers, int ncell_2d,   \
      int ncell_3d, const T* dh, const T* m2h, T* columnwise_matrix, int nrow,          \
      int bandwidth, int alpha, int beta, int gamma_m, int gamma_p, int ndf_w3,         \
      const int* cbm, int ndf_w2h);                                                     \
  void ora_columnwise_op_asm_m2v_lumped_inv_code_##SFX(int cell, int nlayers,            \
      int ncell_2d, int ncell_3d, const T* local_stencil, T* columnwise_matrix,         \
      int nrow, int bandwidth, int ndf, const int* cbm);                                \
  void ora_tri_solve_code_##SFX(int nlayers, T* y, const T* x, const T* tri_0,          \
                                const T* tri_plus, const T* tri_minus, int ndf,         \
                                int undf, const int* map, T* x_new, T* tri_plus_new);   \
  void ora_restrict_scalar_unweighted_code_##SFX(int nlayers, const int* cell_map,      \
      int nx, int ny, int ncell_fine, T* coarse, const T* fine, int undf_coarse,        \
      const int* map_coarse, int ndf, int undf_fine, const int* map_fine, T* work);     \
  void ora_restrict_scalar_weighted_code_##SFX(int nlayers, const int* cell_map,        \
      int nx, int ny, int ncell_fine, T* coarse, const T* fine, const T* weights,       \
      int undf_coarse, const int* map_coarse, int ndf, int undf_fine,                   \
      const int* map_fine, T* work);                                                    \
  void ora_restrict_mass_w3_code_##SFX(int nlayers, const int* cell_map, int nx,        \
      int ny, int ncell_fine, T* coarse, const T* fine, int undf_coarse,                \
      const int* map_coarse, int ndf, int undf_fine, const int* map_fine, T* work);     \
  void ora_prolong_scalar_unweighted_code_##SFX(int nlayers, const int* cell_map,       \
      int nx, int ny, int ncell_fine, T* fine, const T* coarse, int ndf, int undf_fine, \
      const int* map_fine, int undf_coarse, const int* map_coarse);                     \
  void ora_prolong_scalar_weighted_code_##SFX(int nlayers, const int* cell_map,         \
      int nx, int ny, int ncell_fine, T* fine, const T* coarse, const T* weights,       \
      int ndf, int undf_fine, const int* map_fine, int undf_coarse,                     \
      const int* map_coarse);
ORA_DECL_LMA(double, r_double)
ORA_DECL_LMA(float, r_single)

void ora_operator_tri_solve_code(int cell, int nlayers, double* y, const double* x,
                                 int ncell, const double* matrix, int ndf, int undf,
                                 const int* map, double* work /* 5*(nlayers+1) */);
void ora_restrict_w0_code(int nlayers, const int* cell_map, int nx, int ny, int ncell_fine,
                          double* coarse, const double* fine, int undf_coarse,
                          const int* map_coarse, int ndf, int undf_fine, const int* map_fine);
void ora_prolong_w0_code(int nlayers, const int* cell_map, int nx, int ny, int ncell_fine,
                         double* fine, const double* coarse, int ndf, int undf_fine,
                         const int* map_fine, int undf_coarse, const int* map_coarse);
/* OpenMP threads of the whole-mesh routines: sets n (> 0) and returns the
 * number in use (1 without OpenMP). */
int ora_threads(int n);

/* W2 intergrid transfers (components/science/source/kernel/inter_mesh/),
 * per coarse cell, 1-based maps; work holds nlayers+1 values. */
void ora_restrict_w2_code_r_double(int nlayers, const int* cell_map, int nx, int ny,
                                   int ncell_fine, double* coarse, const double* fine,
                                   const int* sel_ew, const int* sel_ns, const int* map_coarse,
                                   int ndf, const int* map_fine, const int* map_w3_2d,
                                   int with_b, double* work);
void ora_restrict_w2_code_r_single(int nlayers, const int* cell_map, int nx, int ny,
                                   int ncell_fine, float* coarse, const float* fine,
                                   const int* sel_ew, const int* sel_ns, const int* map_coarse,
                                   int ndf, const int* map_fine, const int* map_w3_2d,
                                   int with_b, float* work);
void ora_restrict_w2v_code_r_double(int nlayers, const int* cell_map, int nx, int ny,
                                    int ncell_fine, double* coarse, const double* fine,
                                    const int* map_coarse, int ndf, const int* map_fine,
                                    double* work);
void ora_restrict_w2v_code_r_single(int nlayers, const int* cell_map, int nx, int ny,
                                    int ncell_fine, float* coarse, const float* fine,
                                    const int* map_coarse, int ndf, const int* map_fine,
                                    float* work);
void ora_weights_prolong_w2_code(int nlayers, const int* cell_map, int nx, int ny,
                                 int ncell_fine, double* w, int ndf, const int* map_fine);
void ora_prolong_w2_code(int nlayers, const int* cell_map, int nx, int ny, int ncell_fine,
                         double* fine, const double* coarse, const double* w, int ndf,
                         const int* map_fine, const int* map_coarse);

void ora_cma_params(int nlayers, int nint_to, int nface_to, int nint_from, int nface_from,
                    const int* offsets_to, const int* offsets_from, int* out7,
                    int* indirection_to, int* indirection_from);

/* --------------------------- whole-mesh routines ---------------------------- */
/* Status codes shared with the product's C-ABI. */
enum { ORA_OK = 0, ORA_NOT_CONVERGED = 1, ORA_NAN = 2 };

/* W3 Helmholtz operator A = T' - H_off on an extruded cubed sphere:
 *   cm : columnwise_matrix(3, nl, ncol) in Fortran order, rows = levels,
 *        bands (sub, diag, super); the diagonal already holds the sum of
 *        the four face couplings, so T' is also the column-smoother matrix;
 *   hf : hface(4, nl, ncol), coupling of cell (c,k) to its W,S,E,N neighbour;
 *   (A x)(c,k) = sum_j cm(j,k,c) x(c,k-2+j) - sum_f hf(f,k,c) x(links[c][f],k). */
typedef struct { int ncol, nl; const double* cm; const double* hf; const int* links; } ora_helm_d;
typedef struct { int ncol, nl; const float* cm; const float* hf; const int* links; } ora_helm_f;

#define ORA_MAX_LEVELS 8
typedef struct {
  int nlevels, n_pre, n_post, n_coarse;
  double omega;
  ora_helm_d op[ORA_MAX_LEVELS];
  const int* child[ORA_MAX_LEVELS]; /* child[l]: (ncol_{l+1}, 2(y), 2(x)) cells of level l */
  double* work;                     /* internal, sized by ora_mg_work_size */
} ora_mg_d;
typedef struct {
  int nlevels, n_pre, n_post, n_coarse;
  double omega;
  ora_helm_f op[ORA_MAX_LEVELS];
  const int* child[ORA_MAX_LEVELS];
  float* work;
} ora_mg_f;

#define ORA_DECL_REAL(T, S)                                                             \
  void ora_helm_apply_##S(const ora_helm_##S* op, const T* x, T* y);                    \
  void ora_helm_residual_##S(const ora_helm_##S* op, const T* x, const T* b, T* r);     \
  void ora_helm_smooth_##S(const ora_helm_##S* op, double omega, const T* x_in,         \
                           const T* b, T* x_out, T* work /* n + 2*nl */);               \
  void ora_restrict_sum_##S(int ncoarse, int nl, const int* child, const T* fine,       \
                            T* coarse);                                                 \
  void ora_prolong_add_##S(int ncoarse, int nl, const int* child, const T* coarse,      \
                           T* fine);                                                    \
  long ora_mg_work_size_##S(const ora_mg_##S* mg);                                      \
  void ora_mg_apply_##S(ora_mg_##S* mg, const T* b, T* x);                              \
  double ora_dot_##S(long n, const T* x, const T* y);                                   \
  double ora_norm_##S(long n, const T* x);
ORA_DECL_REAL(double, d)
ORA_DECL_REAL(float, f)

/* Galerkin coarse operator R A P with R = restrict_mass_w3 (sum over the four
 * children) and P = prolong_scalar_unweighted (injection).  Outputs cm_c
 * (3*nl*ncoarse) and hf_c (4*nl*ncoarse) in the same layouts. */
void ora_galerkin_coarsen(const ora_helm_d* fine, int ncoarse, const int* child,
                          const int* links_coarse, double* cm_c, double* hf_c);

/* Krylov solvers restated from components/science/source/solver/
 * sci_iterative_solver_mod.f90.  apply(ctx, x, y) computes y = Op(x); the
 * preconditioner's apply(ctx, x, y) computes y = P^{-1} x.  Scalars are
 * computed in double and cast to the vector kind for the updates, as in the
 * reference's r_solver_field_vector_type. */
typedef void (*ora_apply_d)(void* ctx, const double* x, double* y);
typedef void (*ora_apply_f)(void* ctx, const float* x, float* y);

typedef struct {
  int iterations;    /* inner steps performed (CG/Jacobi iterations, GCR directions) */
  double final_err;  /* last monitored relative residual (NaN if unmonitored) */
} ora_solve_info;

#define ORA_DECL_SOLVERS(T, S)                                                          \
  int ora_cg_solve_##S(long n, ora_apply_##S linop, void* lctx, ora_apply_##S prec,     \
                       void* pctx, double r_tol, double a_tol, int max_iter,            \
                       int monitor, T* x, const T* b, T* work /* 3n */,                 \
                       ora_solve_info* info);                                           \
  int ora_gcr_solve_##S(long n, ora_apply_##S linop, void* lctx, ora_apply_##S prec,    \
                        void* pctx, int gcrk, double r_tol, double a_tol, int max_iter, \
                        int monitor, T* x, const T* b, T* work /* (2 gcrk + 3) n */,    \
                        ora_solve_info* info);                                          \
  int ora_jacobi_solve_##S(long n, ora_apply_##S linop, void* lctx, ora_apply_##S prec, \
                           void* pctx, double r_tol, double a_tol, int max_iter,        \
                           int monitor, double rho_relax, T* x, const T* b,             \
                           T* work /* 2n */, ora_solve_info* info);                     \
  int ora_chebyshev_solve_##S(long n, ora_apply_##S linop, void* lctx,                  \
                              ora_apply_##S prec, void* pctx, double lmin, double lmax, \
                              int max_iter, int monitor, T* x, const T* b,              \
                              T* work /* 4n */, ora_solve_info* info);                  \
  int ora_precondition_only_solve_##S(long n, ora_apply_##S linop, void* lctx,          \
                                      ora_apply_##S prec, void* pctx, int monitor, T* x,\
                                      const T* b, T* work /* 2n */,                     \
                                      ora_solve_info* info);                            \
  int ora_bicgstab_solve_##S(long n, ora_apply_##S linop, void* lctx, ora_apply_##S prec,\
                             void* pctx, double r_tol, double a_tol, int max_iter,      \
                             int monitor, T* x, const T* b, T* work /* 8n */,           \
                             ora_solve_info* info);                                     \
  int ora_gmres_solve_##S(long n, ora_apply_##S linop, void* lctx, ora_apply_##S prec,   \
                          void* pctx, int k, double r_tol, double a_tol, int max_iter,  \
                          int monitor, T* x, const T* b, T* work /* (4 + k) n */,       \
                          ora_solve_info* info);                                        \
  int ora_fgmres_solve_##S(long n, ora_apply_##S linop, void* lctx, ora_apply_##S prec,  \
                           void* pctx, int k, double r_tol, double a_tol, int max_iter, \
                           int monitor, T* x, const T* b, T* work /* (5 + 2k) n */,     \
                           ora_solve_info* info);                                       \
  int ora_block_gcr_solve_##S(long n, ora_apply_##S linop, void* lctx, ora_apply_##S prec,\
                              void* pctx, int k, double r_tol, double a_tol, int max_iter,\
                              int monitor, int nf, const int* field_of, T* x, const T* b, \
                              T* work /* (2 + 2k) n */, ora_solve_info* info);            \
  void ora_cma_appinv_mesh_##S(int ncol, int nrow, const T* cm, const T* x, T* lhs);   \
  void ora_cma_app_mesh_##S(int ncol, int nrow, const T* cm, const T* x, T* lhs);      \
  void ora_helm_apply_cb_##S(void* op, const T* x, T* y);                               \
  void ora_mg_apply_cb_##S(void* mg, const T* x, T* y);
ORA_DECL_SOLVERS(double, d)
ORA_DECL_SOLVERS(float, f)

/* Diagonal (Jacobi) preconditioner y = x / diag
 * (sci_diagonal_preconditioner_alg_mod.x90:76-106, X_divideby_Y). */
typedef struct { long n; const double* diag; } ora_diag_prec;
void ora_diag_prec_apply(void* ctx, const double* x, double* y);
/* Null preconditioner y = x (sci_null_preconditioner_alg_mod.x90:73-95). */
void ora_null_prec_apply(void* ctx, const double* x, double* y);
typedef struct { long n; } ora_null_ctx;

/* LMA operator y = A x (apply_mass_matrix_operator: setval_c(y,0) then the
 * matrix_vector kernel over every cell in order,
 * sci_mass_matrix_operator_alg_mod.x90:72-119). */
typedef struct {
  int ncell, nlayers, ndf, undf;
  const double* matrix;  /* local_stencil(ncell*nlayers, ndf, ndf) */
  const int* map;        /* map(ndf, ncell), 1-based */
} ora_lma;
void ora_lma_apply_cb(void* op, const double* x, double* y);
void ora_lma_apply_transpose(const ora_lma* op, const double* x, double* y);
void ora_lma_diagonal(const ora_lma* op, double* diag);

/* Multigrid V-cycle over W2 LMA operators (project-defined set-up of the
 * reference's abstract_hierarchical_preconditioner_type,
 * components/science/source/solver/sci_hierarchical_preconditioner_mod.f90:22-38):
 * flat W2 fields in the reference's dof order, level 0 finest.  Each level
 * smooths with weighted Jacobi, x = x + omega (b - A x) / diag with diag
 * the mm_diagonal of its operator (entries no cell reaches count as 1);
 * the residual goes down with restrict_w2, the coarse correction comes up
 * with prolong_w2 (weights_prolong_w2 weights) and is added; n_coarse sweeps
 * from zero on the coarsest level.  cell_map[l] holds, for each cell of
 * level l+1, its 2x2 cells of level l as Fortran cell_map(2, 2), 1-based;
 * sel_ew / sel_ns[l] are the face selectors of the cells of level l+1. */
#define ORA_W2MG_MAXLEV 8
typedef struct {
  int nlevels, n_pre, n_post, n_coarse;
  double omega;
  ora_lma op[ORA_W2MG_MAXLEV];
  int ncoarse[ORA_W2MG_MAXLEV];
  const int* cell_map[ORA_W2MG_MAXLEV];
  const int* sel_ew[ORA_W2MG_MAXLEV];
  const int* sel_ns[ORA_W2MG_MAXLEV];
  double* work;  /* ora_w2mg_work_size doubles, filled by ora_w2mg_setup */
} ora_w2mg;
long ora_w2mg_work_size(const ora_w2mg* mg);
void ora_w2mg_setup(ora_w2mg* mg);
void ora_w2mg_apply_cb(void* mg, const double* b, double* x);

/* Mixed-precision iterative refinement: FP64 outer residual and update,
 * FP32 inner GCR(k) preconditioned by an FP32 multigrid V-cycle with FP64
 * inner products.  Returns a status; x starts from zero. */
typedef struct {
  int outer_iterations, inner_iterations;
  double final_rel_residual;  /* ||b - A x|| / ||b|| in FP64 */
} ora_mixed_info;
int ora_mixed_gcr_mg_solve(const ora_helm_d* op64, ora_mg_f* mg32, const double* b,
                           double* x, double tol, int max_outer, int gcrk,
                           double inner_tol, int inner_max_iter, ora_mixed_info* info);

/* Mixed-precision refinement with an inner FP32 CG preconditioned by the
 * exact column solve T'^{-1}: x = 0; r = b - A x (FP64) until
 * ||r|| <= tol ||b|| or max_outer corrections; each correction e is
 * cg_solve (monitor on, a_tol 0) on A_32 e = float(r) to inner_tol. */
int ora_mixed_cg_col_solve(const ora_helm_d* op64, const ora_helm_f* op32, const double* b,
                           double* x, double tol, int max_outer, double inner_tol,
                           int max_inner, ora_mixed_info* info);

#ifdef __cplusplus
}
#endif
#endif

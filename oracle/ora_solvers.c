/*
 * Oracle: whole-mesh operators, multigrid and Krylov solvers.
 * TEST INFRASTRUCTURE ONLY (see lfg_oracle.h).
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "lfg_oracle.h"

#define ORA_MAX_NL 4096
/* Loops over more than ORA_OMP_MIN values run on OpenMP threads when the
 * library is built with -fopenmp; inner products sum ORA_DOT_CHUNKS partial
 * sums in a fixed order, so results do not depend on the thread count. */
#define ORA_OMP_MIN 32768
#define ORA_DOT_CHUNKS 256

#define REAL double
#define S d
#define APPINV ora_columnwise_op_appinv_code_r_double
#define APP ora_columnwise_op_app_code_r_double
#include "ora_real.inc"
#undef REAL
#undef S
#undef APPINV
#undef APP

#define REAL float
#define S f
#define APPINV ora_columnwise_op_appinv_code_r_single
#define APP ora_columnwise_op_app_code_r_single
#include "ora_real.inc"
#undef REAL
#undef S
#undef APPINV
#undef APP

/* Galerkin coarse operator R A P (project-defined multigrid set-up).
 * child is (ncoarse, 2(y), 2(x)) with y N->S, x W->E in each coarse cell's
 * local frame, which the children share.  Coarse bands are sums over the
 * children (y outer, x inner); the couplings between two children of the
 * same coarse cell leave the diagonal; a coarse face's coupling is the sum
 * of the two fine faces that make it up. */
void ora_galerkin_coarsen(const ora_helm_d* fine, int ncoarse, const int* child,
                          const int* links_coarse, double* cm_c, double* hf_c) {
  (void)links_coarse;
  const int nl = fine->nl;
  /* children on each side (y, x): W: x=0, S: y=1, E: x=1, N: y=0 */
  static const int side_q[4][2] = {{0, 2}, {2, 3}, {1, 3}, {0, 1}};
  for (int C = 0; C < ncoarse; ++C) {
    const int* ch = child + C * 4;
    for (int k = 0; k < nl; ++k) {
      for (int b = 0; b < 3; ++b) {
        double acc = 0.0;
        for (int q = 0; q < 4; ++q) acc = acc + fine->cm[((long)ch[q] * nl + k) * 3 + b];
        cm_c[((long)C * nl + k) * 3 + b] = acc;
      }
      double dg = cm_c[((long)C * nl + k) * 3 + 1];
      for (int q = 0; q < 4; ++q)
        for (int f = 0; f < 4; ++f) {
          int nb = fine->links[ch[q] * 4 + f];
          if (nb == ch[0] || nb == ch[1] || nb == ch[2] || nb == ch[3])
            dg = dg - fine->hf[((long)ch[q] * nl + k) * 4 + f];
        }
      cm_c[((long)C * nl + k) * 3 + 1] = dg;
      for (int f = 0; f < 4; ++f)
        hf_c[((long)C * nl + k) * 4 + f] = fine->hf[((long)ch[side_q[f][0]] * nl + k) * 4 + f] +
                                           fine->hf[((long)ch[side_q[f][1]] * nl + k) * 4 + f];
    }
  }
}

void ora_diag_prec_apply(void* ctx, const double* x, double* y) {
  const ora_diag_prec* p = (const ora_diag_prec*)ctx;
  for (long i = 0; i < p->n; ++i) y[i] = x[i] / p->diag[i];
}

void ora_null_prec_apply(void* ctx, const double* x, double* y) {
  const ora_null_ctx* p = (const ora_null_ctx*)ctx;
  memcpy(y, x, sizeof(double) * p->n);
}

void ora_lma_apply_cb(void* vop, const double* x, double* y) {
  const ora_lma* op = (const ora_lma*)vop;
  memset(y, 0, sizeof(double) * op->undf);
  for (int cell = 1; cell <= op->ncell; ++cell)
    ora_matrix_vector_code_r_double(cell, op->nlayers, y, x, op->ncell * op->nlayers,
                                    op->matrix, op->ndf, op->undf,
                                    op->map + (long)(cell - 1) * op->ndf, op->ndf, op->undf,
                                    op->map + (long)(cell - 1) * op->ndf);
}

/* y = A^T x over the mesh with the transpose_matrix_vector kernel, which
 * reads the matrix as (ncell_3d, ndf2, ndf1); for a square LMA that is the
 * transpose of the matrix_vector apply. */
void ora_lma_apply_transpose(const ora_lma* op, const double* x, double* y) {
  memset(y, 0, sizeof(double) * op->undf);
  for (int cell = 1; cell <= op->ncell; ++cell)
    ora_transpose_matrix_vector_code_r_double(cell, op->nlayers, y, x,
                                              op->ncell * op->nlayers, op->matrix, op->ndf,
                                              op->undf, op->map + (long)(cell - 1) * op->ndf,
                                              op->ndf, op->undf,
                                              op->map + (long)(cell - 1) * op->ndf);
}

void ora_lma_diagonal(const ora_lma* op, double* diag) {
  memset(diag, 0, sizeof(double) * op->undf);
  for (int cell = 1; cell <= op->ncell; ++cell)
    ora_mm_diagonal_code_r_double(cell, op->nlayers, diag, op->ncell * op->nlayers,
                                  op->matrix, op->ndf, op->undf,
                                  op->map + (long)(cell - 1) * op->ndf);
}

/* Mixed-precision iterative refinement (project-defined).
 *   x = 0, r = b
 *   repeat: e = GCR_32(A_32, MG_32; r as float) from zero to inner_tol,
 *           x += e (FP64), r = b - A_64 x (FP64), stop when ||r||/||b|| <= tol. */
int ora_mixed_gcr_mg_solve(const ora_helm_d* op64, ora_mg_f* mg32, const double* b,
                           double* x, double tol, int max_outer, int gcrk, double inner_tol,
                           int inner_max_iter, ora_mixed_info* info) {
  const long n = (long)op64->ncol * op64->nl;
  double* r = (double*)malloc(sizeof(double) * n);
  float* r32 = (float*)malloc(sizeof(float) * n);
  float* e32 = (float*)malloc(sizeof(float) * n);
  float* work = (float*)malloc(sizeof(float) * (2 * gcrk + 3) * n);
  ora_helm_f* op32 = &mg32->op[0];
  int status = ORA_NOT_CONVERGED;
  memset(x, 0, sizeof(double) * n);
  memcpy(r, b, sizeof(double) * n);
  const double nb = ora_norm_d(n, b);
  info->outer_iterations = 0;
  info->inner_iterations = 0;
  info->final_rel_residual = nb > 0 ? 1.0 : 0.0;
  if (nb < DBL_EPSILON) { status = ORA_OK; goto done; }
  for (int o = 1; o <= max_outer; ++o) {
    for (long i = 0; i < n; ++i) r32[i] = (float)r[i];
    memset(e32, 0, sizeof(float) * n);
    ora_solve_info si;
    int st = ora_gcr_solve_f(n, ora_helm_apply_cb_f, op32, ora_mg_apply_cb_f, mg32, gcrk,
                             inner_tol, 0.0, inner_max_iter, 1, e32, r32, work, &si);
    info->inner_iterations += si.iterations;
    info->outer_iterations = o;
    if (st == ORA_NAN) { status = ORA_NAN; goto done; }
    for (long i = 0; i < n; ++i) x[i] = x[i] + (double)e32[i];
    ora_helm_residual_d(op64, x, b, r);
    info->final_rel_residual = ora_norm_d(n, r) / nb;
    if (isnan(info->final_rel_residual)) { status = ORA_NAN; goto done; }
    if (info->final_rel_residual <= tol) { status = ORA_OK; goto done; }
  }
done:
  free(r); free(r32); free(e32); free(work);
  return status;
}

/* Column preconditioner z = T'^{-1} r: one block-Jacobi sweep from zero
 * with omega = 1 (columnwise_op_appinv on every column). */
typedef struct {
  const ora_helm_f* op;
  float* work;
} ora_colprec_f;
static void ora_colprec_apply_f(void* ctx, const float* r, float* z) {
  const ora_colprec_f* c = (const ora_colprec_f*)ctx;
  ora_helm_smooth_f(c->op, 1.0, NULL, r, z, c->work);
}

/* Mixed-precision refinement with an inner column-preconditioned CG
 * (project-defined; the batched solver's per-problem algorithm):
 *   x = 0; loop: r = b - A_64 x (FP64); stop when ||r|| <= tol ||b|| or
 *   after max_outer corrections; e = cg_solve_32(A_32, T'^{-1}; float(r))
 *   from zero to inner_tol relative (max_inner iterations); x += e. */
int ora_mixed_cg_col_solve(const ora_helm_d* op64, const ora_helm_f* op32, const double* b,
                           double* x, double tol, int max_outer, double inner_tol,
                           int max_inner, ora_mixed_info* info) {
  const long n = (long)op64->ncol * op64->nl;
  double* r = (double*)malloc(sizeof(double) * n);
  float* r32 = (float*)malloc(sizeof(float) * n);
  float* e32 = (float*)malloc(sizeof(float) * n);
  float* work = (float*)malloc(sizeof(float) * 3 * n);
  ora_colprec_f cp = {op32, (float*)malloc(sizeof(float) * (n + 2 * op32->nl))};
  int status = ORA_NOT_CONVERGED;
  double bnorm = 0.0;
  memset(x, 0, sizeof(double) * n);
  info->outer_iterations = 0;
  info->inner_iterations = 0;
  info->final_rel_residual = 0.0;
  for (int o = 0;; ++o) {
    ora_helm_residual_d(op64, x, b, r);
    const double rn = ora_norm_d(n, r);
    if (o == 0) {
      bnorm = rn;
      if (rn < DBL_EPSILON) { status = ORA_OK; break; }
    }
    info->final_rel_residual = rn / bnorm;
    if (isnan(info->final_rel_residual)) { status = ORA_NAN; break; }
    if (info->final_rel_residual <= tol) { status = ORA_OK; break; }
    if (o >= max_outer) { status = ORA_NOT_CONVERGED; break; }
    for (long i = 0; i < n; ++i) r32[i] = (float)r[i];
    memset(e32, 0, sizeof(float) * n);
    ora_solve_info si;
    ora_cg_solve_f(n, ora_helm_apply_cb_f, (void*)op32, ora_colprec_apply_f, &cp, inner_tol,
                   0.0, max_inner, 1, e32, r32, work, &si);
    info->inner_iterations += si.iterations;
    for (long i = 0; i < n; ++i) x[i] = x[i] + (double)e32[i];
    info->outer_iterations = o + 1;
  }
  free(r); free(r32); free(e32); free(work); free(cp.work);
  return status;
}

/* Sets the number of OpenMP threads (n > 0) and returns the number in use;
 * 1 when the library was built without OpenMP. */
int ora_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

/* ------------------------------------------------ W2 multigrid V-cycle
 * Work per level l (undf_l doubles each): diag, r, y, bc, xc, t, w. */
enum { W2_DIAG, W2_R, W2_Y, W2_BC, W2_XC, W2_T, W2_W, W2_NARR };

static double* w2_arr(const ora_w2mg* mg, int l, int which) {
  long off = 0;
  for (int i = 0; i < l; ++i) off += (long)W2_NARR * mg->op[i].undf;
  return mg->work + off + (long)which * mg->op[l].undf;
}

long ora_w2mg_work_size(const ora_w2mg* mg) {
  long n = 0;
  for (int l = 0; l < mg->nlevels; ++l) n += (long)W2_NARR * mg->op[l].undf;
  return n;
}

void ora_w2mg_setup(ora_w2mg* mg) {
  for (int l = 0; l < mg->nlevels; ++l) {
    double* d = w2_arr(mg, l, W2_DIAG);
    ora_lma_diagonal(&mg->op[l], d);
    for (int i = 0; i < mg->op[l].undf; ++i)
      if (d[i] == 0.0) d[i] = 1.0;
    if (l + 1 < mg->nlevels) {
      double* w = w2_arr(mg, l, W2_W);
      memset(w, 0, sizeof(double) * mg->op[l].undf);
      for (int C = 0; C < mg->ncoarse[l]; ++C)
        ora_weights_prolong_w2_code(mg->op[l].nlayers, mg->cell_map[l] + 4 * C, 2, 2, 4, w, 6,
                                    mg->op[l].map);
    }
  }
}

/* x = x + omega (b - A x) / diag */
static void w2_sweep(ora_w2mg* mg, int l, const double* b, double* x) {
  const long n = mg->op[l].undf;
  double *r = w2_arr(mg, l, W2_R), *y = w2_arr(mg, l, W2_Y);
  const double* d = w2_arr(mg, l, W2_DIAG);
  ora_lma_apply_cb(&mg->op[l], x, y);
  for (long i = 0; i < n; ++i) r[i] = b[i] + (-1.0) * y[i];
  for (long i = 0; i < n; ++i) r[i] = r[i] / d[i];
  for (long i = 0; i < n; ++i) x[i] = x[i] + mg->omega * r[i];
}

static void w2_vcycle(ora_w2mg* mg, int l, const double* b, double* x) {
  const long n = mg->op[l].undf;
  const int nl = mg->op[l].nlayers;
  memset(x, 0, sizeof(double) * n);
  if (l == mg->nlevels - 1) {
    for (int i = 0; i < mg->n_coarse; ++i) w2_sweep(mg, l, b, x);
    return;
  }
  for (int i = 0; i < mg->n_pre; ++i) w2_sweep(mg, l, b, x);
  double *r = w2_arr(mg, l, W2_R), *y = w2_arr(mg, l, W2_Y);
  ora_lma_apply_cb(&mg->op[l], x, y);
  for (long i = 0; i < n; ++i) r[i] = b[i] + (-1.0) * y[i];
  double* bc = w2_arr(mg, l + 1, W2_BC);
  double* xc = w2_arr(mg, l + 1, W2_XC);
  double work[ORA_MAX_NL + 1];
  for (int C = 0; C < mg->ncoarse[l]; ++C) {
    const int sel_idx[1] = {C + 1};
    ora_restrict_w2_code_r_double(nl, mg->cell_map[l] + 4 * C, 2, 2, 4, bc, r, mg->sel_ew[l],
                                  mg->sel_ns[l], mg->op[l + 1].map + 6 * C, 6, mg->op[l].map,
                                  sel_idx, 1, work);
  }
  w2_vcycle(mg, l + 1, bc, xc);
  double* t = w2_arr(mg, l, W2_T);
  const double* w = w2_arr(mg, l, W2_W);
  for (int C = 0; C < mg->ncoarse[l]; ++C)
    ora_prolong_w2_code(nl, mg->cell_map[l] + 4 * C, 2, 2, 4, t, xc, w, 6, mg->op[l].map,
                        mg->op[l + 1].map + 6 * C);
  for (long i = 0; i < n; ++i) x[i] = x[i] + 1.0 * t[i];
  for (int i = 0; i < mg->n_post; ++i) w2_sweep(mg, l, b, x);
}

void ora_w2mg_apply_cb(void* vmg, const double* b, double* x) {
  w2_vcycle((ora_w2mg*)vmg, 0, b, x);
}

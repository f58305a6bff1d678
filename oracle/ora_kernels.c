/*
 * Oracle: CPU restatement of the reference's per-column kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: it
 * is compiled into oracle/liblfg_oracle.so, which only the tests, the smoke
 * check and the CPU-baseline leg of the benchmark load.  No product code path
 * calls it.
 *
 * Every routine keeps the reference's calling convention: Fortran 1-based
 * dofmaps, column-major arrays, one call per horizontal cell (the PSy layer
 * loops over cells).  Each one cites the reference routine it restates.
 * Array macros: A2(a,i,j,n1) is a(i,j) of a(n1,*); A3(a,i,j,k,n1,n2) is
 * a(i,j,k) of a(n1,n2,*); V(a,i) is a(i) -- all 1-based.
 */
#include <math.h>
#include <stddef.h>
#include "lfg_oracle.h"

#define V(a, i) (a)[(size_t)(i) - 1]
#define A2(a, i, j, n1) (a)[((size_t)(i) - 1) + (size_t)(n1) * ((size_t)(j) - 1)]
#define A3(a, i, j, k, n1, n2) \
  (a)[((size_t)(i) - 1) + (size_t)(n1) * (((size_t)(j) - 1) + (size_t)(n2) * ((size_t)(k) - 1))]

/* ------------------------------------------------------------------------
 * LMA kernels.
 * ---------------------------------------------------------------------- */

/* components/science/source/kernel/algebra/matrix_vector_kernel_mod.F90:68-140
 * lhs(map1(df)+k) += matrix(ik+k, df, df2) * x(map2(df2)+k), df2 outer. */
#define DEF_MATRIX_VECTOR(T, SFX)                                                     \
  void ora_matrix_vector_code_##SFX(int cell, int nlayers, T* lhs, const T* x,        \
                                    int ncell_3d, const T* matrix, int ndf1,          \
                                    int undf1, const int* map1, int ndf2, int undf2,  \
                                    const int* map2) {                                \
    (void)undf1; (void)undf2;                                                         \
    int ik = (cell - 1) * nlayers + 1;                                                \
    for (int df2 = 1; df2 <= ndf2; ++df2) {                                           \
      int i2 = V(map2, df2);                                                          \
      for (int df = 1; df <= ndf1; ++df) {                                            \
        int i1 = V(map1, df);                                                         \
        for (int k = 0; k < nlayers; ++k)                                             \
          V(lhs, i1 + k) = V(lhs, i1 + k) +                                           \
                           A3(matrix, ik + k, df, df2, ncell_3d, ndf1) * V(x, i2 + k); \
      }                                                                               \
    }                                                                                 \
  }
DEF_MATRIX_VECTOR(double, r_double)
DEF_MATRIX_VECTOR(float, r_single)

/* components/science/source/kernel/algebra/dg_matrix_vector_kernel_mod.F90:68-154
 * As matrix_vector but lhs is zeroed on the cell's dofs first. */
#define DEF_DG_MATRIX_VECTOR(T, SFX)                                                  \
  void ora_dg_matrix_vector_code_##SFX(int cell, int nlayers, T* lhs, const T* x,     \
                                       int ncell_3d, const T* matrix, int ndf1,       \
                                       int undf1, const int* map1, int ndf2,          \
                                       int undf2, const int* map2) {                  \
    for (int df1 = 1; df1 <= ndf1; ++df1) {                                           \
      int i1 = V(map1, df1);                                                          \
      for (int k = 0; k < nlayers; ++k) V(lhs, i1 + k) = (T)0;                        \
    }                                                                                 \
    ora_matrix_vector_code_##SFX(cell, nlayers, lhs, x, ncell_3d, matrix, ndf1,       \
                                 undf1, map1, ndf2, undf2, map2);                     \
  }
DEF_DG_MATRIX_VECTOR(double, r_double)
DEF_DG_MATRIX_VECTOR(float, r_single)

/* components/science/source/kernel/algebra/transpose_matrix_vector_kernel_mod.F90:66-144
 * matrix is (ncell_3d, ndf2, ndf1); lhs(map1(df)+k) += sum_df2 matrix(ik,df2,df) x_e(df2),
 * computed per level as lhs_e = matmul(transpose(matrix(ik,:,:)), x_e). */
#define DEF_TRANSPOSE_MATRIX_VECTOR(T, SFX)                                           \
  void ora_transpose_matrix_vector_code_##SFX(int cell, int nlayers, T* lhs,          \
                                              const T* x, int ncell_3d,               \
                                              const T* matrix, int ndf1, int undf1,   \
                                              const int* map1, int ndf2, int undf2,   \
                                              const int* map2) {                      \
    (void)undf1; (void)undf2;                                                         \
    for (int k = 0; k < nlayers; ++k) {                                               \
      int ik = (cell - 1) * nlayers + k + 1;                                          \
      for (int df = 1; df <= ndf1; ++df) {                                            \
        T acc = (T)0;                                                                 \
        for (int df2 = 1; df2 <= ndf2; ++df2)                                         \
          acc += A3(matrix, ik, df2, df, ncell_3d, ndf2) * V(x, V(map2, df2) + k);    \
        V(lhs, V(map1, df) + k) = V(lhs, V(map1, df) + k) + acc;                      \
      }                                                                               \
    }                                                                                 \
  }
DEF_TRANSPOSE_MATRIX_VECTOR(double, r_double)
DEF_TRANSPOSE_MATRIX_VECTOR(float, r_single)

/* components/science/source/kernel/algebra/sci_mm_diagonal_kernel_mod.F90:68-127 */
#define DEF_MM_DIAGONAL(T, SFX)                                                       \
  void ora_mm_diagonal_code_##SFX(int cell, int nlayers, T* mm_diag, int ncell_3d,    \
                                  const T* mass_matrix, int ndf, int undf,            \
                                  const int* map) {                                   \
    (void)undf;                                                                       \
    for (int k = 0; k < nlayers; ++k) {                                               \
      int ik = (cell - 1) * nlayers + k + 1;                                          \
      for (int df = 1; df <= ndf; ++df)                                               \
        V(mm_diag, V(map, df) + k) =                                                  \
            V(mm_diag, V(map, df) + k) + A3(mass_matrix, ik, df, df, ncell_3d, ndf);  \
    }                                                                                 \
  }
DEF_MM_DIAGONAL(double, r_double)
DEF_MM_DIAGONAL(float, r_single)

/* ------------------------------------------------------------------------
 * CMA kernels (r_solver: both kinds provided).
 * ---------------------------------------------------------------------- */

/* Fortran ceiling/floor of (num / den) computed in r_solver as the reference
 * does: ceiling((alpha*i-gamma_p)/(1.0_r_solver*beta), i_def). */
#define DEF_CMA_APP(T, SFX)                                                           \
  void ora_columnwise_op_app_code_##SFX(                                              \
      int cell, int ncell_2d, T* lhs, const T* x, const T* columnwise_matrix,         \
      int nrow, int ncol, int bandwidth, int alpha, int beta, int gamma_m,            \
      int gamma_p, int ndf1, int undf1, const int* map1,                              \
      const int* indirection_dofmap_to, int ndf2, int undf2, const int* map2,         \
      const int* indirection_dofmap_from) {                                           \
    (void)ncell_2d; (void)ndf1; (void)undf1; (void)ndf2; (void)undf2;                 \
    for (int i = 1; i <= nrow; ++i) {                                                 \
      int mu_i = V(map1, 1) + V(indirection_dofmap_to, i) - 1;                        \
      int j_minus = (int)ceil((T)(alpha * i - gamma_p) / ((T)1 * (T)beta));           \
      int j_plus = (int)floor((T)(alpha * i + gamma_m) / ((T)1 * (T)beta));           \
      int jlo = j_minus > 1 ? j_minus : 1;                                            \
      int jhi = j_plus < ncol ? j_plus : ncol;                                        \
      for (int j = jlo; j <= jhi; ++j) {                                              \
        int mu_j = V(map2, 1) + V(indirection_dofmap_from, j) - 1;                    \
        V(lhs, mu_i) = V(lhs, mu_i) +                                                 \
            A3(columnwise_matrix, j - j_minus + 1, i, cell, bandwidth, nrow) * V(x, mu_j); \
      }                                                                               \
    }                                                                                 \
  }
DEF_CMA_APP(double, r_double)
DEF_CMA_APP(float, r_single)

/* CMA assembly and algebra (components/science/source/kernel/
 * columnwise_operators/): the reference's per-cell loops with local_stencil
 * (ncell_3d, ndf_to, ndf_from) and columnwise_matrix (bandwidth, nrow,
 * ncell_2d) in Fortran order; j_minus / j_plus in the kind T as the
 * reference evaluates them in r_solver. */
#define ORA_JMINUS(T, a, i, gp, b) ((int)ceil((T)((a) * (i) - (gp)) / ((T)1 * (T)(b))))
#define ORA_JPLUS(T, a, i, gm, b) ((int)floor((T)((a) * (i) + (gm)) / ((T)1 * (T)(b))))

/* sci_columnwise_op_asm_kernel_mod.F90, columnwise_op_asm_kernel_code */
#define DEF_CMA_ASM(T, SFX)                                                           \
  void ora_columnwise_op_asm_code_##SFX(                                              \
      int cell, int nlayers, int ncell_2d, int ncell_3d, const T* local_stencil,      \
      T* columnwise_matrix, int nrow, int ncol, int bandwidth, int alpha, int beta,   \
      int gamma_m, int gamma_p, int ndf_to, const int* cbm_to, int ndf_from,          \
      const int* cbm_from) {                                                          \
    (void)ncell_2d; (void)ncol; (void)gamma_m;                                        \
    for (int i = 1; i <= nrow; ++i)                                                   \
      for (int b = 1; b <= bandwidth; ++b)                                            \
        A3(columnwise_matrix, b, i, cell, bandwidth, nrow) = (T)0;                    \
    for (int k = 1; k <= nlayers; ++k) {                                              \
      int ik = (cell - 1) * nlayers + k;                                              \
      for (int df1 = 1; df1 <= ndf_to; ++df1) {                                       \
        int i = A2(cbm_to, df1, k, ndf_to);                                           \
        int j_minus = ORA_JMINUS(T, alpha, i, gamma_p, beta);                         \
        for (int df2 = 1; df2 <= ndf_from; ++df2) {                                   \
          int j = A2(cbm_from, df2, k, ndf_from);                                     \
          A3(columnwise_matrix, j - j_minus + 1, i, cell, bandwidth, nrow) =          \
              A3(columnwise_matrix, j - j_minus + 1, i, cell, bandwidth, nrow) +      \
              A3(local_stencil, ik, df1, df2, ncell_3d, ndf_to);                      \
        }                                                                             \
      }                                                                               \
    }                                                                                 \
  }
DEF_CMA_ASM(double, r_double)
DEF_CMA_ASM(float, r_single)

/* sci_columnwise_op_mul_kernel_mod.F90, columnwise_op_mul_kernel_code: C += A B */
#define DEF_CMA_MUL(T, SFX)                                                           \
  void ora_columnwise_op_mul_code_##SFX(                                              \
      int cell, int ncell_2d, const T* A, int nrow_A, int ncol_A, int bw_A,           \
      int alpha_A, int beta_A, int gm_A, int gp_A, const T* B, int nrow_B,            \
      int ncol_B, int bw_B, int alpha_B, int beta_B, int gm_B, int gp_B, T* C,        \
      int nrow_C, int ncol_C, int bw_C, int alpha_C, int beta_C, int gm_C,            \
      int gp_C) {                                                                     \
    (void)ncell_2d; (void)ncol_B;                                                     \
    for (int i = 1; i <= nrow_C; ++i) {                                               \
      int jmA = ORA_JMINUS(T, alpha_A, i, gp_A, beta_A);                              \
      int jpA = ORA_JPLUS(T, alpha_A, i, gm_A, beta_A);                               \
      int jmC = ORA_JMINUS(T, alpha_C, i, gp_C, beta_C);                              \
      int jpC = ORA_JPLUS(T, alpha_C, i, gm_C, beta_C);                               \
      for (int j = (jmC > 1 ? jmC : 1); j <= (jpC < ncol_C ? jpC : ncol_C); ++j) {     \
        T e = (T)0;                                                                   \
        for (int l = (jmA > 1 ? jmA : 1); l <= (jpA < ncol_A ? jpA : ncol_A); ++l) {   \
          int jmB = ORA_JMINUS(T, alpha_B, l, gp_B, beta_B);                          \
          int jpB = ORA_JPLUS(T, alpha_B, l, gm_B, beta_B);                           \
          if (jmB <= j && j <= jpB)                                                   \
            e = e + A3(A, l - jmA + 1, i, cell, bw_A, nrow_A) *                       \
                        A3(B, j - jmB + 1, l, cell, bw_B, nrow_B);                    \
        }                                                                             \
        A3(C, j - jmC + 1, i, cell, bw_C, nrow_C) =                                   \
            A3(C, j - jmC + 1, i, cell, bw_C, nrow_C) + e;                            \
      }                                                                               \
    }                                                                                 \
  }
DEF_CMA_MUL(double, r_double)
DEF_CMA_MUL(float, r_single)

/* sci_columnwise_op_scaledadd_kernel_mod.F90, columnwise_op_scaledadd_kernel_code:
 * C = alpha A + beta B (B's loop is clipped to A's column count, as there). */
#define DEF_CMA_SCALEDADD(T, SFX)                                                     \
  void ora_columnwise_op_scaledadd_code_##SFX(                                        \
      int cell, int ncell_2d, const T* A, int nrow_A, int ncol_A, int bw_A,           \
      int alpha_A, int beta_A, int gm_A, int gp_A, const T* B, int nrow_B,            \
      int ncol_B, int bw_B, int alpha_B, int beta_B, int gm_B, int gp_B, T* C,        \
      int nrow_C, int ncol_C, int bw_C, int alpha_C, int beta_C, int gm_C,            \
      int gp_C, T alpha, T beta) {                                                    \
    (void)ncell_2d; (void)ncol_B; (void)ncol_C; (void)gm_C;                           \
    for (int i = 1; i <= nrow_C; ++i)                                                 \
      for (int b = 1; b <= bw_C; ++b) A3(C, b, i, cell, bw_C, nrow_C) = (T)0;         \
    for (int i = 1; i <= nrow_A; ++i) {                                               \
      int jmA = ORA_JMINUS(T, alpha_A, i, gp_A, beta_A);                              \
      int jpA = ORA_JPLUS(T, alpha_A, i, gm_A, beta_A);                               \
      int jmB = ORA_JMINUS(T, alpha_B, i, gp_B, beta_B);                              \
      int jpB = ORA_JPLUS(T, alpha_B, i, gm_B, beta_B);                               \
      int jmC = ORA_JMINUS(T, alpha_C, i, gp_C, beta_C);                              \
      for (int j = (jmA > 1 ? jmA : 1); j <= (jpA < ncol_A ? jpA : ncol_A); ++j)       \
        A3(C, j - jmC + 1, i, cell, bw_C, nrow_C) =                                   \
            A3(C, j - jmC + 1, i, cell, bw_C, nrow_C) +                               \
            alpha * A3(A, j - jmA + 1, i, cell, bw_A, nrow_A);                        \
      for (int j = (jmB > 1 ? jmB : 1); j <= (jpB < ncol_A ? jpB : ncol_A); ++j)       \
        A3(C, j - jmC + 1, i, cell, bw_C, nrow_C) =                                   \
            A3(C, j - jmC + 1, i, cell, bw_C, nrow_C) +                               \
            beta * A3(B, j - jmB + 1, i, cell, bw_B, nrow_B);                         \
    }                                                                                 \
  }
DEF_CMA_SCALEDADD(double, r_double)
DEF_CMA_SCALEDADD(float, r_single)

/* sci_columnwise_op_asm_diag_hmht_kernel_mod.F90,
 * columnwise_op_asm_diag_hmht_kernel_code */
#define DEF_CMA_HMHT(T, SFX)                                                          \
  void ora_columnwise_op_asm_diag_hmht_code_##SFX(                                    \
      int cell, int nlayers, int ncell_2d, int ncell_3d, const T* dh,                 \
      const T* m2h, T* columnwise_matrix, int nrow, int bandwidth, int alpha,         \
      int beta, int gamma_m, int gamma_p, int ndf_w3, const int* cbm,                 \
      int ndf_w2h) {                                                                  \
    (void)ncell_2d; (void)gamma_m;                                                    \
    for (int i = 1; i <= nrow; ++i)                                                   \
      for (int b = 1; b <= bandwidth; ++b)                                            \
        A3(columnwise_matrix, b, i, cell, bandwidth, nrow) = (T)0;                    \
    for (int k = 1; k <= nlayers; ++k) {                                              \
      int ik = (cell - 1) * nlayers + k;                                              \
      for (int df1 = 1; df1 <= ndf_w3; ++df1) {                                       \
        int i = A2(cbm, df1, k, ndf_w3);                                              \
        int j_minus = ORA_JMINUS(T, alpha, i, gamma_p, beta);                         \
        for (int df2 = 1; df2 <= ndf_w3; ++df2) {                                     \
          T tmp = (T)0;                                                               \
          for (int df3 = 1; df3 <= ndf_w2h; ++df3)                                    \
            tmp = tmp + A3(dh, ik, df1, df3, ncell_3d, ndf_w3) *                      \
                            A3(dh, ik, df2, df3, ncell_3d, ndf_w3) /                  \
                            A3(m2h, ik, df3, df3, ncell_3d, ndf_w2h);                 \
          int j = A2(cbm, df2, k, ndf_w3);                                            \
          A3(columnwise_matrix, j - j_minus + 1, i, cell, bandwidth, nrow) =          \
              A3(columnwise_matrix, j - j_minus + 1, i, cell, bandwidth, nrow) + tmp; \
        }                                                                             \
      }                                                                               \
    }                                                                                 \
  }
DEF_CMA_HMHT(double, r_double)
DEF_CMA_HMHT(float, r_single)

/* sci_columnwise_op_asm_m2v_lumped_inv_krnl_mod.F90,
 * columnwise_op_asm_m2v_lumped_inv_krnl_code */
#define DEF_CMA_M2V(T, SFX)                                                           \
  void ora_columnwise_op_asm_m2v_lumped_inv_code_##SFX(                               \
      int cell, int nlayers, int ncell_2d, int ncell_3d, const T* local_stencil,      \
      T* columnwise_matrix, int nrow, int bandwidth, int ndf, const int* cbm) {       \
    (void)ncell_2d;                                                                   \
    for (int i = 1; i <= nrow; ++i)                                                   \
      for (int b = 1; b <= bandwidth; ++b)                                            \
        A3(columnwise_matrix, b, i, cell, bandwidth, nrow) = (T)0;                    \
    for (int k = 1; k <= nlayers; ++k) {                                              \
      int ik = (cell - 1) * nlayers + k;                                              \
      for (int df1 = 1; df1 <= ndf; ++df1) {                                          \
        int i = A2(cbm, df1, k, ndf);                                                 \
        A3(columnwise_matrix, 1, i, cell, bandwidth, nrow) =                          \
            A3(columnwise_matrix, 1, i, cell, bandwidth, nrow) +                      \
            A3(local_stencil, ik, df1, df1, ncell_3d, ndf);                           \
      }                                                                               \
    }                                                                                 \
    for (int i = 1; i <= nrow; ++i)                                                   \
      for (int b = 1; b <= bandwidth; ++b)                                            \
        if (A3(columnwise_matrix, b, i, cell, bandwidth, nrow) != (T)0)               \
          A3(columnwise_matrix, b, i, cell, bandwidth, nrow) =                        \
              (T)1 / A3(columnwise_matrix, b, i, cell, bandwidth, nrow);              \
  }
DEF_CMA_M2V(double, r_double)
DEF_CMA_M2V(float, r_single)

/* components/science/source/kernel/columnwise_operators/sci_columnwise_op_appinv_kernel_mod.F90:77-145
 * Thomas algorithm; lhs is overwritten with the solution. */
#define DEF_CMA_APPINV(T, SFX)                                                        \
  void ora_columnwise_op_appinv_code_##SFX(                                           \
      int cell, int ncell_2d, T* lhs, const T* x, const T* columnwise_matrix,         \
      int nrow, int bandwidth, int alpha, int beta, int gamma_m, int gamma_p,         \
      int ndf, int undf, const int* map, const int* indirection_dofmap,               \
      T* c_prime, T* d_prime) {                                                       \
    (void)ncell_2d; (void)alpha; (void)beta; (void)gamma_m; (void)gamma_p;            \
    (void)ndf; (void)undf;                                                            \
    T inv_denom;                                                                      \
    for (int i = 1; i <= nrow; ++i) {                                                 \
      int mu_i = V(map, 1) + V(indirection_dofmap, i) - 1;                            \
      const T a1 = A3(columnwise_matrix, 1, i, cell, bandwidth, nrow);                \
      const T a2 = A3(columnwise_matrix, 2, i, cell, bandwidth, nrow);                \
      const T a3 = A3(columnwise_matrix, 3, i, cell, bandwidth, nrow);                \
      if (i == 1) {                                                                   \
        inv_denom = (T)1 / a2;                                                        \
        V(c_prime, i) = inv_denom * a3;                                               \
        V(d_prime, i) = inv_denom * V(x, mu_i);                                       \
      } else {                                                                        \
        inv_denom = (T)1 / (a2 - a1 * V(c_prime, i - 1));                             \
        if (i < nrow) V(c_prime, i) = inv_denom * a3;                                 \
        V(d_prime, i) = inv_denom * (V(x, mu_i) - a1 * V(d_prime, i - 1));            \
      }                                                                               \
    }                                                                                 \
    for (int i = nrow; i >= 1; --i) {                                                 \
      int mu_i = V(map, 1) + V(indirection_dofmap, i) - 1;                            \
      if (i < nrow) V(d_prime, i) = V(d_prime, i) - V(c_prime, i) * V(d_prime, i + 1);\
      V(lhs, mu_i) = V(d_prime, i);                                                   \
    }                                                                                 \
  }
DEF_CMA_APPINV(double, r_double)
DEF_CMA_APPINV(float, r_single)

/* components/science/source/kernel/solver/sci_tri_solve_kernel_mod.f90:72-156 */
#define DEF_TRI_SOLVE(T, SFX)                                                         \
  void ora_tri_solve_code_##SFX(int nlayers, T* y, const T* x, const T* tri_0,        \
                                const T* tri_plus, const T* tri_minus, int ndf,       \
                                int undf, const int* map, T* x_new,                   \
                                T* tri_plus_new) {                                    \
    (void)ndf; (void)undf;                                                            \
    int k = 0;                                                                        \
    int ij = V(map, 1);                                                               \
    T denom = (T)1 / V(tri_0, ij + k);                                                \
    V(tri_plus_new, 1) = V(tri_plus, ij + k) * denom;                                 \
    V(x_new, 1) = V(x, ij + k) * denom;                                               \
    for (k = 1; k <= nlayers - 1; ++k) {                                              \
      denom = (T)1 / (V(tri_0, ij + k) - V(tri_minus, ij + k) * V(tri_plus_new, k));  \
      V(tri_plus_new, k + 1) = V(tri_plus, ij + k) * denom;                           \
      V(x_new, k + 1) = (V(x, ij + k) - V(tri_minus, ij + k) * V(x_new, k)) * denom;  \
    }                                                                                 \
    k = nlayers - 1;                                                                  \
    V(y, ij + k) = V(x_new, k + 1);                                                   \
    for (k = nlayers - 2; k >= 0; --k)                                                \
      V(y, ij + k) = V(x_new, k + 1) - V(tri_plus_new, k + 1) * V(y, ij + k + 1);     \
  }
DEF_TRI_SOLVE(double, r_double)
DEF_TRI_SOLVE(float, r_single)

/* components/science/source/kernel/solver/sci_operator_tri_solve_kernel_mod.f90:69-120
 * Tridiagonal of nlayers+1 rows assembled from the 2x2 LMA, then Thomas.
 * Work arrays are indexed 0..nlayers (length nlayers+1 each). */
void ora_operator_tri_solve_code(int cell, int nlayers, double* y, const double* x,
                                 int ncell, const double* matrix, int ndf, int undf,
                                 const int* map, double* work) {
  (void)undf;
  double* tri_p = work;
  double* tri_0 = work + (nlayers + 1);
  double* tri_m = work + 2 * (nlayers + 1);
  double* x_new = work + 3 * (nlayers + 1);
  double* tri_p_new = work + 4 * (nlayers + 1);
  tri_0[0] = 0.0;
  tri_m[0] = 0.0;
  for (int k = 0; k <= nlayers - 1; ++k) {
    int ik = 1 + k + (cell - 1) * nlayers;
    tri_0[k] = A3(matrix, ik, 1, 1, ncell, ndf) + tri_0[k];
    tri_p[k] = A3(matrix, ik, 1, 2, ncell, ndf);
    tri_m[k + 1] = A3(matrix, ik, 2, 1, ncell, ndf);
    tri_0[k + 1] = A3(matrix, ik, 2, 2, ncell, ndf);
  }
  tri_p[nlayers] = 0.0;
  int k = 0;
  int ij = V(map, 1);
  double denom = 1.0 / tri_0[k];
  tri_p_new[k] = tri_p[k] * denom;
  x_new[k] = V(x, ij + k) * denom;
  for (k = 1; k <= nlayers; ++k) {
    denom = 1.0 / (tri_0[k] - tri_m[k] * tri_p_new[k - 1]);
    tri_p_new[k] = tri_p[k] * denom;
    x_new[k] = (V(x, ij + k) - tri_m[k] * x_new[k - 1]) * denom;
  }
  k = nlayers;
  V(y, ij + k) = x_new[k];
  for (k = nlayers - 1; k >= 0; --k) V(y, ij + k) = x_new[k] - tri_p_new[k] * V(y, ij + k + 1);
}

/* ------------------------------------------------------------------------
 * Intergrid kernels.  cell_map is cell_map(nx, ny), Fortran order, 1-based
 * fine cell ids; map_fine is map_fine(ndf, ncell_fine).
 * ---------------------------------------------------------------------- */

/* sci_restrict_scalar_unweighted_kernel_mod.F90:71-183 */
#define DEF_RESTRICT_UNWEIGHTED(T, SFX)                                               \
  void ora_restrict_scalar_unweighted_code_##SFX(                                     \
      int nlayers, const int* cell_map, int nx, int ny, int ncell_fine, T* coarse,    \
      const T* fine, int undf_coarse, const int* map_coarse, int ndf, int undf_fine,  \
      const int* map_fine, T* coarse_value) {                                         \
    (void)ncell_fine; (void)undf_coarse; (void)undf_fine;                             \
    T denom = (T)1 / (T)(nx * ny);                                                    \
    int top_df = nlayers - 2 + ndf;                                                   \
    for (int k = 0; k <= top_df; ++k) coarse_value[k] = (T)0;                         \
    for (int y = 1; y <= ny; ++y)                                                     \
      for (int x = 1; x <= nx; ++x) {                                                 \
        int c = A2(cell_map, x, y, nx);                                               \
        for (int k = 0; k <= top_df; ++k)                                             \
          coarse_value[k] = coarse_value[k] + V(fine, A2(map_fine, 1, c, ndf) + k) * denom; \
      }                                                                               \
    for (int k = 0; k <= top_df; ++k) V(coarse, V(map_coarse, 1) + k) = coarse_value[k]; \
  }
DEF_RESTRICT_UNWEIGHTED(double, r_double)
DEF_RESTRICT_UNWEIGHTED(float, r_single)

/* sci_restrict_scalar_weighted_kernel_mod.F90:77-196: fine * denom / weights */
#define DEF_RESTRICT_WEIGHTED(T, SFX)                                                 \
  void ora_restrict_scalar_weighted_code_##SFX(                                       \
      int nlayers, const int* cell_map, int nx, int ny, int ncell_fine, T* coarse,    \
      const T* fine, const T* weights, int undf_coarse, const int* map_coarse,        \
      int ndf, int undf_fine, const int* map_fine, T* coarse_value) {                 \
    (void)ncell_fine; (void)undf_coarse; (void)undf_fine;                             \
    T denom = (T)1 / (T)(nx * ny);                                                    \
    int top_df = nlayers - 2 + ndf;                                                   \
    for (int k = 0; k <= top_df; ++k) coarse_value[k] = (T)0;                         \
    for (int y = 1; y <= ny; ++y)                                                     \
      for (int x = 1; x <= nx; ++x) {                                                 \
        int c = A2(cell_map, x, y, nx);                                               \
        for (int k = 0; k <= top_df; ++k) {                                           \
          int d = A2(map_fine, 1, c, ndf) + k;                                        \
          coarse_value[k] = coarse_value[k] + V(fine, d) * denom / V(weights, d);     \
        }                                                                             \
      }                                                                               \
    for (int k = 0; k <= top_df; ++k) V(coarse, V(map_coarse, 1) + k) = coarse_value[k]; \
  }
DEF_RESTRICT_WEIGHTED(double, r_double)
DEF_RESTRICT_WEIGHTED(float, r_single)

/* sci_restrict_mass_w3_kernel_mod.F90:70-179: plain sum of the fine values */
#define DEF_RESTRICT_MASS_W3(T, SFX)                                                  \
  void ora_restrict_mass_w3_code_##SFX(                                               \
      int nlayers, const int* cell_map, int nx, int ny, int ncell_fine, T* coarse,    \
      const T* fine, int undf_coarse, const int* map_coarse, int ndf, int undf_fine,  \
      const int* map_fine, T* coarse_value) {                                         \
    (void)ncell_fine; (void)undf_coarse; (void)undf_fine;                             \
    int top_df = nlayers - 2 + ndf;                                                   \
    for (int k = 0; k <= top_df; ++k) coarse_value[k] = (T)0;                         \
    for (int y = 1; y <= ny; ++y)                                                     \
      for (int x = 1; x <= nx; ++x) {                                                 \
        int c = A2(cell_map, x, y, nx);                                               \
        for (int k = 0; k <= top_df; ++k)                                             \
          coarse_value[k] = coarse_value[k] + V(fine, A2(map_fine, 1, c, ndf) + k);   \
      }                                                                               \
    for (int k = 0; k <= top_df; ++k) V(coarse, V(map_coarse, 1) + k) = coarse_value[k]; \
  }
DEF_RESTRICT_MASS_W3(double, r_double)
DEF_RESTRICT_MASS_W3(float, r_single)

/* sci_prolong_scalar_unweighted_kernel_mod.F90:74-169: fine += coarse */
#define DEF_PROLONG_UNWEIGHTED(T, SFX)                                                \
  void ora_prolong_scalar_unweighted_code_##SFX(                                      \
      int nlayers, const int* cell_map, int nx, int ny, int ncell_fine, T* fine,      \
      const T* coarse, int ndf, int undf_fine, const int* map_fine, int undf_coarse,  \
      const int* map_coarse) {                                                        \
    (void)ncell_fine; (void)undf_coarse; (void)undf_fine;                             \
    int top_df = nlayers - 2 + ndf;                                                   \
    for (int y = 1; y <= ny; ++y)                                                     \
      for (int x = 1; x <= nx; ++x) {                                                 \
        int c = A2(cell_map, x, y, nx);                                               \
        for (int k = 0; k <= top_df; ++k) {                                           \
          int d = A2(map_fine, 1, c, ndf) + k;                                        \
          V(fine, d) = V(fine, d) + V(coarse, V(map_coarse, 1) + k);                  \
        }                                                                             \
      }                                                                               \
  }
DEF_PROLONG_UNWEIGHTED(double, r_double)
DEF_PROLONG_UNWEIGHTED(float, r_single)

/* sci_prolong_scalar_weighted_kernel_mod.F90:77-178: fine += weights * coarse */
#define DEF_PROLONG_WEIGHTED(T, SFX)                                                  \
  void ora_prolong_scalar_weighted_code_##SFX(                                        \
      int nlayers, const int* cell_map, int nx, int ny, int ncell_fine, T* fine,      \
      const T* coarse, const T* weights, int ndf, int undf_fine, const int* map_fine, \
      int undf_coarse, const int* map_coarse) {                                       \
    (void)ncell_fine; (void)undf_coarse; (void)undf_fine;                             \
    int top_df = nlayers - 2 + ndf;                                                   \
    for (int y = 1; y <= ny; ++y)                                                     \
      for (int x = 1; x <= nx; ++x) {                                                 \
        int c = A2(cell_map, x, y, nx);                                               \
        for (int k = 0; k <= top_df; ++k) {                                           \
          int d = A2(map_fine, 1, c, ndf) + k;                                        \
          V(fine, d) = V(fine, d) + V(weights, d) * V(coarse, V(map_coarse, 1) + k);  \
        }                                                                             \
      }                                                                               \
  }
DEF_PROLONG_WEIGHTED(double, r_double)
DEF_PROLONG_WEIGHTED(float, r_single)

enum { SWB = 1, SEB = 2, NEB = 3, NWB = 4 };

/* sci_restrict_w0_kernel_mod.F90:75-154: injection of the four coarse
 * bottom corners from the corner fine cells, levels 0..nlayers. */
void ora_restrict_w0_code(int nlayers, const int* cell_map, int nx, int ny, int ncell_fine,
                          double* coarse, const double* fine, int undf_coarse,
                          const int* map_coarse, int ndf, int undf_fine,
                          const int* map_fine) {
  (void)ncell_fine; (void)undf_coarse; (void)undf_fine;
  for (int k = 0; k <= nlayers; ++k) {
    V(coarse, V(map_coarse, NWB) + k) = V(fine, A2(map_fine, NWB, A2(cell_map, 1, 1, nx), ndf) + k);
    V(coarse, V(map_coarse, SWB) + k) = V(fine, A2(map_fine, SWB, A2(cell_map, 1, ny, nx), ndf) + k);
    V(coarse, V(map_coarse, NEB) + k) = V(fine, A2(map_fine, NEB, A2(cell_map, nx, 1, nx), ndf) + k);
    V(coarse, V(map_coarse, SEB) + k) = V(fine, A2(map_fine, SEB, A2(cell_map, nx, ny, nx), ndf) + k);
  }
}

/* sci_prolong_w0_kernel_mod.F90:76-194: bilinear weights from the four
 * coarse corners; SE dofs on the last column, NW dofs on the first row and
 * the NE dof of the NE fine cell are filled as well. */
void ora_prolong_w0_code(int nlayers, const int* cell_map, int nx, int ny, int ncell_fine,
                         double* fine, const double* coarse, int ndf, int undf_fine,
                         const int* map_fine, int undf_coarse, const int* map_coarse) {
  (void)ncell_fine; (void)undf_fine; (void)undf_coarse;
  for (int y = 1; y <= ny; ++y) {
    for (int x = 1; x <= nx; ++x) {
      int c = A2(cell_map, x, y, nx);
      double w_sw = (double)y * (double)(nx - x + 1) / (double)(nx * ny);
      double w_nw = (double)(ny - y) * (double)(nx - x + 1) / (double)(nx * ny);
      double w_ne = (double)(ny - y) * (double)(x - 1) / (double)(nx * ny);
      double w_se = (double)y * (double)(x - 1) / (double)(nx * ny);
      for (int k = 0; k <= nlayers; ++k)
        V(fine, A2(map_fine, SWB, c, ndf) + k) =
            w_ne * V(coarse, V(map_coarse, NEB) + k) + w_se * V(coarse, V(map_coarse, SEB) + k) +
            w_sw * V(coarse, V(map_coarse, SWB) + k) + w_nw * V(coarse, V(map_coarse, NWB) + k);
      if (x == nx) {
        w_se = (double)y / (double)ny;
        w_ne = 1.0 - w_se;
        for (int k = 0; k <= nlayers; ++k)
          V(fine, A2(map_fine, SEB, c, ndf) + k) =
              w_ne * V(coarse, V(map_coarse, NEB) + k) + w_se * V(coarse, V(map_coarse, SEB) + k);
      }
      if (y == 1) {
        w_nw = (double)(nx - x + 1) / (double)nx;
        w_ne = 1.0 - w_nw;
        for (int k = 0; k <= nlayers; ++k)
          V(fine, A2(map_fine, NWB, c, ndf) + k) =
              w_ne * V(coarse, V(map_coarse, NEB) + k) + w_nw * V(coarse, V(map_coarse, NWB) + k);
        if (x == nx)
          for (int k = 0; k <= nlayers; ++k)
            V(fine, A2(map_fine, NEB, c, ndf) + k) = V(coarse, V(map_coarse, NEB) + k);
      }
    }
  }
}

/* ------------------------------------------------------------------------
 * CMA parameters: infrastructure/source/operator/columnwise_operator_mod.f90
 * :170-198 (alpha, beta, gamma, gcd division, bandwidth), :350-396
 * (indirection maps) and :427-470 (nrow, ncol), for horizontally
 * discontinuous spaces whose cell dofmap is [bottom face..., interior...,
 * top face...] offsets from the first dof (passed as dof_offsets, 0-based
 * offsets relative to the first dof, ndof_cell entries each).
 * out = {alpha, beta, gamma_m, gamma_p, bandwidth, nrow, ncol}.
 * ---------------------------------------------------------------------- */
static int gcd_int(int a, int b) {
  while (b) { int t = a % b; a = b; b = t; }
  return a;
}

void ora_cma_params(int nlayers, int nint_to, int nface_to, int nint_from, int nface_from,
                    const int* offsets_to, const int* offsets_from, int* out,
                    int* indirection_to, int* indirection_from) {
  int ncell_to = nint_to + 2 * nface_to, ncell_from = nint_from + 2 * nface_from;
  int alpha = nint_from + nface_from;
  int beta = nint_to + nface_to;
  int gamma_m = (ncell_from - 1) * (nint_to + nface_to);
  int gamma_p = (ncell_to - 1) * (nint_from + nface_from);
  int g = gcd_int(alpha, beta);
  alpha /= g; beta /= g; gamma_m /= g; gamma_p /= g;
  int bw = 1 + (int)ceil((double)(gamma_m + gamma_p) / (double)beta);
  int nrow = nlayers * nint_to + (nlayers + 1) * nface_to;
  int ncol = nlayers * nint_from + (nlayers + 1) * nface_from;
  out[0] = alpha; out[1] = beta; out[2] = gamma_m; out[3] = gamma_p;
  out[4] = bw; out[5] = nrow; out[6] = ncol;
  for (int k = 1; k <= nlayers; ++k) {
    for (int df = 1; df <= ncell_to; ++df) {
      int col = offsets_to[df - 1] + 1 + (k - 1);
      int banded = (k - 1) * (nint_to + nface_to) + df;
      indirection_to[banded - 1] = col;
    }
    for (int df = 1; df <= ncell_from; ++df) {
      int col = offsets_from[df - 1] + 1 + (k - 1);
      int banded = (k - 1) * (nint_from + nface_from) + df;
      indirection_from[banded - 1] = col;
    }
  }
}

/* ------------------------------------------------- W2 intergrid transfers
 * components/science/source/kernel/inter_mesh/: per coarse cell, with the
 * reference's W2 dof numbering W=1, S=2, E=3, N=4, B=5, T=6, cell_map(x, y)
 * (x W->E, y N->S) and 1-based maps. */
enum { ORA_W = 1, ORA_S = 2, ORA_E = 3, ORA_N = 4, ORA_B = 5 };

/* fine-cell ranges of each horizontal face of the coarse cell */
static void ora_w2_face_ranges(int nx, int ny, int xs[5], int xe[5], int ys[5], int ye[5]) {
  xs[ORA_N] = 1; xe[ORA_N] = nx; ys[ORA_N] = 1; ye[ORA_N] = 1;
  xs[ORA_S] = 1; xe[ORA_S] = nx; ys[ORA_S] = ny; ye[ORA_S] = ny;
  xs[ORA_W] = 1; xe[ORA_W] = 1; ys[ORA_W] = 1; ye[ORA_W] = ny;
  xs[ORA_E] = nx; xe[ORA_E] = nx; ys[ORA_E] = 1; ye[ORA_E] = ny;
}

/* sci_restrict_w2_kernel_mod.F90 restrict_w2_code_r_double (with_b = 1) and
 * sci_restrict_w2h_kernel_mod.F90 restrict_w2h_code_r_double (with_b = 0) */
#define DEF_RESTRICT_W2(T, SFX)                                                       \
  void ora_restrict_w2_code_##SFX(int nlayers, const int* cell_map, int nx, int ny,   \
                                  int ncell_fine, T* coarse, const T* fine,           \
                                  const int* sel_ew, const int* sel_ns,               \
                                  const int* map_coarse, int ndf,                     \
                                  const int* map_fine, const int* map_w3_2d,          \
                                  int with_b, T* work) {                              \
    (void)ncell_fine;                                                                 \
    int xs[5], xe[5], ys[5], ye[5];                                                   \
    ora_w2_face_ranges(nx, ny, xs, xe, ys, ye);                                       \
    const int ew = V(sel_ew, V(map_w3_2d, 1)), ns = V(sel_ns, V(map_w3_2d, 1));       \
    for (int face = 1; face <= ew + ns; ++face) {                                     \
      int df = face;                                                                  \
      if (face == 3 && ns == 2 && ew == 1) df = ORA_N;                                \
      for (int k = 0; k < nlayers; ++k) work[k] = (T)0;                               \
      for (int y = ys[df]; y <= ye[df]; ++y)                                          \
        for (int x = xs[df]; x <= xe[df]; ++x)                                        \
          for (int k = 0; k < nlayers; ++k)                                           \
            work[k] = work[k] +                                                       \
                V(fine, A2(map_fine, df, A2(cell_map, x, y, nx), ndf) + k);           \
      for (int k = 0; k < nlayers; ++k) V(coarse, V(map_coarse, df) + k) = work[k];   \
    }                                                                                 \
    if (!with_b) return;                                                              \
    for (int k = 0; k <= nlayers; ++k) work[k] = (T)0;                                \
    for (int y = 1; y <= ny; ++y)                                                     \
      for (int x = 1; x <= nx; ++x)                                                   \
        for (int k = 0; k <= nlayers; ++k)                                            \
          work[k] = work[k] + V(fine, A2(map_fine, ORA_B, A2(cell_map, x, y, nx), ndf) + k); \
    for (int k = 0; k <= nlayers; ++k) V(coarse, V(map_coarse, ORA_B) + k) = work[k]; \
  }
DEF_RESTRICT_W2(double, r_double)
DEF_RESTRICT_W2(float, r_single)

/* sci_restrict_w2v_kernel_mod.F90 restrict_w2v_code_r_double: the B column (df 1) */
#define DEF_RESTRICT_W2V(T, SFX)                                                      \
  void ora_restrict_w2v_code_##SFX(int nlayers, const int* cell_map, int nx, int ny,  \
                                   int ncell_fine, T* coarse, const T* fine,          \
                                   const int* map_coarse, int ndf,                    \
                                   const int* map_fine, T* work) {                    \
    (void)ncell_fine;                                                                 \
    for (int k = 0; k <= nlayers; ++k) work[k] = (T)0;                                \
    for (int y = 1; y <= ny; ++y)                                                     \
      for (int x = 1; x <= nx; ++x)                                                   \
        for (int k = 0; k <= nlayers; ++k)                                            \
          work[k] = work[k] + V(fine, A2(map_fine, 1, A2(cell_map, x, y, nx), ndf) + k); \
    for (int k = 0; k <= nlayers; ++k) V(coarse, V(map_coarse, 1) + k) = work[k];     \
  }
DEF_RESTRICT_W2V(double, r_double)
DEF_RESTRICT_W2V(float, r_single)

/* sci_weights_prolong_w2_kernel_mod.F90 weights_prolong_w2_kernel_code */
void ora_weights_prolong_w2_code(int nlayers, const int* cell_map, int nx, int ny,
                                 int ncell_fine, double* w, int ndf, const int* map_fine) {
  (void)ncell_fine;
#define WF(df, x, y, k) V(w, A2(map_fine, df, A2(cell_map, x, y, nx), ndf) + (k))
  for (int k = 0; k < nlayers; ++k) {
    for (int x = 1; x <= nx; ++x) {
      WF(ORA_N, x, 1, k) = 1.0 / (double)nx;
      WF(ORA_S, x, ny, k) = 1.0 / (double)nx;
    }
    for (int y = 1; y <= ny; ++y) {
      WF(ORA_W, 1, y, k) = 1.0 / (double)ny;
      WF(ORA_E, nx, y, k) = 1.0 / (double)ny;
    }
    for (int y = 1; y <= ny; ++y)
      for (int x = 2; x <= nx; ++x) WF(ORA_W, x, y, k) = (double)(nx + 1 - x) / (double)nx;
    for (int x = 1; x <= nx; ++x)
      for (int y = 2; y <= ny; ++y) WF(ORA_N, x, y, k) = (double)(ny + 1 - y) / (double)ny;
  }
  for (int k = 0; k <= nlayers; ++k)
    for (int y = 1; y <= ny; ++y)
      for (int x = 1; x <= nx; ++x) WF(ORA_B, x, y, k) = 1.0 / (double)(nx * ny);
#undef WF
}

/* sci_prolong_w2_kernel_mod.F90 prolong_w2_kernel_code */
void ora_prolong_w2_code(int nlayers, const int* cell_map, int nx, int ny, int ncell_fine,
                         double* fine, const double* coarse, const double* w, int ndf,
                         const int* map_fine, const int* map_coarse) {
  (void)ncell_fine;
#define FI(df, x, y, k) (A2(map_fine, df, A2(cell_map, x, y, nx), ndf) + (k))
#define CO(df, k) V(coarse, V(map_coarse, df) + (k))
  for (int k = 0; k < nlayers; ++k) {
    for (int x = 1; x <= nx; ++x) {
      V(fine, FI(ORA_N, x, 1, k)) = V(w, FI(ORA_N, x, 1, k)) * CO(ORA_N, k);
      V(fine, FI(ORA_S, x, ny, k)) = V(w, FI(ORA_S, x, ny, k)) * CO(ORA_S, k);
    }
    for (int y = 1; y <= ny; ++y) {
      V(fine, FI(ORA_W, 1, y, k)) = V(w, FI(ORA_W, 1, y, k)) * CO(ORA_W, k);
      V(fine, FI(ORA_E, nx, y, k)) = V(w, FI(ORA_E, nx, y, k)) * CO(ORA_E, k);
    }
    for (int y = 1; y <= ny; ++y) {
      const double ew = V(w, FI(ORA_W, 1, y, k));
      for (int x = 2; x <= nx; ++x) {
        const double iw = V(w, FI(ORA_W, x, y, k));
        V(fine, FI(ORA_W, x, y, k)) = ew * (iw * CO(ORA_W, k) + (1.0 - iw) * CO(ORA_E, k));
      }
    }
    for (int x = 1; x <= nx; ++x) {
      const double ew = V(w, FI(ORA_N, x, 1, k));
      for (int y = 2; y <= ny; ++y) {
        const double iw = V(w, FI(ORA_N, x, y, k));
        V(fine, FI(ORA_N, x, y, k)) = ew * (iw * CO(ORA_N, k) + (1.0 - iw) * CO(ORA_S, k));
      }
    }
  }
  for (int y = 1; y <= ny; ++y)
    for (int x = 1; x <= nx; ++x)
      for (int k = 0; k <= nlayers; ++k)
        V(fine, FI(ORA_B, x, y, k)) = V(w, FI(ORA_B, x, y, k)) * CO(ORA_B, k);
#undef FI
#undef CO
}

// Columnwise (CMA) operator assembly on the device: the kernels that build
// the banded column matrices from LMA element matrices and combine them.
//
//   lfg_cma_assemble            columnwise_op_asm_kernel_code
//                               (sci_columnwise_op_asm_kernel_mod.F90)
//   lfg_cma_multiply            columnwise_op_mul_kernel_code          C += A B
//   lfg_cma_scaled_add          columnwise_op_scaledadd_kernel_code    C = a A + b B
//   lfg_cma_assemble_diag_hmht  columnwise_op_asm_diag_hmht_kernel_code
//                               C = diag-weighted D M2h^{-1} D^T per cell
//   lfg_cma_assemble_m2v_lumped_inv
//                               columnwise_op_asm_m2v_lumped_inv_krnl_code
//
// Layout: bands [bw][nrow][ncol] and LMA values [df_to][df_from][layer][cell]
// (level-major, one thread per column or per (row, column), so a warp
// touches 32 consecutive columns).  Every column is written by one thread
// in the reference's loop order, so sums keep the reference's order.
// column_banded_dofmap(df, k) is the 1-based row (or column) of dof df of
// layer k within the column matrix, as columnwise_operator_type builds it
// (infrastructure/source/operator/columnwise_operator_mod.f90:377-393).
#include <cuda_runtime.h>

#include <vector>

#include "lfg_internal.cuh"

namespace {

using namespace lfg;

template <class F>
void dispatch_kind(int kind, F&& f) {
  if (kind == LFG_R_DOUBLE) f(double{});
  else f(float{});
}

// columnwise_op_asm_kernel_code: zero the column, then for every layer k,
// to-dof df1 and from-dof df2 add local_stencil(ik, df1, df2) at row
// i = cb_to(df1, k), band j - j_minus(i) with j = cb_from(df2, k).
template <class T, class TL>
__global__ void k_cma_asm(T* __restrict__ bands, const int* __restrict__ jminus, int ncol,
                          int nrow, int bw, const TL* __restrict__ a, int ndf_to, int ndf_from,
                          int nl, const int* __restrict__ cb_to, const int* __restrict__ cb_from) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  const size_t plane = (size_t)nrow * ncol;
  for (int b = 0; b < bw; ++b)
    for (int i = 0; i < nrow; ++i) bands[b * plane + (size_t)i * ncol + c] = (T)0;
  for (int k = 0; k < nl; ++k)
    for (int d1 = 0; d1 < ndf_to; ++d1) {
      const int i = cb_to[k * ndf_to + d1] - 1;
      const int jm = jminus[i];
      for (int d2 = 0; d2 < ndf_from; ++d2) {
        const int b = cb_from[k * ndf_from + d2] - 1 - jm;
        const size_t o = b * plane + (size_t)i * ncol + c;
        bands[o] = bands[o] + (T)a[(((size_t)d1 * ndf_from + d2) * nl + k) * ncol + c];
      }
    }
}

// The same assembly one thread per (row i, column): the row's
// contributions, (a plane (d1 ndf_from + d2) nl + k, band b) in the
// reference's loop order (k, then d1, then d2), are listed on the host; a
// thread sums them in registers, so every band entry gets its terms in the
// sequential kernel's order (the same bits), and writes each of the row's
// bands once, zeros included.  The sequential kernel's read-modify-write
// chain per level left it latency-bound (C96 x 70 W3 <- Wtheta: 136 us,
// 0.14 of the HBM copy bandwidth).
// INV: every non-zero entry then inverted (the lumped inverse of
// columnwise_op_asm_m2v_lumped_inv, whose contributions are the diagonal
// entries M(d, d) on band 0).  A thread takes kAsmColsPerThread columns of
// its row, so one read of the row's list serves all of them and their
// element loads are in flight together (the list chain left the kernel
// latency-bound: C96 x 70 W3 <- Wtheta 29.8 -> 24.4 us).
constexpr int kAsmColsPerThread = 4;
template <class T, class TL, int BW, bool INV = false>
__global__ void __launch_bounds__(128) k_cma_asm_rows(T* __restrict__ bands, int ncol, int nrow,
                                                      int bw, const TL* __restrict__ a,
                                                      const int* __restrict__ rowptr,
                                                      const int2* __restrict__ contrib) {
  grid_dep_wait();
  constexpr int CPT = kAsmColsPerThread;
  const int c0 = blockIdx.x * blockDim.x * CPT + threadIdx.x;
  const int i = blockIdx.y;
  if (c0 >= ncol) return;
  T acc[CPT][BW];
#pragma unroll
  for (int u = 0; u < CPT; ++u)
#pragma unroll
    for (int b = 0; b < BW; ++b) acc[u][b] = (T)0;
  for (int q = rowptr[i]; q < rowptr[i + 1]; ++q) {
    const int2 e = contrib[q];
    T v[CPT];
#pragma unroll
    for (int u = 0; u < CPT; ++u) {
      const int c = c0 + u * blockDim.x;
      v[u] = c < ncol ? (T)a[(size_t)e.x * ncol + c] : (T)0;
    }
#pragma unroll
    for (int u = 0; u < CPT; ++u)
#pragma unroll
      for (int b = 0; b < BW; ++b)
        if (b == e.y) acc[u][b] = acc[u][b] + v[u];
  }
  const size_t plane = (size_t)nrow * ncol;
#pragma unroll
  for (int u = 0; u < CPT; ++u) {
    const int c = c0 + u * blockDim.x;
    if (c >= ncol) break;
#pragma unroll
    for (int b = 0; b < BW; ++b) {
      T v = acc[u][b];
      if (INV && v != (T)0) v = (T)1 / v;
      if (b < bw) bands[b * plane + (size_t)i * ncol + c] = v;
    }
  }
}

// columnwise_op_asm_diag_hmht one thread per (row i, column): the row's
// entries (layer k, dofs d1, d2 of W3, band b) in the reference's loop
// order, each adding sum over d3 of Dh(d1, d3) Dh(d2, d3) / M2h(d3, d3) at
// layer k, formed in the element matrices' precision as in k_cma_asm_hmht.
// Q > 0 and NDF > 0 (rows of at most Q entries, ndf2h = NDF): every load of
// the row issued before the first product (the loads in flight together; a
// loop over d3 left each thread one load at a time: 85 -> 58 us on C96 x 70
// W3); otherwise loops over any number of entries and dofs.  Rows of one
// entry run 12 blocks per SM (their registers allowed 10: 53.8 -> 51.1 us).
template <class T, class TL, int BW, int Q, int NDF>
__global__ void __launch_bounds__(128, Q == 1 ? 12 : 1) k_cma_hmht_rows(T* __restrict__ bands, int ncol, int nrow,
                                                       int bw, const TL* __restrict__ dh,
                                                       const TL* __restrict__ m2h, int ndf2h,
                                                       int nl, const int* __restrict__ rowptr,
                                                       const int2* __restrict__ contrib) {
  grid_dep_wait();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (c >= ncol) return;
  T acc[BW];
#pragma unroll
  for (int b = 0; b < BW; ++b) acc[b] = (T)0;
  const int q0 = rowptr[i], q1 = rowptr[i + 1];
  if constexpr (Q > 0 && NDF > 0) {
    int2 e[Q];
    TL x1[Q][NDF], x2[Q][NDF], mm[Q][NDF];
#pragma unroll
    for (int u = 0; u < Q; ++u) e[u] = q0 + u < q1 ? contrib[q0 + u] : make_int2(0, -1);
#pragma unroll
    for (int u = 0; u < Q; ++u) {
      const int k = e[u].x & 0xffff, d1 = (e[u].x >> 16) & 0xff,
                d2 = (int)((unsigned)e[u].x >> 24);
      const bool on = e[u].y >= 0;
#pragma unroll
      for (int d3 = 0; d3 < NDF; ++d3) {
        x1[u][d3] = on ? dh[(((size_t)d1 * NDF + d3) * nl + k) * ncol + c] : (TL)0;
        x2[u][d3] = on ? dh[(((size_t)d2 * NDF + d3) * nl + k) * ncol + c] : (TL)0;
        mm[u][d3] = on ? m2h[(((size_t)d3 * NDF + d3) * nl + k) * ncol + c] : (TL)1;
      }
    }
#pragma unroll
    for (int u = 0; u < Q; ++u) {
      TL tmp = (TL)0;
#pragma unroll
      for (int d3 = 0; d3 < NDF; ++d3) tmp = tmp + x1[u][d3] * x2[u][d3] / mm[u][d3];
#pragma unroll
      for (int b = 0; b < BW; ++b)
        if (b == e[u].y) acc[b] = acc[b] + (T)tmp;
    }
  } else {
    for (int q = q0; q < q1; ++q) {
      const int2 e = contrib[q];
      const int k = e.x & 0xffff, d1 = (e.x >> 16) & 0xff, d2 = (int)((unsigned)e.x >> 24);
      TL tmp = (TL)0;
      for (int d3 = 0; d3 < ndf2h; ++d3)
        tmp = tmp + dh[(((size_t)d1 * ndf2h + d3) * nl + k) * ncol + c] *
                        dh[(((size_t)d2 * ndf2h + d3) * nl + k) * ncol + c] /
                        m2h[(((size_t)d3 * ndf2h + d3) * nl + k) * ncol + c];
#pragma unroll
      for (int b = 0; b < BW; ++b)
        if (b == e.y) acc[b] = acc[b] + (T)tmp;
    }
  }
  const size_t plane = (size_t)nrow * ncol;
#pragma unroll
  for (int b = 0; b < BW; ++b)
    if (b < bw) bands[b * plane + (size_t)i * ncol + c] = acc[b];
}

// columnwise_op_mul_kernel_code, one thread per (row i of C, column):
// C(j, i) += sum over ell in A's band of row i of A(ell, i) B(j, ell), for
// the ell whose B band reaches j.
template <class T>
__global__ void k_cma_mul(T* __restrict__ cb, const int* __restrict__ jmC,
                          const int* __restrict__ jpC, int ncolC, int bwC,
                          const T* __restrict__ ab, const int* __restrict__ jmA,
                          const int* __restrict__ jpA, int ncolA,
                          const T* __restrict__ bb, const int* __restrict__ jmB,
                          const int* __restrict__ jpB, int nrowA, int nrowB, int ncol) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (c >= ncol) return;
  const int j0 = max(0, jmC[i]), j1 = min(ncolC - 1, jpC[i]);
  const int l0 = max(0, jmA[i]), l1 = min(ncolA - 1, jpA[i]);
  for (int j = j0; j <= j1; ++j) {
    T e = (T)0;
    for (int l = l0; l <= l1; ++l) {
      if (jmB[l] <= j && j <= jpB[l])
        e = e + ab[((size_t)(l - jmA[i]) * nrowA + i) * ncol + c] *
                    bb[((size_t)(j - jmB[l]) * nrowB + l) * ncol + c];
    }
    const size_t o = ((size_t)(j - jmC[i]) * gridDim.y + i) * ncol + c;
    cb[o] = cb[o] + e;
  }
  (void)bwC;
}

// The same product with A's band span at most MA and C's at most MC: A's and
// C's entries of the row and every B entry a term needs are loaded before
// the first product; the terms are added in the same order.
template <class T, int MA, int MC>
__global__ void __launch_bounds__(128) k_cma_mul_u(T* __restrict__ cb, const int* __restrict__ jmC,
                                                   const int* __restrict__ jpC, int ncolC,
                                                   const T* __restrict__ ab,
                                                   const int* __restrict__ jmA,
                                                   const int* __restrict__ jpA, int ncolA,
                                                   const T* __restrict__ bb,
                                                   const int* __restrict__ jmB,
                                                   const int* __restrict__ jpB, int nrowA,
                                                   int nrowB, int ncol) {
  grid_dep_wait();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (c >= ncol) return;
  const int jmc = jmC[i], jma = jmA[i];
  const int j0 = max(0, jmc), j1 = min(ncolC - 1, jpC[i]);
  const int l0 = max(0, jma), l1 = min(ncolA - 1, jpA[i]);
  T av[MA], cv[MC], bv[MC][MA];
  int jmb[MA], jpb[MA];
#pragma unroll
  for (int u = 0; u < MA; ++u) {
    const int l = l0 + u;
    const bool on = l <= l1;
    jmb[u] = on ? jmB[l] : 1;
    jpb[u] = on ? jpB[l] : 0;
    av[u] = on ? ab[((size_t)(l - jma) * nrowA + i) * ncol + c] : (T)0;
  }
#pragma unroll
  for (int v = 0; v < MC; ++v) {
    const int j = j0 + v;
    cv[v] = j <= j1 ? cb[((size_t)(j - jmc) * gridDim.y + i) * ncol + c] : (T)0;
#pragma unroll
    for (int u = 0; u < MA; ++u) {
      const bool on = j <= j1 && jmb[u] <= j && j <= jpb[u];
      bv[v][u] = on ? bb[((size_t)(j - jmb[u]) * nrowB + l0 + u) * ncol + c] : (T)0;
    }
  }
#pragma unroll
  for (int v = 0; v < MC; ++v) {
    const int j = j0 + v;
    if (j > j1) break;
    T e = (T)0;
#pragma unroll
    for (int u = 0; u < MA; ++u)
      if (jmb[u] <= j && j <= jpb[u]) e = e + av[u] * bv[v][u];
    cb[((size_t)(j - jmc) * gridDim.y + i) * ncol + c] = cv[v] + e;
  }
}

// columnwise_op_scaledadd_kernel_code, one thread per (row i of C, column):
// the row is zeroed, then a A(j, i) added over A's band and b B(j, i) over
// B's band (both clipped to A's column count, as in the reference).
template <class T>
__global__ void k_cma_scaledadd(T* __restrict__ cb, const int* __restrict__ jmC, int nrowC,
                                int bwC, const T* __restrict__ ab, const int* __restrict__ jmA,
                                const int* __restrict__ jpA, int nrowA, int ncolA,
                                const T* __restrict__ bb, const int* __restrict__ jmB,
                                const int* __restrict__ jpB, int nrowB, int ncol, T alpha,
                                T beta) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (c >= ncol) return;
  for (int b = 0; b < bwC; ++b) cb[((size_t)b * nrowC + i) * ncol + c] = (T)0;
  if (i >= nrowA) return;
  for (int j = max(0, jmA[i]); j <= min(ncolA - 1, jpA[i]); ++j) {
    const size_t o = ((size_t)(j - jmC[i]) * nrowC + i) * ncol + c;
    cb[o] = cb[o] + alpha * ab[((size_t)(j - jmA[i]) * nrowA + i) * ncol + c];
  }
  for (int j = max(0, jmB[i]); j <= min(ncolA - 1, jpB[i]); ++j) {
    const size_t o = ((size_t)(j - jmC[i]) * nrowC + i) * ncol + c;
    cb[o] = cb[o] + beta * bb[((size_t)(j - jmB[i]) * nrowB + i) * ncol + c];
  }
}

// columnwise_op_asm_diag_hmht_kernel_code: per layer, the W3 x W3 block
// sum_df3 Dh(df1,df3) Dh(df2,df3) / M2h(df3,df3), placed like the asm kernel.
template <class T, class TL>
__global__ void k_cma_asm_hmht(T* __restrict__ bands, const int* __restrict__ jminus, int ncol,
                               int nrow, int bw, const TL* __restrict__ dh,
                               const TL* __restrict__ m2h, int ndf3, int ndf2h, int nl,
                               const int* __restrict__ cbm) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  const size_t plane = (size_t)nrow * ncol;
  for (int b = 0; b < bw; ++b)
    for (int i = 0; i < nrow; ++i) bands[b * plane + (size_t)i * ncol + c] = (T)0;
  auto D = [&](int d1, int d3, int k) {
    return dh[(((size_t)d1 * ndf2h + d3) * nl + k) * ncol + c];
  };
  for (int k = 0; k < nl; ++k)
    for (int d1 = 0; d1 < ndf3; ++d1) {
      const int i = cbm[k * ndf3 + d1] - 1;
      const int jm = jminus[i];
      for (int d2 = 0; d2 < ndf3; ++d2) {
        TL tmp = (TL)0;
        for (int d3 = 0; d3 < ndf2h; ++d3)
          tmp = tmp + D(d1, d3, k) * D(d2, d3, k) /
                          m2h[(((size_t)d3 * ndf2h + d3) * nl + k) * ncol + c];
        const int b = cbm[k * ndf3 + d2] - 1 - jm;
        const size_t o = b * plane + (size_t)i * ncol + c;
        bands[o] = bands[o] + (T)tmp;
      }
    }
}

// columnwise_op_asm_m2v_lumped_inv_krnl_code: band 1 of row cb(df, k)
// accumulates M(df, df); then every non-zero entry of the column is inverted.
template <class T, class TL>
__global__ void k_cma_asm_m2v(T* __restrict__ bands, int ncol, int nrow, int bw,
                              const TL* __restrict__ m, int ndf, int nl,
                              const int* __restrict__ cbm) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  const size_t plane = (size_t)nrow * ncol;
  for (int b = 0; b < bw; ++b)
    for (int i = 0; i < nrow; ++i) bands[b * plane + (size_t)i * ncol + c] = (T)0;
  for (int k = 0; k < nl; ++k)
    for (int d = 0; d < ndf; ++d) {
      const int i = cbm[k * ndf + d] - 1;
      const size_t o = (size_t)i * ncol + c;
      bands[o] = bands[o] + (T)m[(((size_t)d * ndf + d) * nl + k) * ncol + c];
    }
  for (int b = 0; b < bw; ++b)
    for (int i = 0; i < nrow; ++i) {
      const size_t o = b * plane + (size_t)i * ncol + c;
      if (bands[o] != (T)0) bands[o] = (T)1 / bands[o];
    }
}

// Host copy of the per-row band limits (0-based first / last column).
std::vector<int> host_ints(const int* d, int n) {
  std::vector<int> h(n);
  LFG_CUDA(cudaMemcpy(h.data(), d, sizeof(int) * n, cudaMemcpyDeviceToHost));
  return h;
}

// Checks a column-banded dofmap (ndf x nl, 1-based) against the matrix it
// indexes: rows within [1, nrow]; with to/from maps, every entry lands
// inside the band of its row.  Returns a device copy (caller frees).
int* checked_dofmap(const int* cb, int ndf, int nl, int nmax, const char* what) {
  LFG_REQUIRE(cb && ndf > 0 && nl > 0, std::string(what) + ": missing column-banded dofmap");
  for (int e = 0; e < ndf * nl; ++e)
    LFG_REQUIRE(cb[e] >= 1 && cb[e] <= nmax,
                std::string(what) + ": column-banded dofmap entry out of range");
  int* d = (int*)dmalloc(sizeof(int) * ndf * nl);
  upload(d, cb, sizeof(int) * ndf * nl);
  return d;
}

void check_bands(lfg_cma m, const int* cb_to, int ndf_to, const int* cb_from, int ndf_from,
                 int nl, const char* what) {
  const std::vector<int> jm = host_ints(m->jminus, m->nrow);
  for (int k = 0; k < nl; ++k)
    for (int d1 = 0; d1 < ndf_to; ++d1) {
      const int i = cb_to[k * ndf_to + d1] - 1;
      for (int d2 = 0; d2 < ndf_from; ++d2) {
        const int b = cb_from[k * ndf_from + d2] - 1 - jm[i];
        LFG_REQUIRE(b >= 0 && b < m->bw, std::string(what) +
                                             ": a dof pair falls outside the band of its row");
      }
    }
}

struct DevInts {
  int* p = nullptr;
  ~DevInts() { dfree(p); }
};

// The operator's row lists for an assembly identified by `key` (the kind of
// assembly, the shapes and the dofmaps): rebuilt by build(rows), which
// lists each row's entries in the reference's loop order, only when the key
// differs from the last assembly's.
template <class F>
void cached_rows(lfg_cma m, std::vector<int> key, F&& build) {
  if (key == m->asm_key && m->asm_rowptr) return;
  std::vector<std::vector<int2>> rows(m->nrow);
  build(rows);
  std::vector<int> rowptr(1, 0);
  std::vector<int2> list;
  int maxq = 0;
  for (const auto& r : rows) {
    list.insert(list.end(), r.begin(), r.end());
    rowptr.push_back((int)list.size());
    maxq = std::max(maxq, (int)r.size());
  }
  LFG_CUDA(cudaStreamSynchronize(m->ctx->stream));  // earlier assemblies may read the lists
  dfree(m->asm_rowptr);
  dfree(m->asm_list);
  m->asm_rowptr = nullptr;
  m->asm_list = nullptr;
  m->asm_key.clear();
  m->asm_rowptr = (int*)dmalloc(rowptr.size() * sizeof(int));
  upload(m->asm_rowptr, rowptr.data(), rowptr.size() * sizeof(int));
  m->asm_list = (int*)dmalloc(std::max<size_t>(1, list.size()) * sizeof(int2));
  if (!list.empty()) upload(m->asm_list, list.data(), list.size() * sizeof(int2));
  m->asm_key = std::move(key);
  m->asm_maxq = maxq;
}

// the dofmap's values as a key tail
std::vector<int> with_map(std::vector<int> key, const int* cb, size_t n) {
  key.insert(key.end(), cb, cb + n);
  return key;
}

}  // namespace

extern "C" {

int lfg_cma_get(lfg_cma m, double* cm) {
  if (!m || !cm) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    const size_t n = (size_t)m->bw * m->nrow * m->ncol;
    std::vector<double> dev(n);
    LFG_CUDA(cudaStreamSynchronize(c->stream));
    if (m->kind == LFG_R_DOUBLE) {
      LFG_CUDA(cudaMemcpy(dev.data(), m->bands, n * sizeof(double), cudaMemcpyDeviceToHost));
    } else {
      std::vector<float> f(n);
      LFG_CUDA(cudaMemcpy(f.data(), m->bands, n * sizeof(float), cudaMemcpyDeviceToHost));
      for (size_t e = 0; e < n; ++e) dev[e] = f[e];
    }
    for (int col = 0; col < m->ncol; ++col)
      for (int i = 0; i < m->nrow; ++i)
        for (int b = 0; b < m->bw; ++b)
          cm[((size_t)col * m->nrow + i) * m->bw + b] =
              dev[((size_t)b * m->nrow + i) * m->ncol + col];
  });
}

int lfg_cma_assemble(lfg_cma m, lfg_lma a, const int* cb_to, const int* cb_from) {
  if (!m || !a) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(a->ctx == c && a->ncell == m->ncol, "cma_assemble: LMA and CMA cell counts differ");
    LFG_REQUIRE(cb_to && cb_from, "cma_assemble: null dofmap");
    const int grid = (m->ncol + 127) / 128;
    if (m->bw <= 8) {
      // row-parallel form; the row lists are rebuilt only when the dofmaps
      // differ from the last assembly's
      std::vector<int> key = {0, a->ndf_to, a->ndf_from, a->nl};
      key = with_map(with_map(std::move(key), cb_to, (size_t)a->ndf_to * a->nl), cb_from,
                     (size_t)a->ndf_from * a->nl);
      if (key != m->asm_key || !m->asm_rowptr) {
        DevInts dto, dfrom;  // validation of the dofmaps against the operator
        dto.p = checked_dofmap(cb_to, a->ndf_to, a->nl, m->nrow, "cma_assemble");
        dfrom.p = checked_dofmap(cb_from, a->ndf_from, a->nl, m->ncolumn, "cma_assemble");
        check_bands(m, cb_to, a->ndf_to, cb_from, a->ndf_from, a->nl, "cma_assemble");
        const auto jm = host_ints(m->jminus, m->nrow);
        cached_rows(m, std::move(key), [&](std::vector<std::vector<int2>>& rows) {
          for (int k = 0; k < a->nl; ++k)
            for (int d1 = 0; d1 < a->ndf_to; ++d1) {
              const int i = cb_to[k * a->ndf_to + d1] - 1;
              for (int d2 = 0; d2 < a->ndf_from; ++d2)
                rows[i].push_back(make_int2((d1 * a->ndf_from + d2) * a->nl + k,
                                            cb_from[k * a->ndf_from + d2] - 1 - jm[i]));
            }
        });
        LFG_CUDA(cudaStreamSynchronize(c->stream));  // the dofmap copies are freed on return
      }
      dispatch_kind(m->kind, [&](auto t) {
        using T = decltype(t);
        dispatch_kind(a->kind, [&](auto tl) {
          using TL = decltype(tl);
          auto go = [&](auto k) {
            const int gx = (m->ncol + 128 * kAsmColsPerThread - 1) / (128 * kAsmColsPerThread);
            launch_pdl(c, k, dim3(gx, m->nrow), dim3(128), 0, (T*)m->bands, m->ncol, m->nrow,
                       m->bw, (const TL*)a->a, m->asm_rowptr, (const int2*)m->asm_list);
          };
          if (m->bw <= 2) go(k_cma_asm_rows<T, TL, 2>);
          else if (m->bw <= 4) go(k_cma_asm_rows<T, TL, 4>);
          else go(k_cma_asm_rows<T, TL, 8>);
        });
      });
      // the element matrices read, every band written once
      after_launch(c, "cma_asm",
                   (uint64_t)a->kind * a->ncell * a->nl * a->ndf_to * a->ndf_from +
                       (uint64_t)m->kind * m->bw * m->nrow * m->ncol);
      m->fvalid = false;  // the bands changed
      return;
    }
    DevInts dto, dfrom;
    dto.p = checked_dofmap(cb_to, a->ndf_to, a->nl, m->nrow, "cma_assemble");
    dfrom.p = checked_dofmap(cb_from, a->ndf_from, a->nl, m->ncolumn, "cma_assemble");
    check_bands(m, cb_to, a->ndf_to, cb_from, a->ndf_from, a->nl, "cma_assemble");
    dispatch_kind(m->kind, [&](auto t) {
      using T = decltype(t);
      dispatch_kind(a->kind, [&](auto tl) {
        using TL = decltype(tl);
        k_cma_asm<T, TL><<<grid, 128, 0, c->stream>>>((T*)m->bands, m->jminus, m->ncol, m->nrow,
                                                      m->bw, (const TL*)a->a, a->ndf_to,
                                                      a->ndf_from, a->nl, dto.p, dfrom.p);
      });
    });
    after_launch(c, "cma_asm");
    m->fvalid = false;  // the bands changed
    LFG_CUDA(cudaStreamSynchronize(c->stream));  // the dofmap copies are freed on return
  });
}

int lfg_cma_multiply(lfg_cma C, lfg_cma A, lfg_cma B) {
  if (!C || !A || !B) return LFG_ERR_ARG;
  lfg_ctx c = C->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(A->ctx == c && B->ctx == c, "cma_multiply: operators of another context");
    LFG_REQUIRE(A->kind == C->kind && B->kind == C->kind, "cma_multiply: kinds differ");
    LFG_REQUIRE(A->ncol == C->ncol && B->ncol == C->ncol, "cma_multiply: cell counts differ");
    LFG_REQUIRE(A->nrow == C->nrow && A->ncolumn == B->nrow && B->ncolumn == C->ncolumn,
                "cma_multiply: shapes do not chain (C nrow x ncol = A nrow x B ncol)");
    // every product entry must have a slot in C's band; the widest spans of
    // A's and C's rows pick the kernel.  Both follow from the three shapes
    // (the band limits are functions of alpha, beta, gamma), so a product of
    // the same shapes as the last one skips the host check and stays
    // asynchronous.
    std::vector<int> key;
    for (lfg_cma m : {A, B, C})
      key.insert(key.end(), {m->nrow, m->ncolumn, m->bw, m->alpha, m->beta, m->gm, m->gp});
    int span_a = 0, span_c = 0;
    if (key == C->mul_key) {
      span_a = C->mul_span_a;
      span_c = C->mul_span_c;
    } else {
      const auto jmA = host_ints(A->jminus, A->nrow), jpA = host_ints(A->jplus, A->nrow);
      const auto jmB = host_ints(B->jminus, B->nrow), jpB = host_ints(B->jplus, B->nrow);
      const auto jmC = host_ints(C->jminus, C->nrow), jpC = host_ints(C->jplus, C->nrow);
      for (int i = 0; i < C->nrow; ++i) {
        LFG_REQUIRE(jpC[i] - jmC[i] + 1 <= C->bw, "cma_multiply: C band too narrow");
        span_a = std::max(span_a, std::min(A->ncolumn - 1, jpA[i]) - std::max(0, jmA[i]) + 1);
        span_c = std::max(span_c, std::min(C->ncolumn - 1, jpC[i]) - std::max(0, jmC[i]) + 1);
        for (int l = std::max(0, jmA[i]); l <= std::min(A->ncolumn - 1, jpA[i]); ++l)
          for (int j = std::max(jmB[l], std::max(0, jmC[i]));
               j <= std::min(jpB[l], std::min(C->ncolumn - 1, jpC[i])); ++j)
            LFG_REQUIRE(j - jmC[i] >= 0 && j - jmC[i] < C->bw, "cma_multiply: band overflow");
      }
      C->mul_key = key;
      C->mul_span_a = span_a;
      C->mul_span_c = span_c;
    }
    dim3 grid((C->ncol + 127) / 128, C->nrow);
    dispatch_kind(C->kind, [&](auto t) {
      using T = decltype(t);
      auto go = [&](auto k) {
        launch_pdl(c, k, grid, dim3(128), 0, (T*)C->bands, C->jminus, C->jplus, C->ncolumn,
                   (const T*)A->bands, A->jminus, A->jplus, A->ncolumn, (const T*)B->bands,
                   B->jminus, B->jplus, A->nrow, B->nrow, C->ncol);
      };
      if (span_a <= 2 && span_c <= 4) go(k_cma_mul_u<T, 2, 4>);
      else if (span_a <= 4 && span_c <= 8) go(k_cma_mul_u<T, 4, 8>);
      else
        k_cma_mul<T><<<grid, 128, 0, c->stream>>>(
            (T*)C->bands, C->jminus, C->jplus, C->ncolumn, C->bw, (const T*)A->bands, A->jminus,
            A->jplus, A->ncolumn, (const T*)B->bands, B->jminus, B->jplus, A->nrow, B->nrow,
            C->ncol);
    });
    after_launch(c, "cma_mul");
    C->fvalid = false;  // the bands changed
  });
}

int lfg_cma_scaled_add(lfg_cma C, lfg_cma A, lfg_cma B, double alpha, double beta) {
  if (!C || !A || !B) return LFG_ERR_ARG;
  lfg_ctx c = C->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(A->ctx == c && B->ctx == c, "cma_scaled_add: operators of another context");
    LFG_REQUIRE(A->kind == C->kind && B->kind == C->kind, "cma_scaled_add: kinds differ");
    LFG_REQUIRE(A->ncol == C->ncol && B->ncol == C->ncol, "cma_scaled_add: cell counts differ");
    LFG_REQUIRE(A->nrow <= C->nrow && A->nrow <= B->nrow,
                "cma_scaled_add: C and B need at least A's rows");
    {
      const auto jmA = host_ints(A->jminus, A->nrow), jpA = host_ints(A->jplus, A->nrow);
      const auto jmB = host_ints(B->jminus, B->nrow), jpB = host_ints(B->jplus, B->nrow);
      const auto jmC = host_ints(C->jminus, C->nrow);
      for (int i = 0; i < A->nrow; ++i) {
        for (int j = std::max(0, jmA[i]); j <= std::min(A->ncolumn - 1, jpA[i]); ++j)
          LFG_REQUIRE(j - jmC[i] >= 0 && j - jmC[i] < C->bw, "cma_scaled_add: A outside C's band");
        for (int j = std::max(0, jmB[i]); j <= std::min(A->ncolumn - 1, jpB[i]); ++j) {
          LFG_REQUIRE(j - jmC[i] >= 0 && j - jmC[i] < C->bw, "cma_scaled_add: B outside C's band");
          LFG_REQUIRE(j - jmB[i] < B->bw, "cma_scaled_add: B band too narrow");
        }
      }
    }
    dim3 grid((C->ncol + 127) / 128, C->nrow);
    dispatch_kind(C->kind, [&](auto t) {
      using T = decltype(t);
      k_cma_scaledadd<T><<<grid, 128, 0, c->stream>>>(
          (T*)C->bands, C->jminus, C->nrow, C->bw, (const T*)A->bands, A->jminus, A->jplus,
          A->nrow, A->ncolumn, (const T*)B->bands, B->jminus, B->jplus, B->nrow, C->ncol,
          (T)alpha, (T)beta);
    });
    after_launch(c, "cma_scaledadd");
    C->fvalid = false;  // the bands changed
  });
}

int lfg_cma_assemble_diag_hmht(lfg_cma m, lfg_lma dh, lfg_lma m2h, const int* cbm) {
  if (!m || !dh || !m2h) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(dh->ctx == c && m2h->ctx == c, "cma_assemble_diag_hmht: another context");
    LFG_REQUIRE(dh->ncell == m->ncol && m2h->ncell == m->ncol && dh->nl == m2h->nl,
                "cma_assemble_diag_hmht: cell or layer counts differ");
    LFG_REQUIRE(dh->ndf_from == m2h->ndf_to && m2h->ndf_to == m2h->ndf_from,
                "cma_assemble_diag_hmht: Dh must map W2h -> W3 and M2h be W2h x W2h");
    LFG_REQUIRE(dh->kind == m2h->kind, "cma_assemble_diag_hmht: LMA kinds differ");
    const int grid = (m->ncol + 127) / 128;
    if (m->bw <= 8 && dh->nl < (1 << 16) && dh->ndf_to < 128) {
      std::vector<int> key = {1, dh->ndf_to, dh->ndf_from, dh->nl};
      key = with_map(std::move(key), cbm, (size_t)dh->ndf_to * dh->nl);
      if (key != m->asm_key || !m->asm_rowptr) {
        DevInts d;
        d.p = checked_dofmap(cbm, dh->ndf_to, dh->nl, m->nrow, "cma_assemble_diag_hmht");
        check_bands(m, cbm, dh->ndf_to, cbm, dh->ndf_to, dh->nl, "cma_assemble_diag_hmht");
        const auto jm = host_ints(m->jminus, m->nrow);
        const int n3 = dh->ndf_to;
        cached_rows(m, std::move(key), [&](std::vector<std::vector<int2>>& rows) {
          for (int k = 0; k < dh->nl; ++k)
            for (int d1 = 0; d1 < n3; ++d1) {
              const int i = cbm[k * n3 + d1] - 1;
              for (int d2 = 0; d2 < n3; ++d2)
                rows[i].push_back(make_int2(k | d1 << 16 | d2 << 24, cbm[k * n3 + d2] - 1 - jm[i]));
            }
        });
        LFG_CUDA(cudaStreamSynchronize(c->stream));
      }
      dispatch_kind(m->kind, [&](auto t) {
        using T = decltype(t);
        dispatch_kind(dh->kind, [&](auto tl) {
          using TL = decltype(tl);
          auto go = [&](auto k) {
            launch_pdl(c, k, dim3(grid, m->nrow), dim3(128), 0, (T*)m->bands, m->ncol, m->nrow,
                       m->bw, (const TL*)dh->a, (const TL*)m2h->a, dh->ndf_from, dh->nl,
                       m->asm_rowptr, (const int2*)m->asm_list);
          };
          const int q = m->asm_maxq;
          const bool n4 = dh->ndf_from == 4;
          if (m->bw <= 2) {
            if (n4 && q <= 1) go(k_cma_hmht_rows<T, TL, 2, 1, 4>);
            else if (n4 && q <= 2) go(k_cma_hmht_rows<T, TL, 2, 2, 4>);
            else go(k_cma_hmht_rows<T, TL, 2, 0, 0>);
          } else if (m->bw <= 4) {
            if (n4 && q <= 4) go(k_cma_hmht_rows<T, TL, 4, 4, 4>);
            else go(k_cma_hmht_rows<T, TL, 4, 0, 0>);
          } else {
            go(k_cma_hmht_rows<T, TL, 8, 0, 0>);
          }
        });
      });
      after_launch(c, "cma_asm_diag_hmht");
      m->fvalid = false;
      return;
    }
    DevInts d;
    d.p = checked_dofmap(cbm, dh->ndf_to, dh->nl, m->nrow, "cma_assemble_diag_hmht");
    check_bands(m, cbm, dh->ndf_to, cbm, dh->ndf_to, dh->nl, "cma_assemble_diag_hmht");
    dispatch_kind(m->kind, [&](auto t) {
      using T = decltype(t);
      dispatch_kind(dh->kind, [&](auto tl) {
        using TL = decltype(tl);
        k_cma_asm_hmht<T, TL><<<grid, 128, 0, c->stream>>>(
            (T*)m->bands, m->jminus, m->ncol, m->nrow, m->bw, (const TL*)dh->a,
            (const TL*)m2h->a, dh->ndf_to, dh->ndf_from, dh->nl, d.p);
      });
    });
    after_launch(c, "cma_asm_diag_hmht");
    m->fvalid = false;  // the bands changed
    LFG_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int lfg_cma_assemble_m2v_lumped_inv(lfg_cma m, lfg_lma mm, const int* cbm) {
  if (!m || !mm) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(mm->ctx == c && mm->ncell == m->ncol && mm->ndf_to == mm->ndf_from,
                "cma_assemble_m2v_lumped_inv: LMA must be square with the CMA's cells");
    const int grid = (m->ncol + 127) / 128;
    if (m->bw <= 8) {
      std::vector<int> key = {2, mm->ndf_to, mm->nl};
      key = with_map(std::move(key), cbm, (size_t)mm->ndf_to * mm->nl);
      if (key != m->asm_key || !m->asm_rowptr) {
        DevInts d;
        d.p = checked_dofmap(cbm, mm->ndf_to, mm->nl, m->nrow, "cma_assemble_m2v_lumped_inv");
        const int nd = mm->ndf_to;
        cached_rows(m, std::move(key), [&](std::vector<std::vector<int2>>& rows) {
          for (int k = 0; k < mm->nl; ++k)
            for (int dd = 0; dd < nd; ++dd)
              rows[cbm[k * nd + dd] - 1].push_back(make_int2((dd * nd + dd) * mm->nl + k, 0));
        });
        LFG_CUDA(cudaStreamSynchronize(c->stream));
      }
      dispatch_kind(m->kind, [&](auto t) {
        using T = decltype(t);
        dispatch_kind(mm->kind, [&](auto tl) {
          using TL = decltype(tl);
          auto go = [&](auto k) {
            const int gx = (m->ncol + 128 * kAsmColsPerThread - 1) / (128 * kAsmColsPerThread);
            launch_pdl(c, k, dim3(gx, m->nrow), dim3(128), 0, (T*)m->bands, m->ncol, m->nrow,
                       m->bw, (const TL*)mm->a, m->asm_rowptr, (const int2*)m->asm_list);
          };
          if (m->bw <= 2) go(k_cma_asm_rows<T, TL, 2, true>);
          else if (m->bw <= 4) go(k_cma_asm_rows<T, TL, 4, true>);
          else go(k_cma_asm_rows<T, TL, 8, true>);
        });
      });
      after_launch(c, "cma_asm_m2v_lumped_inv");
      m->fvalid = false;
      return;
    }
    DevInts d;
    d.p = checked_dofmap(cbm, mm->ndf_to, mm->nl, m->nrow, "cma_assemble_m2v_lumped_inv");
    dispatch_kind(m->kind, [&](auto t) {
      using T = decltype(t);
      dispatch_kind(mm->kind, [&](auto tl) {
        using TL = decltype(tl);
        k_cma_asm_m2v<T, TL><<<grid, 128, 0, c->stream>>>((T*)m->bands, m->ncol, m->nrow, m->bw,
                                                          (const TL*)mm->a, mm->ndf_to, mm->nl,
                                                          d.p);
      });
    });
    after_launch(c, "cma_asm_m2v_lumped_inv");
    m->fvalid = false;  // the bands changed
    LFG_CUDA(cudaStreamSynchronize(c->stream));
  });
}

}  // extern "C"

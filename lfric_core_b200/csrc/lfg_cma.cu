// Columnwise-assembled (CMA) operators, the Thomas column solves and the
// intergrid transfers.
//
// Drop-ins for the reference kernels (components/science/source/kernel/):
//   columnwise_operators/sci_columnwise_op_app_kernel_mod.F90:73-124     (lfg_cma_apply)
//   columnwise_operators/sci_columnwise_op_appinv_kernel_mod.F90:77-145  (lfg_cma_apply_inverse)
//   solver/sci_tri_solve_kernel_mod.f90:116-156                          (lfg_tri_solve)
//   solver/sci_operator_tri_solve_kernel_mod.f90:69-120                  (lfg_operator_tri_solve)
//   inter_mesh/sci_restrict_scalar_{unweighted,weighted}_kernel_mod.F90,
//   inter_mesh/sci_restrict_mass_w3_kernel_mod.F90,
//   inter_mesh/sci_prolong_scalar_{unweighted,weighted}_kernel_mod.F90,
//   inter_mesh/sci_restrict_w0_kernel_mod.F90, sci_prolong_w0_kernel_mod.F90.
// The reference calls each once per column from the PSy layer; here one
// launch covers the mesh.  The banded apply and the intergrid transfers
// give a thread one (column, row) or (column, block of levels); the line
// solves give a thread one column, or, for FP64 columns of 13-96 rows, one
// segment of a column (k_cma_subst_seg).
#include "lfg_internal.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>

using namespace lfg;

namespace {

// ------------------------------------------------------------- Thomas
// Source of the tridiagonal rows and of the right-hand side of one column.
enum { SRC_CMA = 0, SRC_FIELDS = 1, SRC_LMA2 = 2 };

template <class T>
struct TriSrc {
  int ncol, nrow;
  const T* __restrict__ bands;  // CMA [3][nrow][ncol]; LMA2 [2][2][nl][ncol]
  const T* __restrict__ t0;     // fields: tri_0, tri_plus, tri_minus [nrow][ncol]
  const T* __restrict__ tp;
  const T* __restrict__ tm;
  const int* __restrict__ ind;  // CMA: 0-based dof offset of each row
  int nl;                       // LMA2: number of layers (nrow = nl + 1)
};

template <class T, int SRC>
__device__ __forceinline__ void tri_row(const TriSrc<T>& s, int k, int c, T& a1, T& a2, T& a3) {
  const size_t N = s.ncol;
  if (SRC == SRC_CMA) {
    const size_t plane = (size_t)s.nrow * N;
    a1 = s.bands[(size_t)k * N + c];
    a2 = s.bands[plane + (size_t)k * N + c];
    a3 = s.bands[2 * plane + (size_t)k * N + c];
  } else if (SRC == SRC_FIELDS) {
    a1 = s.tm[(size_t)k * N + c];
    a2 = s.t0[(size_t)k * N + c];
    a3 = s.tp[(size_t)k * N + c];
  } else {
    // 2x2 LMA M(layer, i, j) at bands[((i*2+j)*nl + layer)*N + c]
    const size_t lay = (size_t)s.nl * N;
    const T m11 = k < s.nl ? s.bands[0 * lay + (size_t)k * N + c] : (T)0;
    const T m22 = k > 0 ? s.bands[3 * lay + (size_t)(k - 1) * N + c] : (T)0;
    a2 = m11 + m22;
    a3 = k < s.nl ? s.bands[1 * lay + (size_t)k * N + c] : (T)0;
    a1 = k > 0 ? s.bands[2 * lay + (size_t)(k - 1) * N + c] : (T)0;
  }
}

template <class T, int SRC>
__device__ __forceinline__ size_t tri_dof(const TriSrc<T>& s, int k) {
  return SRC == SRC_CMA ? (size_t)s.ind[k] : (size_t)k;
}

// lhs = A^{-1} x, one thread per column; c' in shared memory, d' in
// registers (unrolled level loop).
template <class T, int SRC, int MAXNL>
__global__ void k_thomas(TriSrc<T> s, const T* __restrict__ x, T* __restrict__ lhs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* cps = reinterpret_cast<T*>(smem_raw);
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= s.ncol) return;
  const size_t N = s.ncol;
  const int nrow = s.nrow, t = threadIdx.x, bs = blockDim.x;
  T dp[MAXNL];
  T cprev = (T)0, dprev = (T)0;
#pragma unroll
  for (int k = 0; k < MAXNL; ++k) {
    if (k < nrow) {
      T a1, a2, a3;
      tri_row<T, SRC>(s, k, c, a1, a2, a3);
      const T xv = x[tri_dof<T, SRC>(s, k) * N + c];
      T inv, cpk, dpk;
      if (k == 0) {
        inv = (T)1 / a2;
        cpk = inv * a3;
        dpk = inv * xv;
      } else {
        inv = (T)1 / (a2 - a1 * cprev);
        cpk = (k < nrow - 1) ? inv * a3 : (T)0;
        dpk = inv * (xv - a1 * dprev);
      }
      cps[k * bs + t] = cpk;
      dp[k] = dpk;
      cprev = cpk;
      dprev = dpk;
    }
  }
  T znext = (T)0;
#pragma unroll
  for (int k = MAXNL - 1; k >= 0; --k) {
    if (k < nrow) {
      T z = dp[k];
      if (k < nrow - 1) z = z - cps[k * bs + t] * znext;
      znext = z;
      lhs[tri_dof<T, SRC>(s, k) * N + c] = z;
    }
  }
}

// Same algorithm for columns taller than the unrolled variants: c' and d'
// live in a global scratch array of 2*nrow*ncol values.
template <class T, int SRC>
__global__ void k_thomas_scratch(TriSrc<T> s, const T* __restrict__ x, T* __restrict__ lhs,
                                 T* __restrict__ scratch) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= s.ncol) return;
  const size_t N = s.ncol;
  const int nrow = s.nrow;
  T* cp = scratch;
  T* dp = scratch + (size_t)nrow * N;
  T cprev = (T)0, dprev = (T)0;
  for (int k = 0; k < nrow; ++k) {
    T a1, a2, a3;
    tri_row<T, SRC>(s, k, c, a1, a2, a3);
    const T xv = x[tri_dof<T, SRC>(s, k) * N + c];
    T inv, cpk, dpk;
    if (k == 0) {
      inv = (T)1 / a2;
      cpk = inv * a3;
      dpk = inv * xv;
    } else {
      inv = (T)1 / (a2 - a1 * cprev);
      cpk = (k < nrow - 1) ? inv * a3 : (T)0;
      dpk = inv * (xv - a1 * dprev);
    }
    cp[(size_t)k * N + c] = cpk;
    dp[(size_t)k * N + c] = dpk;
    cprev = cpk;
    dprev = dpk;
  }
  T znext = (T)0;
  for (int k = nrow - 1; k >= 0; --k) {
    T z = dp[(size_t)k * N + c];
    if (k < nrow - 1) z = z - cp[(size_t)k * N + c] * znext;
    znext = z;
    lhs[tri_dof<T, SRC>(s, k) * N + c] = z;
  }
}

// Thomas factors of a CMA tridiagonal, one thread per column, in the
// reference's arithmetic (sci_columnwise_op_appinv_kernel_mod.F90:77-145):
// inv_1 = 1/a2, inv_i = 1/(a2 - a1 c'_{i-1}); c'_i = inv_i a3 (not on the
// last row).  They depend on the matrix alone.
template <class T>
__global__ void k_cma_factor(const T* __restrict__ bands, int ncol, int nrow, T* __restrict__ finv,
                             T* __restrict__ fcp) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  const size_t N = ncol, plane = (size_t)nrow * N;
  T cprev = (T)0;
  for (int k = 0; k < nrow; ++k) {
    const size_t i = (size_t)k * N + c;
    const T a1 = bands[i], a2 = bands[plane + i], a3 = bands[2 * plane + i];
    const T inv = k == 0 ? (T)1 / a2 : (T)1 / (a2 - a1 * cprev);
    const T cp = (k == 0 || k < nrow - 1) ? inv * a3 : (T)0;
    finv[i] = inv;
    fcp[i] = cp;
    cprev = cp;
  }
}

// lhs = A^{-1} x on the precomputed factors: d'_k = inv_k (x_k - a1_k d'_{k-1}),
// z_k = d'_k - c'_k z_{k+1}, x and lhs at the rows' dof offsets.  One
// thread per column, d' in shared memory; each sweep walks the column in
// blocks of CSP levels and loads block b+1 before it computes block b.
constexpr int CSP = 8;
template <class T>
__global__ void __launch_bounds__(128) k_cma_subst(const T* __restrict__ bands,
                                                   const T* __restrict__ finv,
                                                   const T* __restrict__ fcp,
                                                   const int* __restrict__ ind, int ncol,
                                                   int nrow, const T* __restrict__ x,
                                                   T* __restrict__ lhs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sd = reinterpret_cast<T*>(smem_raw);  // [nrow][blockDim]
  const int t = threadIdx.x, bs = blockDim.x;
  const int c = blockIdx.x * bs + t;
  if (c >= ncol) return;
  const size_t N = ncol;
  const int nb = (nrow + CSP - 1) / CSP;
  auto lv = [&](int k) { return min(max(k, 0), nrow - 1); };
  T ax[CSP], ai[CSP], as[CSP], bx[CSP], bi[CSP], bsb[CSP];
#pragma unroll
  for (int p = 0; p < CSP; ++p) {
    const int k = lv(p);
    ax[p] = x[(size_t)ind[k] * N + c];
    ai[p] = finv[(size_t)k * N + c];
    as[p] = bands[(size_t)k * N + c];
  }
  T d = (T)0;
  for (int blk = 0; blk < nb; ++blk) {
    const int k0 = blk * CSP;
#pragma unroll
    for (int p = 0; p < CSP; ++p) {
      const int k = lv(k0 + CSP + p);
      bx[p] = x[(size_t)ind[k] * N + c];
      bi[p] = finv[(size_t)k * N + c];
      bsb[p] = bands[(size_t)k * N + c];
    }
#pragma unroll
    for (int p = 0; p < CSP; ++p) {
      const int k = k0 + p;
      const T dn = k == 0 ? ai[p] * ax[p] : ai[p] * (ax[p] - as[p] * d);
      if (k < nrow) {
        d = dn;
        sd[k * bs + t] = d;
      }
    }
#pragma unroll
    for (int p = 0; p < CSP; ++p) {
      ax[p] = bx[p];
      ai[p] = bi[p];
      as[p] = bsb[p];
    }
  }
  T ac[CSP], bc[CSP];
  const int ktop = nrow - 1;
#pragma unroll
  for (int p = 0; p < CSP; ++p) ac[p] = fcp[(size_t)lv(ktop - p) * N + c];
  T z = (T)0;
  for (int blk = 0; blk < nb; ++blk) {
    const int k0 = ktop - blk * CSP;
#pragma unroll
    for (int p = 0; p < CSP; ++p) bc[p] = fcp[(size_t)lv(k0 - CSP - p) * N + c];
#pragma unroll
    for (int p = 0; p < CSP; ++p) {
      const int k = k0 - p;
      if (k >= 0) {
        const T dk = sd[k * bs + t];
        z = k == ktop ? dk : dk - ac[p] * z;
        lhs[(size_t)ind[k] * N + c] = z;
      }
    }
#pragma unroll
    for (int p = 0; p < CSP; ++p) ac[p] = bc[p];
  }
}

// The same substitutions with S warps per 32 columns: warp j of a block
// owns rows [j*L, j*L + L), L = ceil(nrow/S) <= kCmaSeg, of the block's 32
// columns (one column per lane, so every row is one coalesced 32-column
// load) and loads them all at once.  Each thread composes its rows' affine
// maps (forward d_out = D + M d_in, backward z_in = E + Nn z_out); through
// shared memory every segment then applies the maps of the segments before
// it (after it, backward) to find its incoming value, and computes its rows
// with the per-row formulas of k_cma_subst.  Only the value that enters a
// segment is formed through the maps, a rounding-level difference.
constexpr int kCmaSeg = 12;
template <class T, int S>
__global__ void __launch_bounds__(32 * S) k_cma_subst_seg(const T* __restrict__ bands,
                                                          const T* __restrict__ finv,
                                                          const T* __restrict__ fcp,
                                                          const int* __restrict__ ind, int ncol,
                                                          int nrow, const T* __restrict__ x,
                                                          T* __restrict__ lhs) {
  __shared__ T sa[S][32], sm[S][32];
  const int lane = threadIdx.x & 31, j = threadIdx.x >> 5;
  const unsigned c = blockIdx.x * 32u + lane;
  const size_t N = ncol;
  const int L = (nrow + S - 1) / S, k0 = j * L;
  const int nmy = c < N ? max(0, min(L, nrow - k0)) : 0;
  T d[kCmaSeg], iv[kCmaSeg], sb[kCmaSeg], cc[kCmaSeg];
#pragma unroll
  for (int u = 0; u < kCmaSeg; ++u)
    if (u < nmy) {
      const size_t i = (size_t)(k0 + u) * N + c;
      d[u] = x[(size_t)ind[k0 + u] * N + c];
      iv[u] = finv[i];
      sb[u] = bands[i];
      cc[u] = fcp[i];
    }
  T D = (T)0, M = (T)1;
#pragma unroll
  for (int u = 0; u < kCmaSeg; ++u)
    if (u < nmy) {
      D = (d[u] - sb[u] * D) * iv[u];
      M = M * (-sb[u] * iv[u]);
    }
  sa[j][lane] = D;
  sm[j][lane] = M;
  __syncthreads();
  T dv = (T)0;
  for (int q = 0; q < j; ++q) dv = sa[q][lane] + sm[q][lane] * dv;
#pragma unroll
  for (int u = 0; u < kCmaSeg; ++u)
    if (u < nmy) {
      dv = k0 + u == 0 ? iv[u] * d[u] : iv[u] * (d[u] - sb[u] * dv);
      d[u] = dv;
    }
  T E = (T)0, Nn = (T)1;
#pragma unroll
  for (int u = kCmaSeg - 1; u >= 0; --u)
    if (u < nmy) {
      E = d[u] - cc[u] * E;
      Nn = Nn * (-cc[u]);
    }
  __syncthreads();
  sa[j][lane] = E;
  sm[j][lane] = Nn;
  __syncthreads();
  T z = (T)0;
  for (int q = S - 1; q > j; --q) z = sa[q][lane] + sm[q][lane] * z;
#pragma unroll
  for (int u = kCmaSeg - 1; u >= 0; --u)
    if (u < nmy) {
      const int k = k0 + u;
      z = k == nrow - 1 ? d[u] : d[u] - cc[u] * z;
      lhs[(size_t)ind[k] * N + c] = z;
    }
}

// warps per 32 columns for k_cma_subst_seg: the fewest (2, 4 or 8) that
// cut the column into segments of at most kCmaSeg rows; 0 for columns of
// at most kCmaSeg rows (one thread holds them) or taller than 8 * kCmaSeg
int cma_seg_lanes(int nrow) {
  if (nrow <= kCmaSeg) return 0;
  for (int S = 2; S <= 8; S *= 2)
    if ((nrow + S - 1) / S <= kCmaSeg) return S;
  return 0;
}

int col_block(int ncol, int nsm) {
  int per = (ncol + nsm - 1) / nsm;
  int bs = ((per + 31) / 32) * 32;
  return std::max(32, std::min(128, bs));
}

template <class T, int SRC, int MAXNL>
void launch_thomas_t(lfg_ctx c, const TriSrc<T>& s, const T* x, T* lhs) {
  const int bs = col_block(s.ncol, c->num_sms);
  const size_t smem = (size_t)MAXNL * bs * sizeof(T);
  auto kern = k_thomas<T, SRC, MAXNL>;
  ensure_smem_attr((const void*)kern, (int)(MAXNL * 128 * sizeof(T)));
  kern<<<(s.ncol + bs - 1) / bs, bs, smem, c->stream>>>(s, x, lhs);
  // three bands and x read, the solution written
  after_launch(c, "thomas", sizeof(T) * 5 * (uint64_t)s.nrow * s.ncol);
}

template <class T, int SRC>
void launch_thomas(lfg_ctx c, const TriSrc<T>& s, const T* x, T* lhs) {
  if (s.nrow <= 16) launch_thomas_t<T, SRC, 16>(c, s, x, lhs);
  else if (s.nrow <= 32) launch_thomas_t<T, SRC, 32>(c, s, x, lhs);
  else if (s.nrow <= 72) launch_thomas_t<T, SRC, 72>(c, s, x, lhs);
  else {
    T* scratch = (T*)c->scratch(2 * (size_t)s.nrow * s.ncol * sizeof(T));
    const int bs = 128;
    k_thomas_scratch<T, SRC><<<(s.ncol + bs - 1) / bs, bs, 0, c->stream>>>(s, x, lhs, scratch);
    after_launch(c, "thomas_scratch", sizeof(T) * 5 * (uint64_t)s.nrow * s.ncol);
  }
}

// ------------------------------------------------------------- CMA apply
// lhs(ind_to(i)) += sum_j band(j - j_minus(i), i) x(ind_from(j)), one thread
// per (row, column); rows of one column are distinct dofs.
template <class T>
__global__ void k_cma_app(const T* __restrict__ bands, const int* __restrict__ ind_to,
                          const int* __restrict__ ind_from, const int* __restrict__ jminus,
                          const int* __restrict__ jplus, int ncol, int nrow, int ncolumn,
                          const T* __restrict__ x, T* __restrict__ lhs) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (c >= ncol) return;
  const size_t N = ncol, plane = (size_t)nrow * N;
  const int jm = jminus[i];
  const int jlo = max(0, jm), jhi = min(ncolumn - 1, jplus[i]);
  const size_t o = (size_t)ind_to[i] * N + c;
  T acc = lhs[o];
  for (int j = jlo; j <= jhi; ++j)
    acc = acc + bands[(size_t)(j - jm) * plane + (size_t)i * N + c] * x[(size_t)ind_from[j] * N + c];
  lhs[o] = acc;
}

// The same with V adjacent columns per thread (16-byte loads and stores of
// the bands, x and lhs), for fields whose rows start on 16-byte boundaries;
// the same operations in the same order as k_cma_app.
// TRI: the W3 -> W3 tridiagonal with identity row and column maps
// (alpha = beta = gamma_m = gamma_p = 1, bandwidth 3), whose band columns
// i-1, i, i+1 and rows follow from i without reading the index maps.
template <class T, int V, bool TRI>
__global__ void k_cma_app_v(const T* __restrict__ bands, const int* __restrict__ ind_to,
                            const int* __restrict__ ind_from, const int* __restrict__ jminus,
                            const int* __restrict__ jplus, int ncol, int nrow, int ncolumn,
                            const T* __restrict__ x, T* __restrict__ lhs) {
  const int c = (blockIdx.x * blockDim.x + threadIdx.x) * V;
  const int i = blockIdx.y;
  if (c >= ncol) return;
  const size_t N = ncol, plane = (size_t)nrow * N;
  const int jm = TRI ? i - 1 : jminus[i];
  const int jlo = max(0, jm), jhi = min(ncolumn - 1, TRI ? i + 1 : jplus[i]);
  const size_t o = (size_t)(TRI ? i : ind_to[i]) * N + c;
  Vec<T, V> acc = vld<false, T, V>(lhs + o);
  for (int j = jlo; j <= jhi; ++j) {
    const Vec<T, V> a = vld<true, T, V>(bands + (size_t)(j - jm) * plane + (size_t)i * N + c);
    const Vec<T, V> xv = vld<false, T, V>(x + (size_t)(TRI ? j : ind_from[j]) * N + c);
#pragma unroll
    for (int v = 0; v < V; ++v) acc.e[v] = acc.e[v] + a.e[v] * xv.e[v];
  }
  vst<T, V>(lhs + o, acc);
}

// lhs(ind_from(j)) += sum over rows i whose band reaches column j of
// band(j - j_minus(i), i) x(ind_to(i)): the transpose of k_cma_app.  The
// rows reaching each column are listed per column (CSR, rows ascending).
template <class T>
__global__ void k_cma_app_t(const T* __restrict__ bands, const int* __restrict__ ind_to,
                            const int* __restrict__ ind_from, const int* __restrict__ jminus,
                            const int* __restrict__ tptr, const int* __restrict__ trow,
                            int ncol, int nrow, const T* __restrict__ x, T* __restrict__ lhs) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (c >= ncol) return;
  const size_t N = ncol, plane = (size_t)nrow * N;
  const size_t o = (size_t)ind_from[j] * N + c;
  T acc = lhs[o];
  for (int q = tptr[j]; q < tptr[j + 1]; ++q) {
    const int i = trow[q];
    acc = acc + bands[(size_t)(j - jminus[i]) * plane + (size_t)i * N + c] *
                    x[(size_t)ind_to[i] * N + c];
  }
  lhs[o] = acc;
}

// ------------------------------------------------------------- intergrid
// coarse(C,k) from the fine children, y outer and x inner (slot q = y*nx+x).
template <class T, int MODE>
__global__ void k_restrict(T* __restrict__ coarse, const T* __restrict__ fine,
                           const T* __restrict__ w, const int* __restrict__ child, int ncoarse,
                           int nfine, int nq, int nlev) {
  const int C = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (C >= ncoarse || k >= nlev) return;
  const T denom = (T)1 / (T)nq;
  T acc = (T)0;
  for (int q = 0; q < nq; ++q) {
    const size_t i = (size_t)k * nfine + child[(size_t)q * ncoarse + C];
    if (MODE == LFG_RESTRICT_UNWEIGHTED) acc = acc + fine[i] * denom;
    else if (MODE == LFG_RESTRICT_WEIGHTED) acc = acc + fine[i] * denom / w[i];
    else acc = acc + fine[i];
  }
  coarse[(size_t)k * ncoarse + C] = acc;
}

// fine(c,k) (+)= [w(c,k)] coarse(parent(c),k): one thread per (column,
// block of KI levels), columns fastest, grid-stride; the parent index is
// read once per block and the block's loads all issue before its stores.
constexpr int KI = 4;

template <class T, bool WEIGHTED>
__global__ void k_prolong(T* __restrict__ fine, const T* __restrict__ coarse,
                          const T* __restrict__ w, const int* __restrict__ parent, int nfine,
                          int ncoarse, int nlev) {
  const size_t nblk = (size_t)nfine * ((nlev + KI - 1) / KI);
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nblk;
       t += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(t % nfine), k0 = (int)(t / nfine) * KI;
    const int p = parent[c];
    T cv[KI], fv[KI], wv[KI];
#pragma unroll
    for (int kk = 0; kk < KI; ++kk)
      if (k0 + kk < nlev) {
        const size_t i = (size_t)(k0 + kk) * nfine + c;
        cv[kk] = coarse[(size_t)(k0 + kk) * ncoarse + p];
        fv[kk] = fine[i];
        if (WEIGHTED) wv[kk] = w[i];
      }
#pragma unroll
    for (int kk = 0; kk < KI; ++kk)
      if (k0 + kk < nlev)
        fine[(size_t)(k0 + kk) * nfine + c] = WEIGHTED ? fv[kk] + wv[kk] * cv[kk] : fv[kk] + cv[kk];
  }
}

// W0 injection: coarse vertex v takes the value of the coinciding fine vertex.
template <class T>
__global__ void k_restrict_w0(T* __restrict__ coarse, const T* __restrict__ fine,
                              const int* __restrict__ inj, int nvc, int nvf, int nlev) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (v >= nvc || k >= nlev) return;
  coarse[(size_t)k * nvc + v] = fine[(size_t)k * nvf + inj[v]];
}

// W0 bilinear prolongation: every fine vertex takes the value of the last
// write the reference loop would make to it (coarse cell, four weights).
template <class T>
__global__ void k_prolong_w0(T* __restrict__ fine, const T* __restrict__ coarse,
                             const int* __restrict__ src_cell, const double* __restrict__ wts,
                             const int* __restrict__ ccorner, int nvf, int nvc, int ncoarse,
                             int nlev) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (v >= nvf || k >= nlev) return;
  const int C = src_cell[v];
  if (C < 0) return;
  const size_t ko = (size_t)k * nvc;
  // weights stored NE, SE, SW, NW with a term count; corners SW,SE,NE,NW
  const double* w = wts + (size_t)v * 5;
  const int nterm = (int)w[4];
  const T cne = coarse[ko + ccorner[2 * ncoarse + C]];
  const T cse = coarse[ko + ccorner[1 * ncoarse + C]];
  const T csw = coarse[ko + ccorner[0 * ncoarse + C]];
  const T cnw = coarse[ko + ccorner[3 * ncoarse + C]];
  T val;
  if (nterm == 4) val = (T)w[0] * cne + (T)w[1] * cse + (T)w[2] * csw + (T)w[3] * cnw;
  else if (nterm == 2) val = (T)w[0] * cne + (T)w[1] * cse;          // SE dof, last column
  else if (nterm == 3) val = (T)w[0] * cne + (T)w[3] * cnw;          // NW dof, first row
  else val = cne;                                                    // NE dof
  fine[(size_t)k * nvf + v] = val;
}

template <class F>
void dispatch(int kind, F&& f) {
  if (kind == LFG_R_DOUBLE) f(double{});
  else f(float{});
}

// Working storage of lfg_tri_solve_noalloc: c' and d' of every column.  In
// host code this name only stands for the array; the kernel is given the
// device address looked up with cudaGetSymbolAddress.
__device__ __align__(256) unsigned char g_noalloc_scratch[LFG_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
std::vector<void*> g_noalloc_addr;  // per device ordinal, null until looked up

// The array's device address on device `dev` (the current device), looked
// up once.  The lookup and cudaFuncGetAttributes on both kernels make the
// runtime load this library's device code on that device (lazy module
// loading), which may allocate: lfg_ctx_create does it, so a caller that
// made a context on the device never pays it inside lfg_tri_solve_noalloc.
cudaError_t noalloc_lookup(int dev, void** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if ((int)g_noalloc_addr.size() <= dev) g_noalloc_addr.resize(dev + 1, nullptr);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    if (!p) return cudaErrorInvalidSymbol;
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, (const void*)k_thomas_scratch<double, SRC_FIELDS>);
    if (e == cudaSuccess)
      e = cudaFuncGetAttributes(&fa, (const void*)k_thomas_scratch<float, SRC_FIELDS>);
    if (e != cudaSuccess) return e;
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return cudaSuccess;
}

}  // namespace

namespace lfg {
cudaError_t noalloc_prepare(int dev) {
  void* p = nullptr;
  return noalloc_lookup(dev, &p);
}
}  // namespace lfg

extern "C" {

int lfg_tri_solve_noalloc(int kind, int ncol, int nlev, const void* x, const void* tri_0,
                          const void* tri_plus, const void* tri_minus, void* y,
                          void* stream) {
  if ((kind != LFG_R_DOUBLE && kind != LFG_R_SINGLE) || ncol <= 0 || nlev <= 0 || !x ||
      !tri_0 || !tri_plus || !tri_minus || !y)
    return LFG_ERR_ARG;
  if ((size_t)2 * nlev * ncol * kind > (size_t)LFG_NOALLOC_SCRATCH_BYTES) return LFG_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return LFG_ERR_CUDA;
  void* scratch = nullptr;
  if (noalloc_lookup(dev, &scratch) != cudaSuccess) return LFG_ERR_CUDA;
  const int bs = 128, grid = (ncol + bs - 1) / bs;
  cudaStream_t st = (cudaStream_t)stream;
  // launched through cudaLaunchKernel so that the status returned is this
  // launch's own, and no error left by the caller's earlier work is cleared
  cudaError_t e;
  if (kind == LFG_R_DOUBLE) {
    TriSrc<double> s{ncol, nlev, nullptr, (const double*)tri_0, (const double*)tri_plus,
                     (const double*)tri_minus, nullptr, 0};
    const double* xd = (const double*)x;
    double* yd = (double*)y;
    double* wd = (double*)scratch;
    void* args[] = {&s, &xd, &yd, &wd};
    e = cudaLaunchKernel((const void*)k_thomas_scratch<double, SRC_FIELDS>, dim3(grid),
                         dim3(bs), args, 0, st);
  } else {
    TriSrc<float> s{ncol, nlev, nullptr, (const float*)tri_0, (const float*)tri_plus,
                    (const float*)tri_minus, nullptr, 0};
    const float* xf = (const float*)x;
    float* yf = (float*)y;
    float* wf = (float*)scratch;
    void* args[] = {&s, &xf, &yf, &wf};
    e = cudaLaunchKernel((const void*)k_thomas_scratch<float, SRC_FIELDS>, dim3(grid), dim3(bs),
                         args, 0, st);
  }
  return e == cudaSuccess ? LFG_OK : LFG_ERR_CUDA;
}

// ------------------------------------------------------------- CMA objects
int lfg_cma_create(lfg_ctx c, int kind, int ncol, int nrow, int ncolumn, int bw, int alpha,
                   int beta, int gamma_m, int gamma_p, const int* ind_to, const int* ind_from,
                   const double* cm, lfg_cma* out) {
  if (!c || !out) return LFG_ERR_ARG;
  return guard(c, [&] {
    LFG_REQUIRE(kind == LFG_R_DOUBLE || kind == LFG_R_SINGLE, "cma_create: bad kind");
    LFG_REQUIRE(ncol > 0 && nrow > 0 && ncolumn > 0 && bw > 0 && beta > 0 && ind_to &&
                    ind_from,
                "cma_create: bad arguments");
    std::vector<int> it(nrow), iff(ncolumn), jm(nrow), jp(nrow);
    for (int i = 0; i < nrow; ++i) {
      LFG_REQUIRE(ind_to[i] >= 1, "cma_create: indirection maps are 1-based");
      it[i] = ind_to[i] - 1;
      // j_minus = ceiling((alpha*i - gamma_p)/beta) for the 1-based row i
      const int row = i + 1;
      const double q = (double)(alpha * row - gamma_p) / (double)beta;
      jm[i] = (int)std::ceil(q) - 1;  // 0-based first column of the band
      // j_plus = floor((alpha*i + gamma_m)/beta)
      jp[i] = (int)std::floor((double)(alpha * row + gamma_m) / (double)beta) - 1;
      LFG_REQUIRE(jp[i] - jm[i] + 1 <= bw, "cma_create: bandwidth too small for alpha/beta/gamma");
    }
    for (int j = 0; j < ncolumn; ++j) {
      LFG_REQUIRE(ind_from[j] >= 1, "cma_create: indirection maps are 1-based");
      iff[j] = ind_from[j] - 1;
    }
    int max_to = 0, max_from = 0;
    for (int i = 0; i < nrow; ++i) max_to = std::max(max_to, ind_to[i]);
    for (int j = 0; j < ncolumn; ++j) max_from = std::max(max_from, ind_from[j]);
    lfg_cma m = new lfg_cma_s;
    m->ctx = c;
    m->kind = kind;
    m->ncol = ncol;
    m->nrow = nrow;
    m->ncolumn = ncolumn;
    m->bw = bw;
    m->alpha = alpha;
    m->beta = beta;
    m->gm = gamma_m;
    m->gp = gamma_p;
    m->max_ind_to = max_to;
    m->max_ind_from = max_from;
    m->ind_identity = true;
    for (int i = 0; i < nrow; ++i) m->ind_identity &= ind_to[i] == i + 1;
    m->ind_from_identity = true;
    for (int j = 0; j < ncolumn; ++j) m->ind_from_identity &= ind_from[j] == j + 1;
    const size_t n = (size_t)bw * nrow * ncol;
    std::vector<double> dev(n);
    for (int col = 0; col < ncol; ++col)
      for (int i = 0; i < nrow; ++i)
        for (int b = 0; b < bw; ++b)
          dev[((size_t)b * nrow + i) * ncol + col] = cm ? cm[((size_t)col * nrow + i) * bw + b] : 0.0;
    try {
      m->bands = dmalloc(n * kind);
      if (kind == LFG_R_DOUBLE) upload(m->bands, dev.data(), n * sizeof(double));
      else {
        std::vector<float> f(dev.begin(), dev.end());
        upload(m->bands, f.data(), n * sizeof(float));
      }
      m->ind_to = (int*)dmalloc(nrow * sizeof(int));
      m->ind_from = (int*)dmalloc(ncolumn * sizeof(int));
      m->jminus = (int*)dmalloc(nrow * sizeof(int));
      m->jplus = (int*)dmalloc(nrow * sizeof(int));
      upload(m->jplus, jp.data(), nrow * sizeof(int));
      // rows reaching each column, for the transposed apply
      std::vector<int> tptr(ncolumn + 1, 0), trow;
      for (int j = 0; j < ncolumn; ++j) {
        for (int i = 0; i < nrow; ++i)
          if (j >= std::max(0, jm[i]) && j <= std::min(ncolumn - 1, jp[i])) trow.push_back(i);
        tptr[j + 1] = (int)trow.size();
      }
      m->tptr = (int*)dmalloc(tptr.size() * sizeof(int));
      m->trow = (int*)dmalloc(std::max<size_t>(1, trow.size()) * sizeof(int));
      upload(m->tptr, tptr.data(), tptr.size() * sizeof(int));
      if (!trow.empty()) upload(m->trow, trow.data(), trow.size() * sizeof(int));
      upload(m->ind_to, it.data(), nrow * sizeof(int));
      upload(m->ind_from, iff.data(), ncolumn * sizeof(int));
      upload(m->jminus, jm.data(), nrow * sizeof(int));
    } catch (...) {
      lfg_cma_destroy(m);
      throw;
    }
    *out = m;
  });
}

int lfg_cma_destroy(lfg_cma m) {
  if (!m) return LFG_OK;
  dfree(m->bands);
  dfree(m->ind_to);
  dfree(m->ind_from);
  dfree(m->jminus);
  dfree(m->jplus);
  dfree(m->tptr);
  dfree(m->trow);
  dfree(m->finv);
  dfree(m->fcp);
  dfree(m->asm_rowptr);
  dfree(m->asm_list);
  delete m;
  return LFG_OK;
}

int lfg_cma_apply(lfg_cma m, lfg_field lhs, lfg_field x) {
  if (!m) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(lhs && x && lhs->ncol == m->ncol && x->ncol == m->ncol &&
                    lhs->nlev >= m->max_ind_to && x->nlev >= m->max_ind_from &&
                    lhs->kind == m->kind && x->kind == m->kind,
                "cma_apply: fields do not match the operator");
    // 16-byte vectors of columns when every row starts on a 16-byte boundary
    const int V = 16 / m->kind;
    const bool vec = m->ncol % V == 0 && reinterpret_cast<uintptr_t>(x->d) % 16 == 0 &&
                     reinterpret_cast<uintptr_t>(lhs->d) % 16 == 0;
    bool tri = m->bw == 3 && m->alpha == 1 && m->beta == 1 && m->gm == 1 && m->gp == 1 &&
               m->nrow == m->ncolumn && m->ind_identity && m->ind_from_identity;
    dispatch(m->kind, [&](auto tag) {
      using T = decltype(tag);
      if (vec) {
        constexpr int VT = 16 / sizeof(T);
        dim3 grid((m->ncol / VT + 127) / 128, m->nrow);
        auto k = tri ? k_cma_app_v<T, VT, true> : k_cma_app_v<T, VT, false>;
        k<<<grid, 128, 0, c->stream>>>((const T*)m->bands, m->ind_to, m->ind_from, m->jminus,
                                       m->jplus, m->ncol, m->nrow, m->ncolumn, (const T*)x->d,
                                       (T*)lhs->d);
      } else {
        dim3 grid((m->ncol + 127) / 128, m->nrow);
        k_cma_app<T><<<grid, 128, 0, c->stream>>>((const T*)m->bands, m->ind_to, m->ind_from,
                                                  m->jminus, m->jplus, m->ncol, m->nrow,
                                                  m->ncolumn, (const T*)x->d, (T*)lhs->d);
      }
    });
    after_launch(c, "cma_app", (uint64_t)m->kind * m->ncol * ((uint64_t)(m->bw + 2) * m->nrow + m->ncolumn));
  });
}

int lfg_cma_apply_transpose(lfg_cma m, lfg_field lhs, lfg_field x) {
  if (!m) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(lhs && x && lhs->ncol == m->ncol && x->ncol == m->ncol &&
                    lhs->nlev >= m->max_ind_from && x->nlev >= m->max_ind_to &&
                    lhs->kind == m->kind && x->kind == m->kind,
                "cma_apply_transpose: fields do not match the operator");
    dim3 grid((m->ncol + 127) / 128, m->ncolumn);
    dispatch(m->kind, [&](auto tag) {
      using T = decltype(tag);
      k_cma_app_t<T><<<grid, 128, 0, c->stream>>>((const T*)m->bands, m->ind_to, m->ind_from,
                                                  m->jminus, m->tptr, m->trow, m->ncol, m->nrow,
                                                  (const T*)x->d, (T*)lhs->d);
    });
    after_launch(c, "cma_app_t", (uint64_t)m->kind * m->ncol * ((uint64_t)(m->bw + 1) * m->nrow + 2 * (uint64_t)m->ncolumn));
  });
}

int lfg_cma_apply_inverse(lfg_cma m, lfg_field lhs, lfg_field x) {
  if (!m) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(m->bw == 3 && m->nrow == m->ncolumn,
                "cma_apply_inverse: needs a square tridiagonal operator (bandwidth 3)");
    LFG_REQUIRE(lhs && x && lhs->ncol == m->ncol && x->ncol == m->ncol &&
                    lhs->nlev >= m->max_ind_to && x->nlev >= m->max_ind_to &&
                    lhs->kind == m->kind && x->kind == m->kind,
                "cma_apply_inverse: fields do not match the operator");
    const size_t n = (size_t)m->nrow * m->ncol;
    const size_t smem_col = (size_t)m->nrow * m->kind;
    if (smem_col * 32 > 200 * 1024) {  // columns too tall for shared memory
      dispatch(m->kind, [&](auto tag) {
        using T = decltype(tag);
        TriSrc<T> s{m->ncol, m->nrow, (const T*)m->bands, nullptr, nullptr, nullptr, m->ind_to, 0};
        launch_thomas<T, SRC_CMA>(c, s, (const T*)x->d, (T*)lhs->d);
      });
      return;
    }
    if (!m->fvalid) {
      if (!m->finv) {
        m->finv = dmalloc(n * m->kind);
        m->fcp = dmalloc(n * m->kind);
      }
      dispatch(m->kind, [&](auto tag) {
        using T = decltype(tag);
        k_cma_factor<T><<<(m->ncol + 127) / 128, 128, 0, c->stream>>>(
            (const T*)m->bands, m->ncol, m->nrow, (T*)m->finv, (T*)m->fcp);
      });
      after_launch(c, "cma_factor", (uint64_t)m->kind * 5 * m->ncol * m->nrow);
      m->fvalid = true;
    }
    // Fields of exactly nrow levels with the identity row map: the
    // TMA-staged column substitution of the Helmholtz smoother, which does
    // the same arithmetic on the same factors (x_out = 1 * z)
    if (m->ind_identity && lhs->nlev == m->nrow && x->nlev == m->nrow) {
      const void* ptrs[5] = {x->d, m->bands, m->finv, m->fcp, nullptr};
      if (subst_tma_applicable(c, m->ncol, m->nrow, ptrs, 5, m->kind)) {
        if (m->kind == LFG_R_DOUBLE)
          subst_tma(c, m->ncol, m->nrow, (const double*)x->d, (const double*)m->bands,
                    (const double*)m->finv, (const double*)m->fcp, nullptr, 1.0,
                    (double*)lhs->d);
        else
          subst_tma(c, m->ncol, m->nrow, (const float*)x->d, (const float*)m->bands,
                    (const float*)m->finv, (const float*)m->fcp, nullptr, 1.0f,
                    (float*)lhs->d);
        return;
      }
    }
    // FP64: segmented form; FP32 columns (half the bytes per row) measured
    // faster one thread per column
    if (const int S = m->kind == LFG_R_DOUBLE ? cma_seg_lanes(m->nrow) : 0) {
      const unsigned grid = (unsigned)((m->ncol + 31) / 32);
      dispatch(m->kind, [&](auto tag) {
        using T = decltype(tag);
        auto go = [&](void (*k)(const T*, const T*, const T*, const int*, int, int, const T*, T*)) {
          k<<<grid, 32 * S, 0, c->stream>>>((const T*)m->bands, (const T*)m->finv,
                                            (const T*)m->fcp, m->ind_to, m->ncol, m->nrow,
                                            (const T*)x->d, (T*)lhs->d);
        };
        if (S == 2) go(k_cma_subst_seg<T, 2>);
        else if (S == 4) go(k_cma_subst_seg<T, 4>);
        else go(k_cma_subst_seg<T, 8>);
      });
      after_launch(c, "cma_subst_seg", (uint64_t)m->kind * 5 * m->ncol * m->nrow);
      return;
    }
    int bs = 128;
    while (bs > 32 && (m->ncol + bs - 1) / bs < 2 * c->num_sms) bs /= 2;
    while (smem_col * bs > 200 * 1024) bs /= 2;
    dispatch(m->kind, [&](auto tag) {
      using T = decltype(tag);
      ensure_smem_attr((const void*)k_cma_subst<T>, 200 * 1024);
      k_cma_subst<T><<<(m->ncol + bs - 1) / bs, bs, smem_col * bs, c->stream>>>(
          (const T*)m->bands, (const T*)m->finv, (const T*)m->fcp, m->ind_to, m->ncol, m->nrow,
          (const T*)x->d, (T*)lhs->d);
    });
    after_launch(c, "cma_subst", (uint64_t)m->kind * 5 * m->ncol * m->nrow);
  });
}

int lfg_tri_solve(lfg_field y, lfg_field x, lfg_field t0, lfg_field tp, lfg_field tm) {
  if (!y) return LFG_ERR_ARG;
  lfg_ctx c = y->ctx;
  return guard(c, [&] {
    for (lfg_field f : {x, t0, tp, tm})
      LFG_REQUIRE(f && f->ncol == y->ncol && f->nlev == y->nlev && f->kind == y->kind,
                  "tri_solve: fields differ in shape or kind");
    dispatch(y->kind, [&](auto tag) {
      using T = decltype(tag);
      TriSrc<T> s{y->ncol, y->nlev, nullptr, (const T*)t0->d, (const T*)tp->d,
                  (const T*)tm->d, nullptr, 0};
      launch_thomas<T, SRC_FIELDS>(c, s, (const T*)x->d, (T*)y->d);
    });
  });
}

int lfg_operator_tri_solve(lfg_lma m, lfg_field y, lfg_field x) {
  if (!m) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(m->ndf_to == 2 && m->ndf_from == 2, "operator_tri_solve: needs a 2x2 LMA");
    LFG_REQUIRE(y && x && y->ncol == m->ncell && x->ncol == m->ncell &&
                    y->nlev == m->nl + 1 && x->nlev == m->nl + 1 && y->kind == m->kind &&
                    x->kind == m->kind,
                "operator_tri_solve: fields must have nlayers+1 levels per cell");
    dispatch(m->kind, [&](auto tag) {
      using T = decltype(tag);
      TriSrc<T> s{m->ncell, m->nl + 1, (const T*)m->a, nullptr, nullptr, nullptr, nullptr, m->nl};
      launch_thomas<T, SRC_LMA2>(c, s, (const T*)x->d, (T*)y->d);
    });
  });
}

// ------------------------------------------------------------- intergrid
int lfg_intergrid_create(lfg_ctx c, int ncoarse, int nfine, int nx, int ny,
                         const int* cell_map, const int* ccorners, const int* fcorners,
                         lfg_intergrid* out) {
  if (!c || !out) return LFG_ERR_ARG;
  return guard(c, [&] {
    LFG_REQUIRE(ncoarse > 0 && nfine > 0 && nx > 0 && ny > 0 && cell_map,
                "intergrid_create: bad arguments");
    LFG_REQUIRE(nfine == ncoarse * nx * ny, "intergrid_create: nfine != ncoarse*nx*ny");
    const int nq = nx * ny;
    std::vector<int> child((size_t)nq * ncoarse), parent(nfine, -1);
    for (int C = 0; C < ncoarse; ++C)
      for (int q = 0; q < nq; ++q) {
        int f = cell_map[(size_t)C * nq + q];
        LFG_REQUIRE(f >= 0 && f < nfine, "intergrid_create: fine cell id out of range");
        LFG_REQUIRE(parent[f] < 0, "intergrid_create: fine cell in two coarse cells");
        child[(size_t)q * ncoarse + C] = f;
        parent[f] = C;
      }
    lfg_intergrid g = new lfg_intergrid_s;
    g->ctx = c;
    g->ncoarse = ncoarse;
    g->nfine = nfine;
    g->nx = nx;
    g->ny = ny;
    g->h_child.assign(cell_map, cell_map + (size_t)nq * ncoarse);
    // 2x2 maps between structured cubed-sphere meshes: the same child
    // placement in every coarse cell of a panel
    std::vector<int> cedge;
    if (nx == 2 && ny == 2) {
      const long nc = std::lround(std::sqrt((double)ncoarse / 6.0)), nf = 2 * nc;
      bool ok = nc >= 3 && 6 * nc * nc == ncoarse && 6 * nf * nf == nfine && nf < (1 << 14);
      unsigned long long code = 0;
      for (long P = 0; P < 6 && ok; ++P)
        for (int q = 0; q < 4 && ok; ++q) {
          int pos = -1;
          for (long J = 0; J < nc && ok; ++J)
            for (long I = 0; I < nc && ok; ++I) {
              const long C = P * nc * nc + J * nc + I;
              const long d = child[(size_t)q * ncoarse + C] - (P * nf * nf + 2 * J * nf + 2 * I);
              const int dp = d == 0 ? 0 : d == 1 ? 1 : d == nf ? 2 : d == nf + 1 ? 3 : -1;
              if (dp < 0 || (pos >= 0 && dp != pos)) ok = false;
              pos = dp;
            }
          code |= (unsigned long long)pos << (8 * P + 2 * q);
        }
      if (ok) {
        g->pnc = (int)nc;
        g->qpos = code;
        for (long P = 0; P < 6; ++P)
          for (long J = 0; J < nc; ++J)
            for (long I = 0; I < nc; ++I)
              if (I == 0 || J == 0 || I == nc - 1 || J == nc - 1)
                cedge.push_back((int)(P * nc * nc + J * nc + I));
      }
    }
    try {
      g->child = (int*)dmalloc(child.size() * sizeof(int));
      g->parent = (int*)dmalloc(parent.size() * sizeof(int));
      upload(g->child, child.data(), child.size() * sizeof(int));
      upload(g->parent, parent.data(), parent.size() * sizeof(int));
      if (!cedge.empty()) {
        g->cedge = (int*)dmalloc(cedge.size() * sizeof(int));
        upload(g->cedge, cedge.data(), cedge.size() * sizeof(int));
        g->ncedge = (int)cedge.size();
      }
      if (ccorners && fcorners) {
        int nvc = 0, nvf = 0;
        for (size_t i = 0; i < (size_t)4 * ncoarse; ++i) nvc = std::max(nvc, ccorners[i] + 1);
        for (size_t i = 0; i < (size_t)4 * nfine; ++i) nvf = std::max(nvf, fcorners[i] + 1);
        g->nvert_coarse = nvc;
        g->nvert_fine = nvf;
        std::vector<int> cc((size_t)4 * ncoarse);
        for (int C = 0; C < ncoarse; ++C)
          for (int s = 0; s < 4; ++s) cc[(size_t)s * ncoarse + C] = ccorners[4 * C + s];
        // injection table (sci_restrict_w0_kernel_mod.F90:95-150): the NW, SW,
        // NE, SE coarse corners from the corner fine cells
        std::vector<int> inj(nvc, -1);
        const int SWB = 0, SEB = 1, NEB = 2, NWB = 3;
        for (int C = 0; C < ncoarse; ++C) {
          auto cm_at = [&](int x, int y) { return cell_map[(size_t)C * nq + y * nx + x]; };
          inj[ccorners[4 * C + NWB]] = fcorners[4 * cm_at(0, 0) + NWB];
          inj[ccorners[4 * C + SWB]] = fcorners[4 * cm_at(0, ny - 1) + SWB];
          inj[ccorners[4 * C + NEB]] = fcorners[4 * cm_at(nx - 1, 0) + NEB];
          inj[ccorners[4 * C + SEB]] = fcorners[4 * cm_at(nx - 1, ny - 1) + SEB];
        }
        for (int v = 0; v < nvc; ++v)
          LFG_REQUIRE(inj[v] >= 0, "intergrid_create: coarse vertex without fine partner");
        // last-writer table of the bilinear prolongation (reference loop order)
        std::vector<int> src(nvf, -1);
        std::vector<double> wts((size_t)5 * nvf, 0.0);
        auto put = [&](int v, int C, double a, double b, double cc2, double d, int nterm) {
          src[v] = C;
          double* w = &wts[(size_t)5 * v];
          w[0] = a; w[1] = b; w[2] = cc2; w[3] = d; w[4] = nterm;
        };
        for (int C = 0; C < ncoarse; ++C)
          for (int y = 1; y <= ny; ++y)
            for (int x = 1; x <= nx; ++x) {
              const int f = cell_map[(size_t)C * nq + (y - 1) * nx + (x - 1)];
              const double nxy = (double)(nx * ny);
              double wsw = (double)y * (double)(nx - x + 1) / nxy;
              double wnw = (double)(ny - y) * (double)(nx - x + 1) / nxy;
              double wne = (double)(ny - y) * (double)(x - 1) / nxy;
              double wse = (double)y * (double)(x - 1) / nxy;
              put(fcorners[4 * f + SWB], C, wne, wse, wsw, wnw, 4);
              if (x == nx) {
                wse = (double)y / (double)ny;
                wne = 1.0 - wse;
                put(fcorners[4 * f + SEB], C, wne, wse, 0.0, 0.0, 2);
              }
              if (y == 1) {
                wnw = (double)(nx - x + 1) / (double)nx;
                wne = 1.0 - wnw;
                put(fcorners[4 * f + NWB], C, wne, 0.0, 0.0, wnw, 3);
                if (x == nx) put(fcorners[4 * f + NEB], C, 1.0, 0.0, 0.0, 0.0, 1);
              }
            }
        g->ccorner = (int*)dmalloc(cc.size() * sizeof(int));
        upload(g->ccorner, cc.data(), cc.size() * sizeof(int));
        int* d_inj = (int*)dmalloc(inj.size() * sizeof(int));
        upload(d_inj, inj.data(), inj.size() * sizeof(int));
        int* d_src = (int*)dmalloc(src.size() * sizeof(int));
        upload(d_src, src.data(), src.size() * sizeof(int));
        double* d_w = (double*)dmalloc(wts.size() * sizeof(double));
        upload(d_w, wts.data(), wts.size() * sizeof(double));
        g->w0_inj = d_inj;
        g->w0_src = d_src;
        g->w0_w = d_w;
      }
    } catch (...) {
      lfg_intergrid_destroy(g);
      throw;
    }
    *out = g;
  });
}

int lfg_intergrid_destroy(lfg_intergrid g) {
  if (!g) return LFG_OK;
  dfree(g->child);
  dfree(g->parent);
  dfree(g->ccorner);
  dfree(g->w0_inj);
  dfree(g->w0_src);
  dfree(g->w0_w);
  dfree(g->cedge);
  delete g;
  return LFG_OK;
}

int lfg_restrict_scalar(lfg_intergrid g, int mode, lfg_field coarse, lfg_field fine,
                        lfg_field w) {
  if (!g) return LFG_ERR_ARG;
  lfg_ctx c = g->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(coarse && fine && coarse->ncol == g->ncoarse && fine->ncol == g->nfine &&
                    coarse->nlev == fine->nlev && coarse->kind == fine->kind,
                "restrict_scalar: fields do not match the intergrid map");
    LFG_REQUIRE(mode >= 0 && mode <= 2, "restrict_scalar: bad mode");
    if (mode == LFG_RESTRICT_WEIGHTED)
      LFG_REQUIRE(w && w->ncol == fine->ncol && w->nlev == fine->nlev && w->kind == fine->kind,
                  "restrict_scalar: weighted restriction needs fine weights");
    dim3 grid((g->ncoarse + 127) / 128, fine->nlev);
    const int nq = g->nx * g->ny;
    dispatch(fine->kind, [&](auto tag) {
      using T = decltype(tag);
      const T* wp = w ? (const T*)w->d : nullptr;
      if (mode == LFG_RESTRICT_UNWEIGHTED)
        k_restrict<T, LFG_RESTRICT_UNWEIGHTED><<<grid, 128, 0, c->stream>>>((T*)coarse->d, (const T*)fine->d, wp, g->child, g->ncoarse, g->nfine, nq, fine->nlev);
      else if (mode == LFG_RESTRICT_WEIGHTED)
        k_restrict<T, LFG_RESTRICT_WEIGHTED><<<grid, 128, 0, c->stream>>>((T*)coarse->d, (const T*)fine->d, wp, g->child, g->ncoarse, g->nfine, nq, fine->nlev);
      else
        k_restrict<T, LFG_RESTRICT_MASS_W3><<<grid, 128, 0, c->stream>>>((T*)coarse->d, (const T*)fine->d, wp, g->child, g->ncoarse, g->nfine, nq, fine->nlev);
    });
    // fine read (and its weights), coarse written
    after_launch(c, "restrict_scalar",
                 (uint64_t)fine->kind * fine->nlev *
                     ((uint64_t)g->nfine * (mode == LFG_RESTRICT_WEIGHTED ? 2 : 1) + g->ncoarse));
  });
}

int lfg_prolong_scalar(lfg_intergrid g, lfg_field fine, lfg_field coarse, lfg_field w) {
  if (!g) return LFG_ERR_ARG;
  lfg_ctx c = g->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(coarse && fine && coarse->ncol == g->ncoarse && fine->ncol == g->nfine &&
                    coarse->nlev == fine->nlev && coarse->kind == fine->kind,
                "prolong_scalar: fields do not match the intergrid map");
    if (w)
      LFG_REQUIRE(w->ncol == fine->ncol && w->nlev == fine->nlev && w->kind == fine->kind,
                  "prolong_scalar: weights must be a fine field");
    const size_t nblk = (size_t)g->nfine * ((fine->nlev + KI - 1) / KI);
    dispatch(fine->kind, [&](auto tag) {
      using T = decltype(tag);
      auto go = [&](void (*k)(T*, const T*, const T*, const int*, int, int, int)) {
        k<<<occ_grid(c, (const void*)k, 256, nblk), 256, 0, c->stream>>>(
            (T*)fine->d, (const T*)coarse->d, w ? (const T*)w->d : nullptr, g->parent, g->nfine,
            g->ncoarse, fine->nlev);
      };
      if (w) go(k_prolong<T, true>);
      else go(k_prolong<T, false>);
    });
    // fine read and written (weights read), coarse read
    after_launch(c, "prolong_scalar",
                 (uint64_t)fine->kind * fine->nlev *
                     ((uint64_t)g->nfine * (w ? 3 : 2) + g->ncoarse));
  });
}

int lfg_restrict_w0(lfg_intergrid g, lfg_field coarse, lfg_field fine) {
  if (!g) return LFG_ERR_ARG;
  lfg_ctx c = g->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(g->ccorner, "restrict_w0: intergrid map was created without W0 corners");
    LFG_REQUIRE(coarse && fine && coarse->ncol == g->nvert_coarse &&
                    fine->ncol == g->nvert_fine && coarse->nlev == fine->nlev &&
                    coarse->kind == fine->kind,
                "restrict_w0: fields do not match the W0 vertex columns");
    dim3 grid((g->nvert_coarse + 127) / 128, fine->nlev);
    dispatch(fine->kind, [&](auto tag) {
      using T = decltype(tag);
      k_restrict_w0<T><<<grid, 128, 0, c->stream>>>((T*)coarse->d, (const T*)fine->d, g->w0_inj,
                                                    g->nvert_coarse, g->nvert_fine, fine->nlev);
    });
    after_launch(c, "restrict_w0", (uint64_t)fine->kind * fine->nlev * 2 * g->nvert_coarse);
  });
}

int lfg_prolong_w0(lfg_intergrid g, lfg_field fine, lfg_field coarse) {
  if (!g) return LFG_ERR_ARG;
  lfg_ctx c = g->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(g->ccorner, "prolong_w0: intergrid map was created without W0 corners");
    LFG_REQUIRE(coarse && fine && coarse->ncol == g->nvert_coarse &&
                    fine->ncol == g->nvert_fine && coarse->nlev == fine->nlev &&
                    coarse->kind == fine->kind,
                "prolong_w0: fields do not match the W0 vertex columns");
    dim3 grid((g->nvert_fine + 127) / 128, fine->nlev);
    dispatch(fine->kind, [&](auto tag) {
      using T = decltype(tag);
      k_prolong_w0<T><<<grid, 128, 0, c->stream>>>((T*)fine->d, (const T*)coarse->d, g->w0_src,
                                                   g->w0_w, g->ccorner, g->nvert_fine,
                                                   g->nvert_coarse, g->ncoarse, fine->nlev);
    });
    after_launch(c, "prolong_w0",
                 (uint64_t)fine->kind * fine->nlev * ((uint64_t)g->nvert_fine + g->nvert_coarse));
  });
}

}  // extern "C"

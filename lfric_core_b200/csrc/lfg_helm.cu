// Meshes and the W3 Helmholtz operator: apply, residual, block-Jacobi column
// smoother (fused residual + Thomas solve), fused residual + restriction,
// prolongation and the Galerkin coarse operator.
//
// A = T' - H_off: T' is a columnwise-assembled tridiagonal per column
// (columnwise_operator_type with bandwidth 3, infrastructure/source/operator/
// columnwise_operator_mod.f90:42-114) whose diagonal includes the horizontal
// couplings; H_off couples each cell to its four face neighbours on the
// same level.  The column solve is the Thomas algorithm of
// components/science/source/kernel/columnwise_operators/
// sci_columnwise_op_appinv_kernel_mod.F90:77-145 (multiply by the inverse
// denominator, c' not formed on the last row).
//
// Every kernel here is HBM-bandwidth bound (< 1 flop/byte).  The
// element-parallel kernels (apply, right-hand side, residual) give a thread
// one column and KC levels; the substitutions give a thread one column and
// walk its levels (on fine meshes through the TMA kernels of
// lfg_subst_tma.cu; on small meshes S threads share a column in the
// segmented sweep), so at every level a warp reads consecutive columns of
// each level-major array.
//
// H_off is symmetric: the two sides of a face hold one coupling.  A mesh
// names one designated side per face (hsrc); an FP64 operator whose sides
// all equal their designated sides bit for bit (checked once, k_face_check)
// is read through them (the CF kernel variants), 2 coupling words per dof
// instead of 4.
#include "lfg_internal.cuh"

#include <algorithm>
#include <type_traits>

using namespace lfg;

namespace {

template <class T>
struct HelmArgs {
  int ncol, nl;
  const T* __restrict__ sub;
  const T* __restrict__ diag;
  const T* __restrict__ sup;
  const T* __restrict__ h;       // [4][nl][ncol]
  const int* __restrict__ links; // [4][ncol]
  const T* __restrict__ inv;     // Thomas inverse denominators [nl][ncol]
  const T* __restrict__ cp;      // Thomas c' [nl][ncol]
  const int* __restrict__ hsrc;  // [4][ncol] designated side of each face (CF kernels)
};

template <class T>
HelmArgs<T> args_of(lfg_helm op) {
  return HelmArgs<T>{op->ncol, op->nl, (const T*)op->sub, (const T*)op->diag,
                     (const T*)op->sup, (const T*)op->h, op->mesh->links,
                     (const T*)op->inv, (const T*)op->cp, op->mesh->hsrc};
}

// Coupling of side f of a column at level k, at index i = k*ncol + c of
// the per-side array.  CF (every face's two sides equal): read through the
// face's designated side, fc = the column's hsrc codes, so each face's value
// comes from one array element and inside a panel the W and S planes stay
// unread.
template <bool CF, class T>
__device__ __forceinline__ T h_side(const HelmArgs<T>& A, int f, int k, size_t i,
                                    const int (&fc)[4]) {
  const size_t plane = (size_t)A.nl * A.ncol;
  if constexpr (CF)
    return A.h[(size_t)(fc[f] >> 29) * plane + (size_t)k * A.ncol + (fc[f] & 0x1fffffff)];
  else
    return A.h[(size_t)f * plane + i];
}

// hsrc codes of column c (CF), else zeros
template <bool CF, class T>
__device__ __forceinline__ void load_faces(const HelmArgs<T>& A, unsigned c, int (&fc)[4]) {
#pragma unroll
  for (int f = 0; f < 4; ++f) fc[f] = CF ? A.hsrc[(size_t)f * A.ncol + c] : 0;
}

// Levels per thread in the element-parallel kernels: a thread keeps its
// column's neighbour ids in registers over KC consecutive levels, whose
// loads are all independent.
constexpr int KC = 2;

// Levels a thread keeps in registers in the segmented coarse-level sweep.
constexpr int kSegLevels = 12;

// (A x)(c,k) from values already in registers: the T' row (sub, diag,
// super, in the columnwise_op_app order) then minus the four couplings.
// has_m / has_p select the sub / super terms without a branch.
template <class T>
__device__ __forceinline__ T helm_row_v(T sb, T dg, T sp, const T (&hv)[4], T xm, T x0, T xp,
                                        const T (&xn)[4], bool has_m, bool has_p) {
  T acc = has_m ? sb * xm : (T)0;
  acc = acc + dg * x0;
  if (has_p) acc = acc + sp * xp;
#pragma unroll
  for (int f = 0; f < 4; ++f) acc = acc - hv[f] * xn[f];
  return acc;
}

// y = A x (RESID: y = b - A x).  DOT: accumulate <y, w> (w null: <y, y>)
// into a deterministic reduction.  Thread = (column, chunk of KC levels);
// all loads of the chunk are issued before any arithmetic (addresses are
// clamped into the column, so no load sits behind a branch).
template <class T, bool RESID, bool DOT, bool HASW, bool CF>
__global__ void __launch_bounds__(256) k_helm_apply(HelmArgs<T> A, const T* __restrict__ x,
                                                    const T* __restrict__ b, T* __restrict__ y,
                                                    const T* __restrict__ w, Red r) {
  const unsigned N = A.ncol;
  const int nl = A.nl;
  const int nchunk = (nl + KC - 1) / KC;
  const unsigned total = N * (unsigned)nchunk;
  double acc = 0.0;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned kc = t / N, c = t - kc * N;
    int nb[4], fc[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) nb[f] = A.links[f * N + c];
    load_faces<CF>(A, c, fc);
    const int k0 = kc * KC;
    const int kn = min(KC, nl - k0);
    // column values x(k0-1 .. k0+KC) with clamped levels
    T xv[KC + 2];
#pragma unroll
    for (int q = 0; q < KC + 2; ++q) {
      const int k = min(max(k0 - 1 + q, 0), nl - 1);
      xv[q] = x[(size_t)k * N + c];
    }
    // all loads and arithmetic of the chunk first, stores after (the
    // compiler cannot reorder loads across stores through these pointers)
    T vout[KC];
#pragma unroll
    for (int kk = 0; kk < KC; ++kk) {
      const int k = min(k0 + kk, nl - 1);
      const size_t i = (size_t)k * N + c;
      T xn[4], hv[4];
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        xn[f] = x[(size_t)k * N + nb[f]];
        hv[f] = h_side<CF>(A, f, k, i, fc);
      }
      T v = helm_row_v(A.sub[i], A.diag[i], A.sup[i], hv, xv[kk], xv[kk + 1], xv[kk + 2], xn,
                       k > 0, k < nl - 1);
      if (RESID) v = b[i] - v;
      vout[kk] = v;
      if (DOT && kk < kn) acc += (double)v * (double)(HASW ? w[i] : v);
    }
#pragma unroll
    for (int kk = 0; kk < KC; ++kk)
      if (kk < kn) y[(size_t)(k0 + kk) * N + c] = vout[kk];
  }
  if (DOT) red_finish(r, acc);
}

// Thomas factors of T' per column with columnwise_op_appinv's arithmetic:
// inv_k = 1/(diag_k - sub_k c'_{k-1}) (inv_0 = 1/diag_0), c'_k = inv_k sup_k
// (not formed on the last row).
template <class T>
__global__ void k_helm_factor(const T* __restrict__ sub, const T* __restrict__ diag,
                              const T* __restrict__ sup, T* __restrict__ inv, T* __restrict__ cp,
                              int ncol, int nl) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  T cprev = (T)0;
  for (int k = 0; k < nl; ++k) {
    const size_t i = (size_t)k * ncol + c;
    const T iv = k == 0 ? (T)1 / diag[i] : (T)1 / (diag[i] - sub[i] * cprev);
    const T ck = k < nl - 1 ? iv * sup[i] : (T)0;
    inv[i] = iv;
    cp[i] = ck;
    cprev = ck;
  }
}

// The block-Jacobi column sweep of A x = b,
//   x_out = omega T'^{-1} (b + H_off x_in) + (1 - omega) x_in,
// which equals x_in + omega T'^{-1} (b - A x_in), runs as two streaming
// kernels.
//
// (1) k_helm_rhs: r = b + H_off x_in, one thread per (column, chunk of KC
//     levels), loads issued before the stores.
template <class T, bool CF>
__global__ void __launch_bounds__(256) k_helm_rhs(HelmArgs<T> A, const T* __restrict__ xin,
                                                  const T* __restrict__ b, T* __restrict__ r) {
  const unsigned N = A.ncol;
  const int nl = A.nl;
  const size_t plane = (size_t)nl * N;
  const int nchunk = (nl + KC - 1) / KC;
  const unsigned total = N * (unsigned)nchunk;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned kc = t / N, c = t - kc * N;
    int nb[4], fc[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) nb[f] = A.links[f * N + c];
    load_faces<CF>(A, c, fc);
    const int k0 = kc * KC;
    const int kn = min(KC, nl - k0);
    T out[KC];
#pragma unroll
    for (int kk = 0; kk < KC; ++kk) {
      const int k = min(k0 + kk, nl - 1);
      const size_t i = (size_t)k * N + c;
      T hs = (T)0;
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        // a designated side is read by two columns: keep it cacheable
        const T hv = CF ? h_side<CF>(A, f, k, i, fc) : __ldcs(A.h + f * plane + i);
        hs = hs + hv * xin[(size_t)k * N + nb[f]];
      }
      out[kk] = __ldcs(b + i) + hs;
    }
#pragma unroll
    for (int kk = 0; kk < KC; ++kk)
      if (kk < kn) r[(size_t)(k0 + kk) * N + c] = out[kk];
  }
}

// (2) k_helm_subst: the substitutions of columnwise_op_appinv with the
//     per-operator Thomas factors (inverse denominators inv, c'):
//       d'_k = inv_k (r_k - sub_k d'_{k-1}),  z_k = d'_k - c'_k z_{k+1},
//     then x_out = omega z + (1 - omega) x_in.  One thread per column; d'
//     goes to shared memory [level][thread].  The recurrence is two
//     multiply-adds per level, so the kernel lives on memory-level
//     parallelism: each sweep walks the column in blocks of SP levels and
//     loads block b+1 (clamped addresses, no conditional loads) before it
//     computes block b.
constexpr int SP = 16;

template <class T, bool XIN>
__global__ void __launch_bounds__(128) k_helm_subst(
    int ncol, int nl, const T* __restrict__ r, const T* __restrict__ sub,
    const T* __restrict__ inv, const T* __restrict__ cp, const T* __restrict__ xin, T omega,
    T* __restrict__ xout) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sd = reinterpret_cast<T*>(smem_raw);     // [nl][blockDim]
  const int t = threadIdx.x, bs = blockDim.x;
  const unsigned c = blockIdx.x * bs + t;
  if (c >= (unsigned)ncol) return;
  const size_t N = ncol;
  const int nb = (nl + SP - 1) / SP;
  auto at = [&](int k) { return (size_t)min(max(k, 0), nl - 1) * N + c; };
  // forward sweep
  T ar[SP], ai[SP], as[SP], br[SP], bi[SP], bsb[SP];
#pragma unroll
  for (int p = 0; p < SP; ++p) {
    const size_t i = at(p);
    ar[p] = r[i];
    ai[p] = inv[i];
    as[p] = sub[i];
  }
  T d = (T)0;
  for (int blk = 0; blk < nb; ++blk) {
    const int k0 = blk * SP;
#pragma unroll
    for (int p = 0; p < SP; ++p) {
      const size_t i = at(k0 + SP + p);
      br[p] = r[i];
      bi[p] = inv[i];
      bsb[p] = sub[i];
    }
#pragma unroll
    for (int p = 0; p < SP; ++p) {
      const int k = k0 + p;
      const T dn = k == 0 ? ai[p] * ar[p] : ai[p] * (ar[p] - as[p] * d);
      if (k < nl) {
        d = dn;
        sd[k * bs + t] = d;
      }
    }
#pragma unroll
    for (int p = 0; p < SP; ++p) {
      ar[p] = br[p];
      ai[p] = bi[p];
      as[p] = bsb[p];
    }
  }
  // backward sweep
  const T om1 = (T)1 - omega;
  auto xv_at = [&](int k) -> T { return xin[(size_t)min(max(k, 0), nl - 1) * N + c]; };
  T ac[SP], ax[SP], bc[SP], bx[SP];
  const int ktop = nl - 1;
#pragma unroll
  for (int p = 0; p < SP; ++p) {
    ac[p] = cp[at(ktop - p)];
    if (XIN) ax[p] = xv_at(ktop - p);
  }
  T z = (T)0;
  for (int blk = 0; blk < nb; ++blk) {
    const int k0 = ktop - blk * SP;
#pragma unroll
    for (int p = 0; p < SP; ++p) {
      bc[p] = cp[at(k0 - SP - p)];
      if (XIN) bx[p] = xv_at(k0 - SP - p);
    }
#pragma unroll
    for (int p = 0; p < SP; ++p) {
      const int k = k0 - p;
      if (k >= 0) {
        const T dk = sd[k * bs + t];
        z = (k == ktop) ? dk : dk - ac[p] * z;
        T v = omega * z;
        if (XIN) v = v + om1 * ax[p];
        xout[(size_t)k * N + c] = v;
      }
    }
#pragma unroll
    for (int p = 0; p < SP; ++p) {
      ac[p] = bc[p];
      if (XIN) ax[p] = bx[p];
    }
  }
}

// bc(C,k) = sum over the children q (y outer, x inner) of (b - A x)(child,k):
// residual fused with restrict_mass_w3 (sci_restrict_mass_w3_kernel_mod.F90:126-179).
// Thread = (coarse column, chunk of KR levels), loads issued before use.
constexpr int KR = 2;
template <class T, bool CF>
__global__ void __launch_bounds__(256) k_helm_resid_restrict(HelmArgs<T> A,
                                                             const T* __restrict__ x,
                                                             const T* __restrict__ b,
                                                             T* __restrict__ bc,
                                                             const int* __restrict__ child,
                                                             int ncoarse, int nq) {
  const unsigned NC = ncoarse, N = A.ncol;
  const int nl = A.nl;
  const int nchunk = (nl + KR - 1) / KR;
  const unsigned total = NC * (unsigned)nchunk;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned kc = t / NC, C = t - kc * NC;
    const int k0 = kc * KR;
    const int kn = min(KR, nl - k0);
    T acc[KR];
#pragma unroll
    for (int kk = 0; kk < KR; ++kk) acc[kk] = (T)0;
    for (int q = 0; q < nq; ++q) {
      const unsigned c = child[q * NC + C];
      int nb[4], fc[4];
#pragma unroll
      for (int f = 0; f < 4; ++f) nb[f] = A.links[f * N + c];
      load_faces<CF>(A, c, fc);
      T xv[KR + 2];
#pragma unroll
      for (int u = 0; u < KR + 2; ++u) {
        const int k = min(max(k0 - 1 + u, 0), nl - 1);
        xv[u] = x[(size_t)k * N + c];
      }
#pragma unroll
      for (int kk = 0; kk < KR; ++kk) {
        const int k = min(k0 + kk, nl - 1);
        const size_t i = (size_t)k * N + c;
        T xn[4], hv[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          xn[f] = x[(size_t)k * N + nb[f]];
          hv[f] = h_side<CF>(A, f, k, i, fc);
        }
        const T v = helm_row_v(A.sub[i], A.diag[i], A.sup[i], hv, xv[kk], xv[kk + 1],
                               xv[kk + 2], xn, k > 0, k < nl - 1);
        acc[kk] = acc[kk] + (b[i] - v);
      }
    }
#pragma unroll
    for (int kk = 0; kk < KR; ++kk)
      if (kk < kn) bc[(size_t)(k0 + kk) * NC + C] = acc[kk];
  }
}

// fine(c,k) += coarse(parent(c),k)   (prolong_scalar_unweighted on W3)
// One thread per (column, block of KP levels), columns fastest, grid-stride:
// the parent index is read once per block and the block's loads are all
// issued before its stores.
constexpr int KP = 4;
template <class T>
__global__ void k_prolong_add(T* __restrict__ fine, const T* __restrict__ coarse,
                              const int* __restrict__ parent, int nfine, int ncoarse, int nl) {
  const size_t nblk = (size_t)nfine * ((nl + KP - 1) / KP);
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nblk;
       t += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(t % nfine), k0 = (int)(t / nfine) * KP;
    const int p = parent[c];
    T fv[KP], cv[KP];
#pragma unroll
    for (int kk = 0; kk < KP; ++kk)
      if (k0 + kk < nl) {
        fv[kk] = fine[(size_t)(k0 + kk) * nfine + c];
        cv[kk] = coarse[(size_t)(k0 + kk) * ncoarse + p];
      }
#pragma unroll
    for (int kk = 0; kk < KP; ++kk)
      if (k0 + kk < nl) fine[(size_t)(k0 + kk) * nfine + c] = fv[kk] + cv[kk];
  }
}

// Galerkin coarse operator, one thread per coarse column (FP64).
__global__ void k_galerkin(HelmArgs<double> F, double* __restrict__ csub,
                           double* __restrict__ cdiag, double* __restrict__ csup,
                           double* __restrict__ ch_out, const int* __restrict__ child,
                           int ncoarse) {
  const int C = blockIdx.x * blockDim.x + threadIdx.x;
  if (C >= ncoarse) return;
  const size_t N = F.ncol, NC = ncoarse;
  const size_t plane = (size_t)F.nl * N, cplane = (size_t)F.nl * NC;
  int ch[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) ch[q] = child[q * ncoarse + C];
  // children on each side: W: x=0 -> q {0,2}; S: y=1 -> {2,3}; E: x=1 -> {1,3}; N: y=0 -> {0,1}
  const int side_q[4][2] = {{0, 2}, {2, 3}, {1, 3}, {0, 1}};
  for (int k = 0; k < F.nl; ++k) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int q = 0; q < 4; ++q) {
      const size_t i = (size_t)k * N + ch[q];
      s0 = s0 + F.sub[i];
      s1 = s1 + F.diag[i];
      s2 = s2 + F.sup[i];
    }
    for (int q = 0; q < 4; ++q)
      for (int f = 0; f < 4; ++f) {
        const int nb = F.links[f * N + ch[q]];
        if (nb == ch[0] || nb == ch[1] || nb == ch[2] || nb == ch[3])
          s1 = s1 - F.h[f * plane + (size_t)k * N + ch[q]];
      }
    const size_t o = (size_t)k * NC + C;
    csub[o] = s0;
    cdiag[o] = s1;
    csup[o] = s2;
    for (int f = 0; f < 4; ++f)
      ch_out[f * cplane + o] = F.h[f * plane + (size_t)k * N + ch[side_q[f][0]]] +
                               F.h[f * plane + (size_t)k * N + ch[side_q[f][1]]];
  }
}

template <class TO, class TI>
__global__ void k_convert(TO* __restrict__ y, const TI* __restrict__ x, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = (TO)x[i];
}

// Whole sweep for meshes with few columns (the coarse multigrid levels),
// where one thread per column leaves most of the GPU idle and every level of
// the serial recurrences costs a memory latency.  S threads share a column,
// each owning L = ceil(nl/S) consecutive levels (at most LMAX, kept in
// registers), and the block has 128/S columns.  The right-hand side
// r = b + H_off x_in is formed in place, so the sweep is one kernel.  Both recurrences of the
// substitution,
//   d_k = (r_k - sub_k d_{k-1}) inv_k,   z_k = d_k - c'_k z_{k+1},
// are affine in the carried value: each thread composes its segment's map,
// an inclusive scan of the maps over the S segments (shuffles of width S)
// gives every segment its incoming value, and each segment then replays
// its levels with exactly the sequential formulas from that value.
template <class T, bool XIN, int S, bool CF>
__global__ void __launch_bounds__(128) k_helm_sweep_seg(HelmArgs<T> A, const T* __restrict__ b,
                                                        const T* __restrict__ xin, T omega,
                                                        T* __restrict__ xout) {
  constexpr int LMAX = kSegLevels;
  const int tid = threadIdx.x, j = tid % S;
  const unsigned c = blockIdx.x * (128 / S) + tid / S;
  const size_t N = A.ncol;
  const int nl = A.nl;
  const int L = (nl + S - 1) / S, k0 = j * L;
  const int nmy = c < N ? max(0, min(L, nl - k0)) : 0;
  int nb[4] = {0, 0, 0, 0}, fc[4] = {0, 0, 0, 0};
  if (XIN && nmy > 0) {
#pragma unroll
    for (int f = 0; f < 4; ++f) nb[f] = A.links[f * N + c];
    load_faces<CF>(A, c, fc);
  }
  T d[LMAX], iv[LMAX], sb[LMAX];
#pragma unroll
  for (int u = 0; u < LMAX; ++u) {
    if (u < nmy) {
      const int k = k0 + u;
      const size_t i = (size_t)k * N + c;
      T rv = b[i];
      if (XIN) {
        T hs = (T)0;
#pragma unroll
        for (int f = 0; f < 4; ++f) hs = hs + h_side<CF>(A, f, k, i, fc) * xin[(size_t)k * N + nb[f]];
        rv = rv + hs;
      }
      d[u] = rv;
      iv[u] = A.inv[i];
      sb[u] = A.sub[i];
    }
  }
  // forward: this segment's map d_out = D + M d_in
  T D = (T)0, M = (T)1;
#pragma unroll
  for (int u = 0; u < LMAX; ++u)
    if (u < nmy) {
      D = (d[u] - sb[u] * D) * iv[u];
      M = M * (-sb[u] * iv[u]);
    }
#pragma unroll
  for (int off = 1; off < S; off <<= 1) {
    const T Dp = __shfl_up_sync(0xffffffffu, D, off, S);
    const T Mp = __shfl_up_sync(0xffffffffu, M, off, S);
    if (j >= off) {
      D = D + M * Dp;
      M = M * Mp;
    }
  }
  T dv = __shfl_up_sync(0xffffffffu, D, 1, S);
  if (j == 0) dv = (T)0;
#pragma unroll
  for (int u = 0; u < LMAX; ++u)
    if (u < nmy) {
      dv = k0 + u == 0 ? iv[u] * d[u] : iv[u] * (d[u] - sb[u] * dv);
      d[u] = dv;
    }
  // backward: z_in of a segment is z at the first level of the next one
  T cc[LMAX];
#pragma unroll
  for (int u = 0; u < LMAX; ++u)
    if (u < nmy) cc[u] = A.cp[(size_t)(k0 + u) * N + c];
  T E = (T)0, Nn = (T)1;
#pragma unroll
  for (int u = LMAX - 1; u >= 0; --u)
    if (u < nmy) {
      E = d[u] - cc[u] * E;
      Nn = Nn * (-cc[u]);
    }
#pragma unroll
  for (int off = 1; off < S; off <<= 1) {
    const T Ep = __shfl_down_sync(0xffffffffu, E, off, S);
    const T Np = __shfl_down_sync(0xffffffffu, Nn, off, S);
    if (j + off < S) {
      E = E + Nn * Ep;
      Nn = Nn * Np;
    }
  }
  T z = __shfl_down_sync(0xffffffffu, E, 1, S);
  if (j == S - 1) z = (T)0;
  const T om1 = (T)1 - omega;
#pragma unroll
  for (int u = LMAX - 1; u >= 0; --u)
    if (u < nmy) {
      const int k = k0 + u;
      const size_t i = (size_t)k * N + c;
      z = k == nl - 1 ? d[u] : d[u] - cc[u] * z;
      T v = omega * z;
      if (XIN) v = v + om1 * xin[i];
      xout[i] = v;
    }
}

// Threads per column for the segmented sweep (0: use the per-column kernels):
// enough threads to cover the GPU, and segments of at most kSegLevels.
inline int seg_threads(lfg_ctx c, int ncol, int nl) {
  const long want = 2L * c->num_sms * 128;
  if ((long)ncol >= want) return 0;
  int S = 1;
  while ((long)ncol * S < want && S < 32) S *= 2;
  while ((nl + S - 1) / S > kSegLevels && S < 32) S *= 2;
  if ((nl + S - 1) / S > kSegLevels || S < 4) return 0;
  return S;
}

// Coupling words per dof the kernels read: 4 per side, 2 through the
// designated sides.
inline double coupling_words(lfg_helm op) { return op->hsym ? 2.0 : 4.0; }

template <class T, bool XIN>
void launch_sweep_seg(lfg_ctx c, int S, HelmArgs<T> A, const T* b, const T* xin, T omega,
                      T* xout, double hwords) {
  const int cols = 128 / S;
  const unsigned grid = (unsigned)((A.ncol + cols - 1) / cols);
  auto go = [&](auto cf) {
    constexpr bool CF = decltype(cf)::value;
    switch (S) {
      case 4: k_helm_sweep_seg<T, XIN, 4, CF><<<grid, 128, 0, c->stream>>>(A, b, xin, omega, xout); break;
      case 8: k_helm_sweep_seg<T, XIN, 8, CF><<<grid, 128, 0, c->stream>>>(A, b, xin, omega, xout); break;
      case 16: k_helm_sweep_seg<T, XIN, 16, CF><<<grid, 128, 0, c->stream>>>(A, b, xin, omega, xout); break;
      default: k_helm_sweep_seg<T, XIN, 32, CF><<<grid, 128, 0, c->stream>>>(A, b, xin, omega, xout); break;
    }
  };
  if (XIN && hwords < 4.0) go(std::true_type{});
  else go(std::false_type{});
  // b, inv, sub, c' read and x written; x_in and the couplings with XIN
  after_launch(c, "helm_sweep_seg",
               (uint64_t)(sizeof(T) * (XIN ? 6 + hwords : 5) * (double)A.ncol * A.nl));
}

template <class T, bool XIN>
void launch_subst(lfg_ctx c, int ncol, int nl, const T* r, const T* sub, const T* inv,
                  const T* cp, const T* xin, T omega, T* xout) {
  const void* ptrs[5] = {r, sub, inv, cp, xin};
  if (subst_tma_applicable(c, ncol, nl, ptrs, 5, (int)sizeof(T))) {
    subst_tma(c, ncol, nl, r, sub, inv, cp, XIN ? xin : nullptr, omega, xout);
    return;
  }
  // spread small meshes over every SM
  int bs = 128;
  while (bs > 32 && (ncol + bs - 1) / bs < 2 * c->num_sms) bs /= 2;
  constexpr size_t cap = 200 * 1024;
  if ((size_t)nl * 32 * sizeof(T) > cap)
    throw Error(LFG_ERR_ARG, "helm_smooth: column too tall for shared memory");
  while ((size_t)nl * bs * sizeof(T) > cap) bs /= 2;
  auto kern = k_helm_subst<T, XIN>;
  ensure_smem_attr((const void*)kern, (int)cap);
  kern<<<(ncol + bs - 1) / bs, bs, (size_t)nl * bs * sizeof(T), c->stream>>>(
      ncol, nl, r, sub, inv, cp, xin, omega, xout);
  // r, inv, sub, c' read and x written; x_in with XIN
  after_launch(c, "helm_subst", sizeof(T) * (XIN ? 6 : 5) * (uint64_t)ncol * nl);
}

// r = b + H_off x (k_helm_rhs)
template <class T>
void launch_rhs(lfg_helm op, const T* x, const T* b, T* r) {
  lfg_ctx c = op->ctx;
  const size_t work = (size_t)op->ncol * ((op->nl + KC - 1) / KC);
  auto rk = op->hsym ? k_helm_rhs<T, true> : k_helm_rhs<T, false>;
  rk<<<occ_grid(c, (const void*)rk, 256, work), 256, 0, c->stream>>>(args_of<T>(op), x, b, r);
  // x, b and the couplings read, r written
  after_launch(c, "helm_rhs",
               (uint64_t)(sizeof(T) * (3 + coupling_words(op)) * (double)op->ncol * op->nl));
}

template <class T>
void smooth_t(lfg_helm op, double omega, lfg_field x_in, lfg_field b, lfg_field x_out,
              void* rbuf) {
  lfg_ctx c = op->ctx;
  const T om = (T)omega;
  const T* sub = (const T*)op->sub;
  const T* inv = (const T*)op->inv;
  const T* cp = (const T*)op->cp;
  if (const int S = seg_threads(c, op->ncol, op->nl)) {
    const HelmArgs<T> A = args_of<T>(op);
    if (!x_in)
      launch_sweep_seg<T, false>(c, S, A, (const T*)b->d, nullptr, om, (T*)x_out->d, 4.0);
    else
      launch_sweep_seg<T, true>(c, S, A, (const T*)b->d, (const T*)x_in->d, om, (T*)x_out->d,
                                coupling_words(op));
    return;
  }
  if (!x_in) {
    launch_subst<T, false>(c, op->ncol, op->nl, (const T*)b->d, sub, inv, cp, nullptr, om,
                           (T*)x_out->d);
    return;
  }
  T* r = (T*)rbuf;
  launch_rhs<T>(op, (const T*)x_in->d, (const T*)b->d, r);
  launch_subst<T, true>(c, op->ncol, op->nl, r, sub, inv, cp, (const T*)x_in->d, om,
                        (T*)x_out->d);
}

// k_helm_apply<T, RESID, DOT, HASW, CF> for the operator's coupling storage
template <class T, bool RESID, bool DOT, bool HASW>
void launch_apply(lfg_helm op, const T* x, const T* b, T* y, const T* w, Red r) {
  lfg_ctx c = op->ctx;
  const int bs = 256;
  const size_t work = (size_t)op->ncol * ((op->nl + KC - 1) / KC);
  auto k = op->hsym ? k_helm_apply<T, RESID, DOT, HASW, true>
                    : k_helm_apply<T, RESID, DOT, HASW, false>;
  k<<<occ_grid(c, (const void*)k, bs, work), bs, 0, c->stream>>>(args_of<T>(op), x, b, y, w, r);
}

void check_field(lfg_helm op, lfg_field f, const char* what) {
  LFG_REQUIRE(f, std::string(what) + ": null field");
  LFG_REQUIRE(f->ncol == op->ncol && f->nlev == op->nl && f->kind == op->kind,
              std::string(what) + ": field does not match the operator (shape or kind)");
}

}  // namespace

namespace lfg {

void helm_apply(lfg_helm op, lfg_field y, lfg_field x, lfg_field dot_with, int slot) {
  check_field(op, y, "helm_apply");
  check_field(op, x, "helm_apply");
  lfg_ctx c = op->ctx;
  Red r = slot >= 0 ? c->red(slot) : Red{nullptr, nullptr, nullptr};
  auto go = [&](auto tag) {
    using T = decltype(tag);
    const T* xd = (const T*)x->d;
    T* yd = (T*)y->d;
    if (slot >= 0 && dot_with)
      launch_apply<T, false, true, true>(op, xd, nullptr, yd, (const T*)dot_with->d, r);
    else if (slot >= 0)
      launch_apply<T, false, true, false>(op, xd, nullptr, yd, nullptr, r);
    else
      launch_apply<T, false, false, false>(op, xd, nullptr, yd, nullptr, r);
  };
  if (op->kind == LFG_R_DOUBLE) go(double{});
  else go(float{});
  // x, the three bands and the couplings read, y written; w read for <y, w>
  const double words = 5 + coupling_words(op) + (slot >= 0 && dot_with ? 1 : 0);
  after_launch(c, "helm_apply", (uint64_t)(op->kind * words * (double)op->ncol * op->nl));
}

void helm_residual(lfg_helm op, lfg_field r_out, lfg_field x, lfg_field b, int slot) {
  check_field(op, r_out, "helm_residual");
  check_field(op, x, "helm_residual");
  check_field(op, b, "helm_residual");
  lfg_ctx c = op->ctx;
  Red r = slot >= 0 ? c->red(slot) : Red{nullptr, nullptr, nullptr};
  auto go = [&](auto tag) {
    using T = decltype(tag);
    if (slot >= 0)
      launch_apply<T, true, true, false>(op, (const T*)x->d, (const T*)b->d, (T*)r_out->d,
                                         nullptr, r);
    else
      launch_apply<T, true, false, false>(op, (const T*)x->d, (const T*)b->d, (T*)r_out->d,
                                          nullptr, r);
  };
  if (op->kind == LFG_R_DOUBLE) go(double{});
  else go(float{});
  // x, b, the three bands and the couplings read, r written
  after_launch(c, "helm_residual",
               (uint64_t)(op->kind * (6 + coupling_words(op)) * (double)op->ncol * op->nl));
}

void helm_smooth(lfg_helm op, double omega, lfg_field x_in, lfg_field b, lfg_field x_out,
                 void* rbuf) {
  check_field(op, b, "helm_smooth");
  check_field(op, x_out, "helm_smooth");
  if (x_in) {
    check_field(op, x_in, "helm_smooth");
    LFG_REQUIRE(x_in->d != x_out->d, "helm_smooth: x_out may not alias x_in");
  }
  if (x_in && !rbuf) rbuf = op->ctx->scratch((size_t)op->ncol * op->nl * op->kind);
  if (op->kind == LFG_R_DOUBLE) smooth_t<double>(op, omega, x_in, b, x_out, rbuf);
  else smooth_t<float>(op, omega, x_in, b, x_out, rbuf);
}

void helm_residual_restrict(lfg_helm op, lfg_intergrid ig, lfg_field x, lfg_field b,
                            lfg_field bc) {
  check_field(op, x, "residual_restrict");
  check_field(op, b, "residual_restrict");
  LFG_REQUIRE(ig->nfine == op->ncol && bc->ncol == ig->ncoarse && bc->nlev == op->nl &&
                  bc->kind == op->kind && ig->nx * ig->ny <= 4,
              "residual_restrict: bad coarse field");
  lfg_ctx c = op->ctx;
  const int bs = 256;
  const size_t work = (size_t)ig->ncoarse * ((op->nl + KR - 1) / KR);
  auto go = [&](auto tag) {
    using T = decltype(tag);
    auto k = op->hsym ? k_helm_resid_restrict<T, true> : k_helm_resid_restrict<T, false>;
    k<<<occ_grid(c, (const void*)k, bs, work), bs, 0, c->stream>>>(
        args_of<T>(op), (const T*)x->d, (const T*)b->d, (T*)bc->d, ig->child, ig->ncoarse,
        ig->nx * ig->ny);
  };
  if (op->kind == LFG_R_DOUBLE) go(double{});
  else go(float{});
  // x, b, the three bands and the couplings read, the coarse right-hand side written
  after_launch(c, "resid_restrict",
               (uint64_t)(op->kind * (double)op->nl *
                          ((5 + coupling_words(op)) * (double)op->ncol + ig->ncoarse)));
}

void prolong_add(lfg_intergrid ig, lfg_field fine, lfg_field coarse) {
  LFG_REQUIRE(fine->ncol == ig->nfine && coarse->ncol == ig->ncoarse &&
                  fine->nlev == coarse->nlev && fine->kind == coarse->kind,
              "prolong_add: bad fields");
  lfg_ctx c = fine->ctx;
  const size_t work = (size_t)ig->nfine * ((fine->nlev + KP - 1) / KP);
  if (fine->kind == LFG_R_DOUBLE)
    k_prolong_add<double><<<occ_grid(c, (const void*)k_prolong_add<double>, 256, work), 256, 0, c->stream>>>((double*)fine->d, (const double*)coarse->d, ig->parent, ig->nfine, ig->ncoarse, fine->nlev);
  else
    k_prolong_add<float><<<occ_grid(c, (const void*)k_prolong_add<float>, 256, work), 256, 0, c->stream>>>((float*)fine->d, (const float*)coarse->d, ig->parent, ig->nfine, ig->ncoarse, fine->nlev);
  after_launch(c, "prolong_add",
               (uint64_t)fine->kind * fine->nlev * (2 * (uint64_t)ig->nfine + ig->ncoarse));
}

}  // namespace lfg

// ================================================================ C ABI
static lfg_helm new_helm(lfg_ctx c, lfg_mesh mesh, int kind, int nl) {
  lfg_helm op = new lfg_helm_s;
  op->ctx = c;
  op->mesh = mesh;
  op->kind = kind;
  op->ncol = mesh->ncol;
  op->nl = nl;
  const size_t n = (size_t)op->ncol * nl;
  try {
    op->sub = dmalloc(n * kind);
    op->diag = dmalloc(n * kind);
    op->sup = dmalloc(n * kind);
    op->h = dmalloc(4 * n * kind);
    op->inv = dmalloc(n * kind);
    op->cp = dmalloc(n * kind);
  } catch (...) {
    dfree(op->sub); dfree(op->diag); dfree(op->sup); dfree(op->h); dfree(op->inv);
    dfree(op->cp);
    delete op;
    throw;
  }
  return op;
}

__device__ __forceinline__ bool same_bits(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b);
}
__device__ __forceinline__ bool same_bits(float a, float b) {
  return __float_as_uint(a) == __float_as_uint(b);
}

// *bad = 1 unless every side's coupling equals its face's designated side
// bit for bit
template <class T>
__global__ void k_face_check(const T* __restrict__ h, const int* __restrict__ hsrc, int ncol,
                             int nl, unsigned* bad) {
  const size_t plane = (size_t)nl * ncol, n = 4 * plane;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(t / plane);
    const size_t r = t - (size_t)f * plane;
    const int k = (int)(r / ncol), c = (int)(r - (size_t)k * ncol);
    const int v = hsrc[(size_t)f * ncol + c];
    const T a = h[t], b = h[(size_t)(v >> 29) * plane + (size_t)k * ncol + (v & 0x1fffffff)];
    if (!same_bits(a, b)) *bad = 1u;
  }
}

// Thomas factors of the operator's T' (after its bands change), and whether
// its kernels may read each face through one side.
static void factor_helm(lfg_helm op) {
  lfg_ctx c = op->ctx;
  const int bs = 128, grid = (op->ncol + bs - 1) / bs;
  if (op->kind == LFG_R_DOUBLE)
    k_helm_factor<double><<<grid, bs, 0, c->stream>>>((const double*)op->sub, (const double*)op->diag, (const double*)op->sup, (double*)op->inv, (double*)op->cp, op->ncol, op->nl);
  else
    k_helm_factor<float><<<grid, bs, 0, c->stream>>>((const float*)op->sub, (const float*)op->diag, (const float*)op->sup, (float*)op->inv, (float*)op->cp, op->ncol, op->nl);
  after_launch(c, "helm_factor", (uint64_t)op->kind * op->ncol * op->nl * 5);
  // Designated-side reads for FP64 operators (C192x70: apply 202 -> 143 us,
  // smoother sweep 274 -> 245 us); the FP32 kernels measured no faster with
  // them and keep the per-side reads.
  op->hsym = false;
  lfg_mesh m = op->mesh;
  if (m->hsrc && op->kind == LFG_R_DOUBLE) {
    unsigned* bad = (unsigned*)dmalloc(sizeof(unsigned));
    try {
      LFG_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned), c->stream));
      const size_t n4 = 4 * (size_t)op->ncol * op->nl;
      k_face_check<double><<<c->stream_grid(n4), kThreads, 0, c->stream>>>(
          (const double*)op->h, m->hsrc, op->ncol, op->nl, bad);
      after_launch(c, "face_check", (uint64_t)sizeof(double) * n4);
      unsigned flag = 1;
      LFG_CUDA(cudaMemcpyAsync(&flag, bad, sizeof(flag), cudaMemcpyDeviceToHost, c->stream));
      LFG_CUDA(cudaStreamSynchronize(c->stream));
      op->hsym = flag == 0;
    } catch (...) {
      dfree(bad);
      throw;
    }
    dfree(bad);
  }
  LFG_CUDA(cudaStreamSynchronize(c->stream));
}

extern "C" {

int lfg_mesh_create(lfg_ctx c, int ncol, const int* links, lfg_mesh* out) {
  if (!c || !out) return LFG_ERR_ARG;
  return guard(c, [&] {
    LFG_REQUIRE(ncol > 0 && links, "mesh_create: bad arguments");
    std::vector<int> soa((size_t)4 * ncol);
    for (int i = 0; i < ncol; ++i)
      for (int f = 0; f < 4; ++f) {
        int nb = links[4 * i + f];
        LFG_REQUIRE(nb >= 0 && nb < ncol, "mesh_create: neighbour id out of range");
        soa[(size_t)f * ncol + i] = nb;
      }
    // Pair every side (i, f) with an unpaired side (nb, g) of its neighbour
    // that links back to i; then the designated side of each face: the
    // larger side index, then the smaller column.
    bool paired = (size_t)ncol < ((size_t)1 << 29);
    std::vector<int> pair_side(paired ? (size_t)4 * ncol : 0, -1);  // g * ncol + nb
    for (int i = 0; i < ncol && paired; ++i)
      for (int f = 0; f < 4 && paired; ++f) {
        if (pair_side[(size_t)f * ncol + i] >= 0) continue;
        const int nb = links[4 * i + f];
        int g = 0;
        while (g < 4 && !(links[4 * nb + g] == i && pair_side[(size_t)g * ncol + nb] < 0))
          ++g;
        if (g == 4) {
          paired = false;
          break;
        }
        pair_side[(size_t)f * ncol + i] = g * ncol + nb;
        pair_side[(size_t)g * ncol + nb] = f * ncol + i;
      }
    std::vector<int> hsrc;
    if (paired) {
      hsrc.resize((size_t)4 * ncol);
      for (int i = 0; i < ncol; ++i)
        for (int f = 0; f < 4; ++f) {
          const int ps = pair_side[(size_t)f * ncol + i], g = ps / ncol, nb = ps % ncol;
          const bool mine = f > g || (f == g && i <= nb);
          hsrc[(size_t)f * ncol + i] = mine ? (f << 29 | i) : (g << 29 | nb);
        }
    }
    lfg_mesh m = new lfg_mesh_s;
    m->ctx = c;
    m->ncol = ncol;
    m->h_links.assign(links, links + (size_t)4 * ncol);
    try {
      m->links = (int*)dmalloc(soa.size() * sizeof(int));
      upload(m->links, soa.data(), soa.size() * sizeof(int));
      if (paired) {
        m->hsrc = (int*)dmalloc(hsrc.size() * sizeof(int));
        upload(m->hsrc, hsrc.data(), hsrc.size() * sizeof(int));
      }
    } catch (...) {
      dfree(m->links);
      dfree(m->hsrc);
      delete m;
      throw;
    }
    *out = m;
  });
}

int lfg_mesh_destroy(lfg_mesh m) {
  if (!m) return LFG_OK;
  dfree(m->links);
  dfree(m->hsrc);
  delete m;
  return LFG_OK;
}

int lfg_helm_create(lfg_ctx c, int kind, lfg_mesh mesh, int nl, const double* cm,
                    const double* hface, lfg_helm* out) {
  if (!c || !out) return LFG_ERR_ARG;
  return guard(c, [&] {
    LFG_REQUIRE(mesh && cm && hface && nl > 0, "helm_create: bad arguments");
    LFG_REQUIRE(kind == LFG_R_DOUBLE || kind == LFG_R_SINGLE, "helm_create: bad kind");
    const int ncol = mesh->ncol;
    const size_t n = (size_t)ncol * nl;
    std::vector<double> sub(n), dg(n), sp(n), h(4 * n);
    for (int col = 0; col < ncol; ++col)
      for (int k = 0; k < nl; ++k) {
        const size_t src = (size_t)col * nl + k, dst = (size_t)k * ncol + col;
        sub[dst] = cm[src * 3 + 0];
        dg[dst] = cm[src * 3 + 1];
        sp[dst] = cm[src * 3 + 2];
        for (int f = 0; f < 4; ++f) h[f * n + dst] = hface[src * 4 + f];
      }
    lfg_helm op = new_helm(c, mesh, kind, nl);
    auto put = [&](void* d, const std::vector<double>& v) {
      if (kind == LFG_R_DOUBLE) {
        upload(d, v.data(), v.size() * sizeof(double));
      } else {
        std::vector<float> f(v.begin(), v.end());
        upload(d, f.data(), f.size() * sizeof(float));
      }
    };
    try {
      put(op->sub, sub);
      put(op->diag, dg);
      put(op->sup, sp);
      put(op->h, h);
      factor_helm(op);
    } catch (...) {
      lfg_helm_destroy(op);
      throw;
    }
    *out = op;
  });
}

int lfg_helm_destroy(lfg_helm op) {
  if (!op) return LFG_OK;
  dfree(op->sub);
  dfree(op->diag);
  dfree(op->sup);
  dfree(op->h);
  dfree(op->inv);
  dfree(op->cp);
  delete op;
  return LFG_OK;
}

int lfg_helm_apply(lfg_helm op, lfg_field y, lfg_field x) {
  if (!op) return LFG_ERR_ARG;
  return guard(op->ctx, [&] { helm_apply(op, y, x, nullptr, -1); });
}

int lfg_helm_smooth(lfg_helm op, double omega, lfg_field x_in, lfg_field b, lfg_field x_out) {
  if (!op) return LFG_ERR_ARG;
  return guard(op->ctx, [&] { helm_smooth(op, omega, x_in, b, x_out, nullptr); });
}

int lfg_helm_residual_restrict(lfg_helm op, lfg_intergrid ig, lfg_field x, lfg_field b,
                               lfg_field coarse_b) {
  if (!op || !ig || !x || !b || !coarse_b) return LFG_ERR_ARG;
  return guard(op->ctx, [&] { helm_residual_restrict(op, ig, x, b, coarse_b); });
}

int lfg_helm_sweep_rhs(lfg_helm op, lfg_field x, lfg_field b, lfg_field r) {
  if (!op) return LFG_ERR_ARG;
  return guard(op->ctx, [&] {
    check_field(op, x, "helm_sweep_rhs");
    check_field(op, b, "helm_sweep_rhs");
    check_field(op, r, "helm_sweep_rhs");
    LFG_REQUIRE(r->d != x->d, "helm_sweep_rhs: r may not alias x");
    if (op->kind == LFG_R_DOUBLE)
      launch_rhs<double>(op, (const double*)x->d, (const double*)b->d, (double*)r->d);
    else
      launch_rhs<float>(op, (const float*)x->d, (const float*)b->d, (float*)r->d);
  });
}

int lfg_helm_coarsen(lfg_helm fine, lfg_intergrid ig, lfg_mesh cmesh, int kind,
                     lfg_helm* out) {
  if (!fine || !out) return LFG_ERR_ARG;
  lfg_ctx c = fine->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(fine->kind == LFG_R_DOUBLE, "helm_coarsen: the fine operator must be r_double");
    LFG_REQUIRE(ig && cmesh && ig->nfine == fine->ncol && ig->ncoarse == cmesh->ncol &&
                    ig->nx == 2 && ig->ny == 2,
                "helm_coarsen: intergrid map does not match (2x2 maps only)");
    lfg_helm c64 = new_helm(c, cmesh, LFG_R_DOUBLE, fine->nl);
    const int bs = 128, grid = (cmesh->ncol + bs - 1) / bs;
    k_galerkin<<<grid, bs, 0, c->stream>>>(args_of<double>(fine), (double*)c64->sub,
                                           (double*)c64->diag, (double*)c64->sup,
                                           (double*)c64->h, ig->child, cmesh->ncol);
    try {
      after_launch(c, "galerkin");
      factor_helm(c64);
    } catch (...) {
      lfg_helm_destroy(c64);
      throw;
    }
    if (kind == LFG_R_DOUBLE) {
      *out = c64;
      return;
    }
    lfg_helm c32 = nullptr;
    int st = lfg_helm_copy_kind(c64, kind, &c32);
    lfg_helm_destroy(c64);
    if (st != LFG_OK) throw Error(st, c->last_error);
    *out = c32;
  });
}

int lfg_helm_copy_kind(lfg_helm src, int kind, lfg_helm* out) {
  if (!src || !out) return LFG_ERR_ARG;
  lfg_ctx c = src->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(kind == LFG_R_DOUBLE || kind == LFG_R_SINGLE, "helm_copy_kind: bad kind");
    lfg_helm d = new_helm(c, src->mesh, kind, src->nl);
    const size_t n = (size_t)src->ncol * src->nl;
    void* s_arr[4] = {src->sub, src->diag, src->sup, src->h};
    void* d_arr[4] = {d->sub, d->diag, d->sup, d->h};
    for (int a = 0; a < 4; ++a) {
      const size_t m = a == 3 ? 4 * n : n;
      const int g = c->stream_grid(m);
      if (src->kind == kind)
        LFG_CUDA(cudaMemcpyAsync(d_arr[a], s_arr[a], m * kind, cudaMemcpyDeviceToDevice, c->stream));
      else if (kind == LFG_R_SINGLE)
        k_convert<float, double><<<g, kThreads, 0, c->stream>>>((float*)d_arr[a], (const double*)s_arr[a], m);
      else
        k_convert<double, float><<<g, kThreads, 0, c->stream>>>((double*)d_arr[a], (const float*)s_arr[a], m);
      if (src->kind != kind) after_launch(c, "convert", (uint64_t)m * (src->kind + kind));
    }
    try {
      factor_helm(d);
    } catch (...) {
      lfg_helm_destroy(d);
      throw;
    }
    *out = d;
  });
}

}  // extern "C"

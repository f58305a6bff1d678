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
#include <cmath>
#include <initializer_list>
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

// Shapes of the segmented coarse-level sweep: S threads per column, each
// keeping at most LM levels in registers (the register arrays are sized LM,
// so a shape fits its segments tightly: 70 levels are 4 x 18, 8 x 9,
// 16 x 5 or 32 x 3).  The last shape takes columns up to 384 levels.
struct SegShape {
  int S, LM;
};
constexpr SegShape kSegShapes[] = {{4, 18}, {8, 9}, {16, 5}, {32, 3}, {32, 12}};

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

// What the element-parallel kernels compute: y = A x, y = b - A x, or the
// sweep's right-hand side y = b + H_off x.
enum { M_APPLY = 0, M_RESID = 1, M_RHS = 2 };

// Levels k0 .. k0+KC-1 of column c through the links table (every mesh):
// all loads of the chunk are issued before any arithmetic (addresses are
// clamped into the column, so no load sits behind a branch), the stores
// after (the compiler cannot reorder loads across stores through these
// pointers).  DOT accumulates <y, w> (HASW) or <y, y> into acc.  y is
// stored in TO (the values and acc are formed in T).
template <class T, int MODE, bool DOT, bool HASW, bool CF, class TO = T>
__device__ __forceinline__ void col_levels(const HelmArgs<T>& A, unsigned c, int k0,
                                           const T* __restrict__ x, const T* __restrict__ b,
                                           TO* __restrict__ y, const T* __restrict__ w,
                                           double& acc) {
  const unsigned N = A.ncol;
  const int nl = A.nl;
  const size_t plane = (size_t)nl * N;
  const int kn = min(KC, nl - k0);
  int nb[4], fc[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) nb[f] = A.links[f * N + c];
  load_faces<CF>(A, c, fc);
  T vout[KC];
  if constexpr (MODE == M_RHS) {
#pragma unroll
    for (int kk = 0; kk < KC; ++kk) {
      const int k = min(k0 + kk, nl - 1);
      const size_t i = (size_t)k * N + c;
      T hs = (T)0;
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        // a designated side is read by two columns: keep it cacheable
        const T hv = CF ? h_side<CF>(A, f, k, i, fc) : __ldcs(A.h + f * plane + i);
        hs = hs + hv * x[(size_t)k * N + nb[f]];
      }
      vout[kk] = __ldcs(b + i) + hs;
    }
  } else {
    // column values x(k0-1 .. k0+KC) with clamped levels
    T xv[KC + 2];
#pragma unroll
    for (int q = 0; q < KC + 2; ++q) {
      const int k = min(max(k0 - 1 + q, 0), nl - 1);
      xv[q] = x[(size_t)k * N + c];
    }
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
      if (MODE == M_RESID) v = b[i] - v;
      vout[kk] = v;
      if (DOT && kk < kn) acc += (double)v * (double)(HASW ? w[i] : v);
    }
  }
#pragma unroll
  for (int kk = 0; kk < KC; ++kk)
    if (kk < kn) y[(size_t)(k0 + kk) * N + c] = (TO)vout[kk];
}

// y = A x (RESID: y = b - A x).  DOT: accumulate <y, w> (w null: <y, y>)
// into a deterministic reduction.  Thread = (column, chunk of KC levels).
// TO: y's kind (FP32 for the mixed refinement's FP64 residual, rounded once
// as a separate conversion would round it).
template <class T, bool RESID, bool DOT, bool HASW, bool CF, class TO = T>
__global__ void __launch_bounds__(256) k_helm_apply(HelmArgs<T> A, const T* __restrict__ x,
                                                    const T* __restrict__ b, TO* __restrict__ y,
                                                    const T* __restrict__ w, Red r) {
  grid_dep_wait();
  const unsigned N = A.ncol;
  const int nchunk = (A.nl + KC - 1) / KC;
  const unsigned total = N * (unsigned)nchunk;
  double acc = 0.0;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned kc = t / N, c = t - kc * N;
    col_levels<T, RESID ? M_RESID : M_APPLY, DOT, HASW, CF, TO>(A, c, (int)kc * KC, x, b, y, w,
                                                               acc);
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
  grid_dep_wait();
  const unsigned N = A.ncol;
  const int nchunk = (A.nl + KC - 1) / KC;
  const unsigned total = N * (unsigned)nchunk;
  double acc = 0.0;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned kc = t / N, c = t - kc * N;
    col_levels<T, M_RHS, false, false, CF>(A, c, (int)kc * KC, xin, b, r, nullptr, acc);
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
  grid_dep_wait();
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
// child_resid: (b - A x) at levels k0 .. k0+NLV-1 of fine column c through
// the links table (every mesh), loads issued before use.
constexpr int KR = 2;
template <class T, bool CF, int NLV>
__device__ __forceinline__ void child_resid(const HelmArgs<T>& A, const T* __restrict__ x,
                                            const T* __restrict__ b, unsigned c, int k0,
                                            T (&r)[NLV]) {
  const unsigned N = A.ncol;
  const int nl = A.nl;
  int nb[4], fc[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) nb[f] = A.links[f * N + c];
  load_faces<CF>(A, c, fc);
  T xv[NLV + 2];
#pragma unroll
  for (int u = 0; u < NLV + 2; ++u) {
    const int k = min(max(k0 - 1 + u, 0), nl - 1);
    xv[u] = x[(size_t)k * N + c];
  }
#pragma unroll
  for (int kk = 0; kk < NLV; ++kk) {
    const int k = min(k0 + kk, nl - 1);
    const size_t i = (size_t)k * N + c;
    T xn[4], hv[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      xn[f] = x[(size_t)k * N + nb[f]];
      hv[f] = h_side<CF>(A, f, k, i, fc);
    }
    const T v = helm_row_v(A.sub[i], A.diag[i], A.sup[i], hv, xv[kk], xv[kk + 1], xv[kk + 2],
                           xn, k > 0, k < nl - 1);
    r[kk] = b[i] - v;
  }
}

// One thread sums all nq children of coarse column C (the panel kernel's
// border columns).
template <class T, bool CF, int NLV = KR>
__device__ __forceinline__ void resid_restrict_col(const HelmArgs<T>& A,
                                                   const T* __restrict__ x,
                                                   const T* __restrict__ b, T* __restrict__ bc,
                                                   const int* __restrict__ child, unsigned NC,
                                                   int nq, unsigned C, int k0) {
  const int kn = min(NLV, A.nl - k0);
  T acc[NLV];
#pragma unroll
  for (int kk = 0; kk < NLV; ++kk) acc[kk] = (T)0;
  for (int q = 0; q < nq; ++q) {
    T r[NLV];
    child_resid<T, CF, NLV>(A, x, b, (unsigned)child[q * NC + C], k0, r);
#pragma unroll
    for (int kk = 0; kk < NLV; ++kk) acc[kk] = acc[kk] + r[kk];
  }
#pragma unroll
  for (int kk = 0; kk < NLV; ++kk)
    if (kk < kn) bc[(size_t)(k0 + kk) * NC + C] = acc[kk];
}

// Thread = (child slot q, coarse column C, chunk of KR levels): the four
// slots of a coarse column are adjacent lanes, so a warp reads its eight
// coarse columns' children (two rows of fine columns on a structured mesh)
// with every child's load chain in flight at once; lane q = 0 gathers the
// other slots' residuals by shuffle and sums them in slot order.  Every
// lane of a warp runs the same trips (the loop bound is rounded up to the
// warp), so the shuffles see all 32 lanes.
template <class T, bool CF>
__global__ void __launch_bounds__(256) k_helm_resid_restrict(HelmArgs<T> A,
                                                             const T* __restrict__ x,
                                                             const T* __restrict__ b,
                                                             T* __restrict__ bc,
                                                             const int* __restrict__ child,
                                                             int ncoarse, int nq) {
  grid_dep_wait();
  const unsigned NC = ncoarse;
  const int nchunk = (A.nl + KR - 1) / KR;
  const unsigned total = NC * (unsigned)nchunk * 4u;
  const unsigned trips = (total + 31u) & ~31u;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < trips; t += gridDim.x * blockDim.x) {
    const unsigned g = t >> 2, q = t & 3u;
    const unsigned kc = g / NC, C = g - kc * NC;
    const int k0 = (int)kc * KR;
    T r[KR];
#pragma unroll
    for (int kk = 0; kk < KR; ++kk) r[kk] = (T)0;
    if (t < total && q < (unsigned)nq)
      child_resid<T, CF, KR>(A, x, b, (unsigned)child[q * NC + C], k0, r);
#pragma unroll
    for (int kk = 0; kk < KR; ++kk) {
      const T r1 = __shfl_down_sync(0xffffffffu, r[kk], 1);
      const T r2 = __shfl_down_sync(0xffffffffu, r[kk], 2);
      const T r3 = __shfl_down_sync(0xffffffffu, r[kk], 3);
      if (q == 0 && t < total && kk < A.nl - k0) {
        T acc = (T)0;
        acc = acc + r[kk];
        if (nq > 1) acc = acc + r1;
        if (nq > 2) acc = acc + r2;
        if (nq > 3) acc = acc + r3;
        bc[(size_t)(k0 + kk) * NC + C] = acc;
      }
    }
  }
}

// ------------------------------------------------ structured panel kernels
// On a structured cubed-sphere mesh (lfg_mesh_create detects it) every cell
// off a panel's border finds its neighbours by arithmetic: side f of column
// c links to c + base[(f + roll) & 3], base = {-1, +n, +1, -n}.  The panel
// kernels give a thread V adjacent columns of one level (FP32 V = 4, FP64
// V = 2: 16-byte loads and stores of every column-aligned array) with no
// index load before its data loads.  Each panel row's first and last
// kPanelMargin columns and its first and last rows (the mesh's border
// groups) read their neighbour ids from the links table, still with vector
// loads of their own arrays, in the threads just before the same level's
// interior ones, so that a border group and the interior groups beside it
// share their sectors in L2.  The results equal the per-column kernels'
// element by element: the same operations in the same order.
struct PanelArgs {
  int n;             // cells per panel side
  unsigned roll;     // 2 bits per panel
  const int* edge;   // first columns of the border groups
  int edge_count;
};

// Side f's coupling for V adjacent interior columns c0.. of level k, at
// index i0 = k*N + c0 of the per-side arrays.  CF: sides f >= 2 are read as
// they are; a side f < 2 reads its neighbour's side f + 2 at the offset its
// roll gives (code g: 0 -> -1, 1 -> +n, 2 -> +1, 3 -> -n), from the vector
// of side f + 2 already loaded (g even: shifted by one, plus one value past
// the group's end) or from the row above or below (g odd).
template <bool CF, class T, int V>
__device__ __forceinline__ void panel_couplings(const HelmArgs<T>& A, size_t plane, size_t i0,
                                                int n, int roll, T (&hv)[4][V]) {
  if constexpr (!CF) {
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const Vec<T, V> q = vld<true, T, V>(A.h + f * plane + i0);
#pragma unroll
      for (int v = 0; v < V; ++v) hv[f][v] = q.e[v];
    }
  } else {
#pragma unroll
    for (int f = 2; f < 4; ++f) {
      const Vec<T, V> q = vld<false, T, V>(A.h + f * plane + i0);
#pragma unroll
      for (int v = 0; v < V; ++v) hv[f][v] = q.e[v];
    }
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      const int g = (f + roll) & 3;
      const T* hp = A.h + (f + 2) * plane + i0;
      const Vec<T, V> row = vld<false, T, V>(hp + (g == 1 ? n : g == 3 ? -n : 0));
      const T edge = hp[g == 0 ? -1 : V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T left = v > 0 ? hv[f + 2][v - 1] : edge;
        const T right = v < V - 1 ? hv[f + 2][v + 1] : edge;
        hv[f][v] = g == 0 ? left : g == 2 ? right : row.e[v];
      }
    }
  }
}

// Outputs of V adjacent columns c0.. at levels k0 .. k0+KL-1 (kn of them
// below the top) from their neighbours' x (xn) and couplings (hv) and the
// columns' own x (xc), in the per-column code's order of operations.
template <class T, int V, int KL, int MODE, bool DOT, bool HASW>
__device__ __forceinline__ void panel_finish(const HelmArgs<T>& A, int k0, unsigned c0,
                                             const T* __restrict__ x,
                                             const T* __restrict__ b, T* __restrict__ y,
                                             const T* __restrict__ w,
                                             const Vec<T, V> (&xc)[KL],
                                             const T (&xn)[KL][4][V], const T (&hv)[KL][4][V],
                                             double& acc) {
  const unsigned N = A.ncol;
  const int nl = A.nl;
  const int kn = min(KL, nl - k0);
  Vec<T, V> out[KL];
  if constexpr (MODE == M_RHS) {
#pragma unroll
    for (int kk = 0; kk < KL; ++kk) {
      const size_t i0 = (size_t)min(k0 + kk, nl - 1) * N + c0;
      const Vec<T, V> bb = vld<true, T, V>(b + i0);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        T hs = (T)0;
#pragma unroll
        for (int f = 0; f < 4; ++f) hs = hs + hv[kk][f][v] * xn[kk][f][v];
        out[kk].e[v] = bb.e[v] + hs;
      }
    }
  } else {
    const Vec<T, V> xm = vld<false, T, V>(x + (size_t)max(k0 - 1, 0) * N + c0);
    const Vec<T, V> xp = vld<false, T, V>(x + (size_t)min(k0 + KL, nl - 1) * N + c0);
#pragma unroll
    for (int kk = 0; kk < KL; ++kk) {
      const int k = min(k0 + kk, nl - 1);
      const size_t i0 = (size_t)k * N + c0;
      const bool hm = k > 0, hp = k < nl - 1;
      const Vec<T, V> sb = vld<true, T, V>(A.sub + i0);
      const Vec<T, V> dg = vld<true, T, V>(A.diag + i0);
      const Vec<T, V> sp = vld<true, T, V>(A.sup + i0);
      const Vec<T, V>& below = kk == 0 ? xm : xc[kk > 0 ? kk - 1 : 0];
      const Vec<T, V>& above = kk == KL - 1 ? xp : xc[kk < KL - 1 ? kk + 1 : 0];
      Vec<T, V> bb, ww;
      if constexpr (MODE == M_RESID) bb = vld<true, T, V>(b + i0);
      if constexpr (DOT && HASW) ww = vld<false, T, V>(w + i0);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        T xv[4], hh[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          xv[f] = xn[kk][f][v];
          hh[f] = hv[kk][f][v];
        }
        T val = helm_row_v(sb.e[v], dg.e[v], sp.e[v], hh, below.e[v], xc[kk].e[v], above.e[v],
                           xv, hm, hp);
        if (MODE == M_RESID) val = bb.e[v] - val;
        out[kk].e[v] = val;
        if (DOT && kk < kn) acc += (double)val * (double)(HASW ? ww.e[v] : val);
      }
    }
  }
#pragma unroll
  for (int kk = 0; kk < KL; ++kk)
    if (kk < kn) vst<T, V>(y + (size_t)(k0 + kk) * N + c0, out[kk]);
}

// V adjacent interior columns c0.. of levels k0 ..: neighbours by arithmetic.
template <class T, int V, int KL, int MODE, bool DOT, bool HASW, bool CF>
__device__ __forceinline__ void panel_interior(const HelmArgs<T>& A, int n, int roll, int k0,
                                               unsigned c0, const T* __restrict__ x,
                                               const T* __restrict__ b, T* __restrict__ y,
                                               const T* __restrict__ w, double& acc) {
  const size_t plane = (size_t)A.nl * A.ncol;
  Vec<T, V> xc[KL];
  T hv[KL][4][V], xn[KL][4][V];
#pragma unroll
  for (int kk = 0; kk < KL; ++kk) {
    const size_t i0 = (size_t)min(k0 + kk, A.nl - 1) * A.ncol + c0;
    const T* xk = x + (i0 - c0);
    xc[kk] = vld<false, T, V>(xk + c0);
    const Vec<T, V> xu = vld<false, T, V>(xk + c0 - n);
    const Vec<T, V> xd = vld<false, T, V>(xk + c0 + n);
    const T xl = xk[c0 - 1], xr = xk[c0 + V];
    panel_couplings<CF>(A, plane, i0, n, roll, hv[kk]);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const int g = (f + roll) & 3;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T left = v > 0 ? xc[kk].e[v > 0 ? v - 1 : 0] : xl;
        const T right = v < V - 1 ? xc[kk].e[v < V - 1 ? v + 1 : 0] : xr;
        xn[kk][f][v] = g == 0 ? left : g == 2 ? right : g == 1 ? xd.e[v] : xu.e[v];
      }
    }
  }
  panel_finish<T, V, KL, MODE, DOT, HASW>(A, k0, c0, x, b, y, w, xc, xn, hv, acc);
}

// V adjacent columns c0.. of levels k0 .. on a panel's border: neighbour
// ids (and designated sides) through the links (hsrc) tables, loaded as
// V-wide vectors, then one gather per neighbour; the columns' own arrays
// as vectors.
template <class T, int V, int KL, int MODE, bool DOT, bool HASW, bool CF>
__device__ __forceinline__ void panel_border(const HelmArgs<T>& A, int k0, unsigned c0,
                                             const T* __restrict__ x, const T* __restrict__ b,
                                             T* __restrict__ y, const T* __restrict__ w,
                                             double& acc) {
  const unsigned N = A.ncol;
  const size_t plane = (size_t)A.nl * N;
  Vec<int, V> nb[4], fc[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    nb[f] = vld<false, int, V>(A.links + (size_t)f * N + c0);
    if (CF) fc[f] = vld<false, int, V>(A.hsrc + (size_t)f * N + c0);
  }
  Vec<T, V> xc[KL];
  T hv[KL][4][V], xn[KL][4][V];
#pragma unroll
  for (int kk = 0; kk < KL; ++kk) {
    const size_t L = (size_t)min(k0 + kk, A.nl - 1) * N;
    xc[kk] = vld<false, T, V>(x + L + c0);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      Vec<T, V> hq;
      if constexpr (!CF) hq = vld<true, T, V>(A.h + f * plane + L + c0);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        xn[kk][f][v] = x[L + nb[f].e[v]];
        if constexpr (CF) {
          const int code = fc[f].e[v];
          hv[kk][f][v] = A.h[(size_t)(code >> 29) * plane + L + (code & 0x1fffffff)];
        } else {
          hv[kk][f][v] = hq.e[v];
        }
      }
    }
  }
  panel_finish<T, V, KL, MODE, DOT, HASW>(A, k0, c0, x, b, y, w, xc, xn, hv, acc);
}

// The shape of a panel kernel's thread: V adjacent columns (16-byte
// loads) and KL levels; `on`: whether the element-parallel panel kernels
// are used for this kind at all.  FP64 keeps the per-column kernels: with
// its faces read through their designated sides they measured faster at
// C192x70 (apply 142 against 158 us, sweep right-hand side 127 against
// 134 us, residual + restriction 207 against 250 us).
template <class T>
struct PanelShape {
  static constexpr int V = 16 / (int)sizeof(T);
  static constexpr int KL = 1;
  static constexpr bool on = sizeof(T) == 4;
};

// Threads: for every chunk of KL levels, the border groups (kPanelMargin
// columns each, as kPanelMargin / V V-groups), then the interior V-groups
// of every panel row; a chunk's threads are one contiguous range, so a
// border group and its interior neighbours are read at about the same time.
template <class T, int MODE, bool DOT, bool HASW, bool CF>
__global__ void __launch_bounds__(256) k_helm_panel(HelmArgs<T> A, PanelArgs P,
                                                    const T* __restrict__ x,
                                                    const T* __restrict__ b, T* __restrict__ y,
                                                    const T* __restrict__ w, Red r) {
  grid_dep_wait();
  constexpr int V = PanelShape<T>::V, KL = PanelShape<T>::KL;
  constexpr unsigned SPLIT = kPanelMargin / V;
  const unsigned n = P.n;
  const unsigned rowg = (n - 2 * kPanelMargin) / V, prow = (n - 2) * rowg;
  const unsigned nbord = (unsigned)P.edge_count * SPLIT, per = nbord + 6 * prow;
  const unsigned total = per * (unsigned)((A.nl + KL - 1) / KL);
  double acc = 0.0;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned kc = t / per, u = t - kc * per;
    const int k0 = (int)kc * KL;
    if (u < nbord) {
      const unsigned c0 = (unsigned)P.edge[u / SPLIT] + (u % SPLIT) * V;
      panel_border<T, V, KL, MODE, DOT, HASW, CF>(A, k0, c0, x, b, y, w, acc);
    } else {
      const unsigned g = u - nbord;
      const unsigned p = g / prow, rem = g - p * prow, jr = rem / rowg, gi = rem - jr * rowg;
      const unsigned c0 = p * n * n + (jr + 1) * n + kPanelMargin + gi * V;
      panel_interior<T, V, KL, MODE, DOT, HASW, CF>(A, (int)n, (P.roll >> (2 * p)) & 3, k0, c0,
                                                    x, b, y, w, acc);
    }
  }
  if (DOT) red_finish(r, acc);
}

// Residual + restriction on structured meshes: a thread takes one interior
// coarse column (off its panel's border) and one level; its four children
// are two pairs of adjacent fine columns in two adjacent fine rows, so
// every fine array is read as 2-wide vectors, and the fine neighbours come
// from the rows above and below the pairs and one value on either side.
// The children's residuals are summed in the cell map's slot order (the
// per-panel placement qpos), as the per-coarse-column code does; the
// coarse border columns (cedge) run that code, one level each, in the
// threads just before the same level's interior ones.  No minimum of
// blocks per SM: a bound of four (64 registers a thread) spilled and
// measured 113.7 against 112.0 us at C192x70.
template <class T, bool CF>
__global__ void __launch_bounds__(256) k_helm_resid_restrict_panel(
    HelmArgs<T> A, PanelArgs P, const T* __restrict__ x, const T* __restrict__ b,
    T* __restrict__ bc, const int* __restrict__ child, int ncoarse, unsigned long long qpos,
    const int* __restrict__ cedge, int ncedge) {
  grid_dep_wait();
  const unsigned N = A.ncol, nf = P.n, nc = nf / 2, NC = ncoarse;
  const int nl = A.nl;
  const size_t plane = (size_t)nl * N;
  const unsigned ni = nc - 2, pint = ni * ni;
  const unsigned per = (unsigned)ncedge + 6 * pint;
  const unsigned total = per * (unsigned)nl;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned k = t / per, u = t - k * per;
    if (u < (unsigned)ncedge) {
      resid_restrict_col<T, CF, 1>(A, x, b, bc, child, NC, 4, (unsigned)cedge[u], (int)k);
      continue;
    }
    const unsigned g = u - ncedge;
    const unsigned p = g / pint, rem = g - p * pint, J = rem / ni + 1, I = rem - (J - 1) * ni + 1;
    const unsigned C = p * nc * nc + J * nc + I;
    const unsigned f0 = p * nf * nf + 2 * J * nf + 2 * I, f1 = f0 + nf;
    const int roll = (P.roll >> (2 * p)) & 3;
    const bool hm = k > 0, hp = k + 1 < (unsigned)nl;
    const size_t L = (size_t)k * N;
    const T* xk = x + L;
    // x: rows above, of and below the two pairs; one value either side
    const Vec<T, 2> xa = vld<false, T, 2>(xk + f0 - nf), x0 = vld<false, T, 2>(xk + f0),
                    x1 = vld<false, T, 2>(xk + f1), xb = vld<false, T, 2>(xk + f1 + nf);
    const T x0l = xk[f0 - 1], x0r = xk[f0 + 2], x1l = xk[f1 - 1], x1r = xk[f1 + 2];
    const Vec<T, 2> x0m = vld<false, T, 2>(x + (size_t)(hm ? k - 1 : k) * N + f0),
                    x1m = vld<false, T, 2>(x + (size_t)(hm ? k - 1 : k) * N + f1),
                    x0p = vld<false, T, 2>(x + (size_t)(hp ? k + 1 : k) * N + f0),
                    x1p = vld<false, T, 2>(x + (size_t)(hp ? k + 1 : k) * N + f1);
    // couplings of both rows (the rows are n apart: two one-row loads each)
    T hv0[4][2], hv1[4][2];
    panel_couplings<CF, T, 2>(A, plane, L + f0, (int)nf, roll, hv0);
    panel_couplings<CF, T, 2>(A, plane, L + f1, (int)nf, roll, hv1);
    const Vec<T, 2> sb0 = vld<true, T, 2>(A.sub + L + f0), sb1 = vld<true, T, 2>(A.sub + L + f1);
    const Vec<T, 2> dg0 = vld<true, T, 2>(A.diag + L + f0), dg1 = vld<true, T, 2>(A.diag + L + f1);
    const Vec<T, 2> sp0 = vld<true, T, 2>(A.sup + L + f0), sp1 = vld<true, T, 2>(A.sup + L + f1);
    const Vec<T, 2> b0 = vld<true, T, 2>(b + L + f0), b1 = vld<true, T, 2>(b + L + f1);
    // residual of child position pos = 2 dy + dx
    T res[4];
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        const Vec<T, 2>& xr = dy ? x1 : x0;
        const T left = dx ? xr.e[0] : (dy ? x1l : x0l);
        const T right = dx ? (dy ? x1r : x0r) : xr.e[1];
        const T down = dy ? xb.e[dx] : x1.e[dx];
        const T up = dy ? x0.e[dx] : xa.e[dx];
        T xn[4], hh[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          const int gg = (f + roll) & 3;
          xn[f] = gg == 0 ? left : gg == 2 ? right : gg == 1 ? down : up;
          hh[f] = dy ? hv1[f][dx] : hv0[f][dx];
        }
        const T v = helm_row_v(dy ? sb1.e[dx] : sb0.e[dx], dy ? dg1.e[dx] : dg0.e[dx],
                               dy ? sp1.e[dx] : sp0.e[dx], hh, dy ? x1m.e[dx] : x0m.e[dx],
                               xr.e[dx], dy ? x1p.e[dx] : x0p.e[dx], xn, hm, hp);
        res[2 * dy + dx] = (dy ? b1.e[dx] : b0.e[dx]) - v;
      }
    const unsigned code = (unsigned)(qpos >> (8 * p));
    T acc = (T)0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int pos = (code >> (2 * q)) & 3;
      acc = acc + (pos == 0 ? res[0] : pos == 1 ? res[1] : pos == 2 ? res[2] : res[3]);
    }
    bc[(size_t)k * NC + C] = acc;
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
  grid_dep_wait();
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
template <class T, bool XIN, int S, int LMAX, bool CF>
__global__ void __launch_bounds__(128) k_helm_sweep_seg(HelmArgs<T> A, const T* __restrict__ b,
                                                        const T* __restrict__ xin, T omega,
                                                        T* __restrict__ xout) {
  grid_dep_wait();
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

// Shape of the segmented sweep (S = 0: use the per-column kernels).  Meshes
// with fewer than two columns per resident thread slot of 128-thread blocks
// are segmented; the first shape whose threads cover one such slot per
// column-thread and whose segments fit is taken: fewer threads per column
// and longer segments measured faster than more of both (C48 x 70 FP32
// sweep 13.9 us at 4 x 18 against 16.0 at 8 x 12 registers; C24 x 70 8.1 us
// at 8 x 9 against 9.4 at 16 x 12).
inline SegShape seg_shape(lfg_ctx c, int ncol, int nl) {
  const long slots = (long)c->num_sms * 128;
  if ((long)ncol >= 2 * slots) return {0, 0};
  for (const SegShape& s : kSegShapes)
    if ((long)ncol * s.S >= slots && (nl + s.S - 1) / s.S <= s.LM) return s;
  for (const SegShape& s : kSegShapes)
    if ((nl + s.S - 1) / s.S <= s.LM) return s;
  return {0, 0};
}

// Coupling words per dof the kernels read: 4 per side, 2 through the
// designated sides.
inline double coupling_words(lfg_helm op) { return op->hsym ? 2.0 : 4.0; }

template <class T, bool XIN>
void launch_sweep_seg(lfg_ctx c, SegShape sh, HelmArgs<T> A, const T* b, const T* xin, T omega,
                      T* xout, double hwords) {
  const int cols = 128 / sh.S;
  const unsigned grid = (unsigned)((A.ncol + cols - 1) / cols);
  auto go = [&](auto cf) {
    constexpr bool CF = decltype(cf)::value;
    auto run = [&](auto k) { launch_pdl(c, k, grid, 128, 0, A, b, xin, omega, xout); };
    static_assert(sizeof(kSegShapes) / sizeof(SegShape) == 5, "one case per shape");
    if (sh.S == 4) run(k_helm_sweep_seg<T, XIN, kSegShapes[0].S, kSegShapes[0].LM, CF>);
    else if (sh.S == 8) run(k_helm_sweep_seg<T, XIN, kSegShapes[1].S, kSegShapes[1].LM, CF>);
    else if (sh.S == 16) run(k_helm_sweep_seg<T, XIN, kSegShapes[2].S, kSegShapes[2].LM, CF>);
    else if (sh.LM == 3) run(k_helm_sweep_seg<T, XIN, kSegShapes[3].S, kSegShapes[3].LM, CF>);
    else run(k_helm_sweep_seg<T, XIN, kSegShapes[4].S, kSegShapes[4].LM, CF>);
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
  launch_pdl(c, kern, (ncol + bs - 1) / bs, bs, (size_t)nl * bs * sizeof(T), ncol, nl, r, sub,
             inv, cp, xin, omega, xout);
  // r, inv, sub, c' read and x written; x_in with XIN
  after_launch(c, "helm_subst", sizeof(T) * (XIN ? 6 : 5) * (uint64_t)ncol * nl);
}

// The panel kernels apply when the mesh is a structured cubed sphere with
// an edge list, the operator's designated-side reads (if any) follow the
// panel pattern, and every field is 16-byte aligned (wrapped fields may
// not be).
template <class T>
bool panel_ok(lfg_helm op, std::initializer_list<const void*> ptrs) {
  if constexpr (!PanelShape<T>::on) {
    return false;
  } else {
    const lfg_mesh m = op->mesh;
    if (!m->pedge || (op->hsym && !m->pcf)) return false;
    for (const void* p : ptrs)
      if (p && reinterpret_cast<uintptr_t>(p) % 16 != 0) return false;
    return true;
  }
}

inline PanelArgs panel_args(lfg_helm op) {
  const lfg_mesh m = op->mesh;
  return PanelArgs{m->pn, m->proll, m->pedge, m->npedge};
}

// Threads of a panel kernel: every level's border and interior V-groups.
template <class T>
size_t panel_work(lfg_helm op) {
  const size_t n = op->mesh->pn, V = PanelShape<T>::V, KL = PanelShape<T>::KL;
  const size_t groups = 6 * (n - 2) * ((n - 2 * kPanelMargin) / V);
  return (groups + (size_t)op->mesh->npedge * (kPanelMargin / V)) * ((op->nl + KL - 1) / KL);
}

// y = A x / b - A x / b + H_off x through the panel kernel
template <class T, int MODE, bool DOT, bool HASW>
void launch_panel(lfg_helm op, const T* x, const T* b, T* y, const T* w, Red r) {
  if constexpr (PanelShape<T>::on) {  // only the shapes panel_ok admits are built
    lfg_ctx c = op->ctx;
    auto k = op->hsym ? k_helm_panel<T, MODE, DOT, HASW, true>
                      : k_helm_panel<T, MODE, DOT, HASW, false>;
    launch_pdl(c, k, occ_grid(c, (const void*)k, 256, panel_work<T>(op)), 256, 0,
               args_of<T>(op), panel_args(op), x, b, y, w, r);
  }
}

// r = b + H_off x (k_helm_rhs, or the panel kernel)
template <class T>
void launch_rhs(lfg_helm op, const T* x, const T* b, T* r) {
  lfg_ctx c = op->ctx;
  const size_t work = (size_t)op->ncol * ((op->nl + KC - 1) / KC);
  if (panel_ok<T>(op, {x, b, r}))
    launch_panel<T, M_RHS, false, false>(op, x, b, r, nullptr, Red{nullptr, nullptr, nullptr});
  else {
    auto rk = op->hsym ? k_helm_rhs<T, true> : k_helm_rhs<T, false>;
    launch_pdl(c, rk, occ_grid(c, (const void*)rk, 256, work), 256, 0, args_of<T>(op), x, b, r);
  }
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
  if (const SegShape sh = seg_shape(c, op->ncol, op->nl); sh.S) {
    const HelmArgs<T> A = args_of<T>(op);
    if (!x_in)
      launch_sweep_seg<T, false>(c, sh, A, (const T*)b->d, nullptr, om, (T*)x_out->d, 4.0);
    else
      launch_sweep_seg<T, true>(c, sh, A, (const T*)b->d, (const T*)x_in->d, om, (T*)x_out->d,
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
  if (panel_ok<T>(op, {x, b, y, w})) {
    launch_panel<T, RESID ? M_RESID : M_APPLY, DOT, HASW>(op, x, b, y, w, r);
    return;
  }
  const int bs = 256;
  const size_t work = (size_t)op->ncol * ((op->nl + KC - 1) / KC);
  auto k = op->hsym ? k_helm_apply<T, RESID, DOT, HASW, true>
                    : k_helm_apply<T, RESID, DOT, HASW, false>;
  launch_pdl(c, k, occ_grid(c, (const void*)k, bs, work), bs, 0, args_of<T>(op), x, b, y, w, r);
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

void helm_residual_lower(lfg_helm op, lfg_field r_out, lfg_field x, lfg_field b, int slot) {
  LFG_REQUIRE(op->kind == LFG_R_DOUBLE, "helm_residual_lower: the operator must be r_double");
  LFG_REQUIRE(r_out && r_out->kind == LFG_R_SINGLE && r_out->ncol == op->ncol &&
                  r_out->nlev == op->nl,
              "helm_residual_lower: r must be an r_single field of the operator's shape");
  check_field(op, x, "helm_residual_lower");
  check_field(op, b, "helm_residual_lower");
  LFG_REQUIRE(slot >= 0, "helm_residual_lower: a reduction slot is required");
  lfg_ctx c = op->ctx;
  const Red r = c->red(slot);
  const int bs = 256;
  const size_t work = (size_t)op->ncol * ((op->nl + KC - 1) / KC);
  auto k = op->hsym ? k_helm_apply<double, true, true, false, true, float>
                    : k_helm_apply<double, true, true, false, false, float>;
  launch_pdl(c, k, occ_grid(c, (const void*)k, bs, work), bs, 0, args_of<double>(op),
             (const double*)x->d, (const double*)b->d, (float*)r_out->d, (const double*)nullptr,
             r);
  // x, b, the three bands and the couplings read in FP64, r written in FP32
  after_launch(c, "helm_residual_lower",
               (uint64_t)((8 * (5 + coupling_words(op)) + 4) * (double)op->ncol * op->nl));
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
  // the panel form: structured fine mesh and 2x2 map, 16-byte aligned
  // fields, and at least 8 waves of coarse columns x levels (its thread runs
  // four children's load chains; on fewer waves the lane-per-child kernel
  // hides the latency better: 30 against 42 us at C96 -> C48, 7 against
  // 24 us at C48 -> C24, 117 against 113 us at C192 -> C96)
  const bool panel = (op->kind == LFG_R_SINGLE ? PanelShape<float>::on
                                               : PanelShape<double>::on) &&
                     ig->pnc > 0 && op->mesh->pn == 2 * ig->pnc &&
                     6.0 * ig->pnc * ig->pnc * op->nl >= 8.0 * c->num_sms * 2048 &&
                     !(op->hsym && !op->mesh->pcf) &&
                     reinterpret_cast<uintptr_t>(x->d) % 16 == 0 &&
                     reinterpret_cast<uintptr_t>(b->d) % 16 == 0;
  auto go = [&](auto tag) {
    using T = decltype(tag);
    if constexpr (PanelShape<T>::on) {
      if (panel) {
        const size_t ni = ig->pnc - 2;
        const size_t pwork = (6 * ni * ni + (size_t)ig->ncedge) * op->nl;
        auto k = op->hsym ? k_helm_resid_restrict_panel<T, true>
                          : k_helm_resid_restrict_panel<T, false>;
        const lfg_mesh m = op->mesh;
        launch_pdl(c, k, occ_grid(c, (const void*)k, bs, pwork), bs, 0, args_of<T>(op),
                   PanelArgs{m->pn, m->proll, nullptr, 0}, (const T*)x->d, (const T*)b->d,
                   (T*)bc->d, (const int*)ig->child, ig->ncoarse, ig->qpos,
                   (const int*)ig->cedge, ig->ncedge);
        return;
      }
    }
    auto k = op->hsym ? k_helm_resid_restrict<T, true> : k_helm_resid_restrict<T, false>;
    launch_pdl(c, k, occ_grid(c, (const void*)k, bs, 4 * work), bs, 0, args_of<T>(op),
               (const T*)x->d, (const T*)b->d, (T*)bc->d, (const int*)ig->child, ig->ncoarse,
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
    launch_pdl(c, k_prolong_add<double>, occ_grid(c, (const void*)k_prolong_add<double>, 256, work),
               256, 0, (double*)fine->d, (const double*)coarse->d, (const int*)ig->parent,
               ig->nfine, ig->ncoarse, fine->nlev);
  else
    launch_pdl(c, k_prolong_add<float>, occ_grid(c, (const void*)k_prolong_add<float>, 256, work),
               256, 0, (float*)fine->d, (const float*)coarse->d, (const int*)ig->parent,
               ig->nfine, ig->ncoarse, fine->nlev);
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

// Structured cubed-sphere numbering: 6 panels of n x n cells, n^2 = ncol/6,
// numbered row-major per panel, with every cell off the panel's border
// linked to c + base[(f + roll) & 3], base = {-1, +n, +1, -n}, for one roll
// per panel.  Sets m->pn, m->proll (and m->pcf when the interior's
// designated sides follow the same pattern); leaves pn = 0 otherwise.
static void detect_panels(lfg_mesh m, const int* links, const int* hsrc) {
  const long ncol = m->ncol;
  const long n = std::lround(std::sqrt((double)ncol / 6.0));
  if (n < 3 || 6 * n * n != ncol || n >= (1 << 14)) return;
  const int base[4] = {-1, (int)n, 1, -(int)n};
  unsigned roll_code = 0;
  bool cf = hsrc != nullptr;
  for (int p = 0; p < 6; ++p) {
    int roll = -1;
    for (long j = 1; j < n - 1; ++j)
      for (long i = 1; i < n - 1; ++i) {
        const long cc = p * n * n + j * n + i;
        if (roll < 0) {
          for (int r = 0; r < 4 && roll < 0; ++r) {
            bool all = true;
            for (int f = 0; f < 4; ++f) all &= links[4 * cc + f] - cc == base[(f + r) & 3];
            if (all) roll = r;
          }
          if (roll < 0) return;
        }
        for (int f = 0; f < 4; ++f) {
          const long nb = cc + base[(f + roll) & 3];
          if (links[4 * cc + f] != nb) return;
          if (cf) {
            const int want = f >= 2 ? (f << 29 | (int)cc) : ((f + 2) << 29 | (int)nb);
            cf = hsrc[(size_t)f * ncol + cc] == want;
          }
        }
      }
    roll_code |= (unsigned)roll << (2 * p);
  }
  m->pn = (int)n;
  m->proll = roll_code;
  m->pcf = cf;
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
    detect_panels(m, links, paired ? hsrc.data() : nullptr);
    // border groups of the panel kernels: the first column of every
    // kPanelMargin-wide group in rows 0 and n-1, and of the first and last
    // group of every other row
    std::vector<int> edge;
    if (m->pn % kPanelMargin == 0 && m->pn >= 3 * kPanelMargin) {
      const int n = m->pn;
      for (int p = 0; p < 6; ++p)
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; i += kPanelMargin)
            if (j == 0 || j == n - 1 || i == 0 || i == n - kPanelMargin)
              edge.push_back(p * n * n + j * n + i);
    }
    try {
      m->links = (int*)dmalloc(soa.size() * sizeof(int));
      upload(m->links, soa.data(), soa.size() * sizeof(int));
      if (paired) {
        m->hsrc = (int*)dmalloc(hsrc.size() * sizeof(int));
        upload(m->hsrc, hsrc.data(), hsrc.size() * sizeof(int));
      }
      if (!edge.empty()) {
        m->pedge = (int*)dmalloc(edge.size() * sizeof(int));
        upload(m->pedge, edge.data(), edge.size() * sizeof(int));
        m->npedge = (int)edge.size();
      }
    } catch (...) {
      dfree(m->links);
      dfree(m->hsrc);
      dfree(m->pedge);
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
  dfree(m->pedge);
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

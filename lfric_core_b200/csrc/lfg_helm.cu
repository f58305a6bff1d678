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
// Every kernel here is HBM-bandwidth bound (< 1 flop/byte).  One thread owns
// one column and walks its levels, so at every level a warp reads 32
// consecutive columns of each level-major array; the neighbour ids of a
// column are read once, not once per level.
#include "lfg_internal.cuh"

#include <algorithm>

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
};

template <class T>
HelmArgs<T> args_of(lfg_helm op) {
  return HelmArgs<T>{op->ncol, op->nl, (const T*)op->sub, (const T*)op->diag,
                     (const T*)op->sup, (const T*)op->h, op->mesh->links};
}

// (A x)(c,k) with the reference's order: T' row first (sub, diag, super,
// as the columnwise_op_app loop over j), then minus the W,S,E,N couplings.
template <class T>
__device__ __forceinline__ T helm_row(const HelmArgs<T>& A, size_t i, int k, T xm, T x0, T xp,
                                      const T (&xn)[4]) {
  const size_t plane = (size_t)A.nl * A.ncol;
  T acc = (T)0;
  if (k > 0) acc = acc + A.sub[i] * xm;
  acc = acc + A.diag[i] * x0;
  if (k < A.nl - 1) acc = acc + A.sup[i] * xp;
#pragma unroll
  for (int f = 0; f < 4; ++f) acc = acc - A.h[f * plane + i] * xn[f];
  return acc;
}

// y = A x (RESID: y = b - A x).  DOT: accumulate <y, w> (w null: <y, y>)
// into a deterministic reduction.
template <class T, bool RESID, bool DOT>
__global__ void __launch_bounds__(256) k_helm_apply(HelmArgs<T> A, const T* __restrict__ x,
                                                    const T* __restrict__ b, T* __restrict__ y,
                                                    const T* __restrict__ w, Red r) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double acc = 0.0;
  if (c < A.ncol) {
    const size_t N = A.ncol;
    int nb[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) nb[f] = A.links[f * N + c];
    T xm = (T)0, x0 = x[c], xp;
#pragma unroll 4
    for (int k = 0; k < A.nl; ++k) {
      const size_t i = (size_t)k * N + c;
      xp = (k + 1 < A.nl) ? x[i + N] : (T)0;
      T xn[4];
#pragma unroll
      for (int f = 0; f < 4; ++f) xn[f] = x[(size_t)k * N + nb[f]];
      T v = helm_row(A, i, k, xm, x0, xp, xn);
      if (RESID) v = b[i] - v;
      y[i] = v;
      if (DOT) {
        const T ww = w ? w[i] : v;
        acc += (double)v * (double)ww;
      }
      xm = x0;
      x0 = xp;
    }
  }
  if (DOT) red_finish(r, acc);
}

// One block-Jacobi column sweep of A x = b:
//   x_out = omega T'^{-1} (b + H_off x_in + kappa T' x_in),  kappa = 1/omega - 1,
// which equals x_in + omega T'^{-1} (b - A x_in).  XIN false: x_in = 0.
// PRO: x_in is the prolongation-corrected iterate x_in + P xc (P = add the
// parent's coarse value), formed on the fly.  c' of the Thomas forward sweep
// is kept in shared memory and d' in registers (DP_SMEM: also in shared
// memory); both are indexed by the unrolled level loop.
template <class T, int MAXNL, bool XIN, bool PRO, bool DP_SMEM>
__global__ void k_helm_smooth(HelmArgs<T> A, T omega, T kappa, const T* __restrict__ xin,
                              const T* __restrict__ b, T* __restrict__ xout,
                              const int* __restrict__ parent, const T* __restrict__ xc,
                              int ncoarse) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* cps = reinterpret_cast<T*>(smem_raw);
  T* dps = cps + MAXNL * blockDim.x;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.ncol) return;
  const int nl = A.nl;
  const size_t N = A.ncol;
  const size_t plane = (size_t)nl * N;
  const int t = threadIdx.x, bs = blockDim.x;
  int nb[4], pn[4] = {0, 0, 0, 0}, pc = 0;
  if (XIN) {
#pragma unroll
    for (int f = 0; f < 4; ++f) nb[f] = A.links[f * N + c];
    if (PRO) {
      pc = parent[c];
#pragma unroll
      for (int f = 0; f < 4; ++f) pn[f] = parent[nb[f]];
    }
  }
  auto X = [&](int col, int pcol, int k) -> T {
    T v = xin[(size_t)k * N + col];
    if (PRO) v = v + xc[(size_t)k * ncoarse + pcol];
    return v;
  };
  T dp[DP_SMEM ? 1 : MAXNL];
  T cprev = (T)0, dprev = (T)0;
  T xm = (T)0, x0 = (T)0, xp = (T)0;
  if (XIN) x0 = X(c, pc, 0);
#pragma unroll
  for (int k = 0; k < MAXNL; ++k) {
    if (k < nl) {
      const size_t i = (size_t)k * N + c;
      const T sb = A.sub[i], dg = A.diag[i], sp = A.sup[i];
      T rhs = b[i];
      if (XIN) {
        xp = (k + 1 < nl) ? X(c, pc, k + 1) : (T)0;
        T hs = (T)0;
#pragma unroll
        for (int f = 0; f < 4; ++f) hs = hs + A.h[f * plane + i] * X(nb[f], pn[f], k);
        T tx = (T)0;
        if (k > 0) tx = tx + sb * xm;
        tx = tx + dg * x0;
        if (k < nl - 1) tx = tx + sp * xp;
        rhs = rhs + hs + kappa * tx;
      }
      T inv, cpk, dpk;
      if (k == 0) {
        inv = (T)1 / dg;
        cpk = inv * sp;
        dpk = inv * rhs;
      } else {
        inv = (T)1 / (dg - sb * cprev);
        cpk = (k < nl - 1) ? inv * sp : (T)0;
        dpk = inv * (rhs - sb * dprev);
      }
      cps[k * bs + t] = cpk;
      if (DP_SMEM) dps[k * bs + t] = dpk; else dp[DP_SMEM ? 0 : k] = dpk;
      cprev = cpk;
      dprev = dpk;
      xm = x0;
      x0 = xp;
    }
  }
  T znext = (T)0;
#pragma unroll
  for (int k = MAXNL - 1; k >= 0; --k) {
    if (k < nl) {
      T z = DP_SMEM ? dps[k * bs + t] : dp[DP_SMEM ? 0 : k];
      if (k < nl - 1) z = z - cps[k * bs + t] * znext;
      znext = z;
      xout[(size_t)k * N + c] = omega * z;
    }
  }
}

// bc(C,k) = sum over the children q (y outer, x inner) of (b - A x)(child,k):
// residual fused with restrict_mass_w3 (sci_restrict_mass_w3_kernel_mod.F90:126-179).
template <class T>
__global__ void __launch_bounds__(128) k_helm_resid_restrict(HelmArgs<T> A,
                                                             const T* __restrict__ x,
                                                             const T* __restrict__ b,
                                                             T* __restrict__ bc,
                                                             const int* __restrict__ child,
                                                             int ncoarse, int nq) {
  const int C = blockIdx.x * blockDim.x + threadIdx.x;
  if (C >= ncoarse) return;
  const size_t N = A.ncol;
  int ch[4], nb[4][4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    ch[q] = q < nq ? child[q * ncoarse + C] : 0;
#pragma unroll
    for (int f = 0; f < 4; ++f) nb[q][f] = A.links[f * N + ch[q]];
  }
#pragma unroll 2
  for (int k = 0; k < A.nl; ++k) {
    T acc = (T)0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (q < nq) {
        const size_t i = (size_t)k * N + ch[q];
        const T xm = k > 0 ? x[i - N] : (T)0;
        const T xp = k + 1 < A.nl ? x[i + N] : (T)0;
        T xn[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) xn[f] = x[(size_t)k * N + nb[q][f]];
        acc = acc + (b[i] - helm_row(A, i, k, xm, x[i], xp, xn));
      }
    }
    bc[(size_t)k * ncoarse + C] = acc;
  }
}

// fine(c,k) += coarse(parent(c),k)   (prolong_scalar_unweighted on W3)
template <class T>
__global__ void k_prolong_add(T* __restrict__ fine, const T* __restrict__ coarse,
                              const int* __restrict__ parent, int nfine, int ncoarse, int nl) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nfine) return;
  const int p = parent[c];
  for (int k = 0; k < nl; ++k)
    fine[(size_t)k * nfine + c] = fine[(size_t)k * nfine + c] + coarse[(size_t)k * ncoarse + p];
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

// dynamic shared memory one block may use (B200: up to 227 KB per block)
constexpr size_t kSmemCap = 200 * 1024;

int smooth_block(int ncol, int nsm) {
  // spread small meshes over every SM; 128 threads per block for large ones
  int per = (ncol + nsm - 1) / nsm;
  int bs = ((per + 31) / 32) * 32;
  return std::max(32, std::min(128, bs));
}

template <class T, int MAXNL, bool XIN, bool PRO, bool DPS>
void launch_smooth_t(lfg_helm op, T omega, T kappa, const T* xin, const T* b, T* xout,
                     const int* parent, const T* xc, int ncoarse) {
  lfg_ctx c = op->ctx;
  constexpr size_t per_thread = (size_t)MAXNL * sizeof(T) * (DPS ? 2 : 1);
  constexpr int max_bs = (int)std::min<size_t>(128, (kSmemCap / per_thread) / 32 * 32);
  static_assert(max_bs >= 32, "smoother column too tall for shared memory");
  const int bs = std::min(max_bs, smooth_block(op->ncol, c->num_sms));
  const size_t smem = per_thread * bs;
  auto kern = k_helm_smooth<T, MAXNL, XIN, PRO, DPS>;
  static bool attr_set = false;
  if (!attr_set) {
    LFG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(per_thread * max_bs)));
    attr_set = true;
  }
  const int grid = (op->ncol + bs - 1) / bs;
  kern<<<grid, bs, smem, c->stream>>>(args_of<T>(op), omega, kappa, xin, b, xout, parent, xc,
                                      ncoarse);
  after_launch(c, "helm_smooth");
}

template <class T, bool XIN, bool PRO>
void launch_smooth_nl(lfg_helm op, T omega, T kappa, const T* xin, const T* b, T* xout,
                      const int* parent, const T* xc, int ncoarse) {
  const int nl = op->nl;
  if (nl <= 16)
    launch_smooth_t<T, 16, XIN, PRO, false>(op, omega, kappa, xin, b, xout, parent, xc, ncoarse);
  else if (nl <= 32)
    launch_smooth_t<T, 32, XIN, PRO, false>(op, omega, kappa, xin, b, xout, parent, xc, ncoarse);
  else if (nl <= 72)
    launch_smooth_t<T, 72, XIN, PRO, false>(op, omega, kappa, xin, b, xout, parent, xc, ncoarse);
  else if (nl <= 128)
    launch_smooth_t<T, 128, XIN, PRO, true>(op, omega, kappa, xin, b, xout, parent, xc, ncoarse);
  else
    throw Error(LFG_ERR_ARG, "helm_smooth: more than 128 levels is not supported");
}

template <class T>
void smooth_t(lfg_helm op, double omega, lfg_field x_in, lfg_field b, lfg_field x_out,
              lfg_intergrid ig, lfg_field xc) {
  const T om = (T)omega;
  const T kap = (T)(1.0 / omega - 1.0);
  const T* xi = x_in ? (const T*)x_in->d : nullptr;
  if (!x_in)
    launch_smooth_nl<T, false, false>(op, om, kap, nullptr, (const T*)b->d, (T*)x_out->d,
                                      nullptr, nullptr, 0);
  else if (!ig)
    launch_smooth_nl<T, true, false>(op, om, kap, xi, (const T*)b->d, (T*)x_out->d, nullptr,
                                     nullptr, 0);
  else
    launch_smooth_nl<T, true, true>(op, om, kap, xi, (const T*)b->d, (T*)x_out->d, ig->parent,
                                    (const T*)xc->d, ig->ncoarse);
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
  const int bs = 128, grid = (op->ncol + bs - 1) / bs;
  LFG_REQUIRE(grid <= kMaxRedBlocks || slot < 0, "helm_apply: mesh too large for a fused dot");
  Red r = slot >= 0 ? c->red(slot) : Red{nullptr, nullptr, nullptr};
  if (op->kind == LFG_R_DOUBLE) {
    using T = double;
    if (slot >= 0)
      k_helm_apply<T, false, true><<<grid, bs, 0, c->stream>>>(args_of<T>(op), (const T*)x->d, nullptr, (T*)y->d, dot_with ? (const T*)dot_with->d : nullptr, r);
    else
      k_helm_apply<T, false, false><<<grid, bs, 0, c->stream>>>(args_of<T>(op), (const T*)x->d, nullptr, (T*)y->d, nullptr, r);
  } else {
    using T = float;
    if (slot >= 0)
      k_helm_apply<T, false, true><<<grid, bs, 0, c->stream>>>(args_of<T>(op), (const T*)x->d, nullptr, (T*)y->d, dot_with ? (const T*)dot_with->d : nullptr, r);
    else
      k_helm_apply<T, false, false><<<grid, bs, 0, c->stream>>>(args_of<T>(op), (const T*)x->d, nullptr, (T*)y->d, nullptr, r);
  }
  after_launch(c, "helm_apply");
}

void helm_residual(lfg_helm op, lfg_field r_out, lfg_field x, lfg_field b, int slot) {
  check_field(op, r_out, "helm_residual");
  check_field(op, x, "helm_residual");
  check_field(op, b, "helm_residual");
  lfg_ctx c = op->ctx;
  const int bs = 128, grid = (op->ncol + bs - 1) / bs;
  LFG_REQUIRE(grid <= kMaxRedBlocks || slot < 0, "helm_residual: mesh too large for a fused norm");
  Red r = slot >= 0 ? c->red(slot) : Red{nullptr, nullptr, nullptr};
  if (op->kind == LFG_R_DOUBLE) {
    using T = double;
    if (slot >= 0)
      k_helm_apply<T, true, true><<<grid, bs, 0, c->stream>>>(args_of<T>(op), (const T*)x->d, (const T*)b->d, (T*)r_out->d, nullptr, r);
    else
      k_helm_apply<T, true, false><<<grid, bs, 0, c->stream>>>(args_of<T>(op), (const T*)x->d, (const T*)b->d, (T*)r_out->d, nullptr, r);
  } else {
    using T = float;
    if (slot >= 0)
      k_helm_apply<T, true, true><<<grid, bs, 0, c->stream>>>(args_of<T>(op), (const T*)x->d, (const T*)b->d, (T*)r_out->d, nullptr, r);
    else
      k_helm_apply<T, true, false><<<grid, bs, 0, c->stream>>>(args_of<T>(op), (const T*)x->d, (const T*)b->d, (T*)r_out->d, nullptr, r);
  }
  after_launch(c, "helm_residual");
}

void helm_smooth(lfg_helm op, double omega, lfg_field x_in, lfg_field b, lfg_field x_out,
                 lfg_intergrid ig, lfg_field xc) {
  check_field(op, b, "helm_smooth");
  check_field(op, x_out, "helm_smooth");
  if (x_in) {
    check_field(op, x_in, "helm_smooth");
    LFG_REQUIRE(x_in->d != x_out->d, "helm_smooth: x_out may not alias x_in");
  }
  if (ig) {
    LFG_REQUIRE(x_in && xc && ig->nfine == op->ncol && xc->ncol == ig->ncoarse &&
                    xc->nlev == op->nl && xc->kind == op->kind,
                "helm_smooth: bad prolongation arguments");
  }
  if (op->kind == LFG_R_DOUBLE) smooth_t<double>(op, omega, x_in, b, x_out, ig, xc);
  else smooth_t<float>(op, omega, x_in, b, x_out, ig, xc);
}

void helm_residual_restrict(lfg_helm op, lfg_intergrid ig, lfg_field x, lfg_field b,
                            lfg_field bc) {
  check_field(op, x, "residual_restrict");
  check_field(op, b, "residual_restrict");
  LFG_REQUIRE(ig->nfine == op->ncol && bc->ncol == ig->ncoarse && bc->nlev == op->nl &&
                  bc->kind == op->kind && ig->nx * ig->ny <= 4,
              "residual_restrict: bad coarse field");
  lfg_ctx c = op->ctx;
  const int bs = 128, grid = (ig->ncoarse + bs - 1) / bs;
  if (op->kind == LFG_R_DOUBLE)
    k_helm_resid_restrict<double><<<grid, bs, 0, c->stream>>>(args_of<double>(op), (const double*)x->d, (const double*)b->d, (double*)bc->d, ig->child, ig->ncoarse, ig->nx * ig->ny);
  else
    k_helm_resid_restrict<float><<<grid, bs, 0, c->stream>>>(args_of<float>(op), (const float*)x->d, (const float*)b->d, (float*)bc->d, ig->child, ig->ncoarse, ig->nx * ig->ny);
  after_launch(c, "resid_restrict");
}

void prolong_add(lfg_intergrid ig, lfg_field fine, lfg_field coarse) {
  LFG_REQUIRE(fine->ncol == ig->nfine && coarse->ncol == ig->ncoarse &&
                  fine->nlev == coarse->nlev && fine->kind == coarse->kind,
              "prolong_add: bad fields");
  lfg_ctx c = fine->ctx;
  const int bs = 128, grid = (ig->nfine + bs - 1) / bs;
  if (fine->kind == LFG_R_DOUBLE)
    k_prolong_add<double><<<grid, bs, 0, c->stream>>>((double*)fine->d, (const double*)coarse->d, ig->parent, ig->nfine, ig->ncoarse, fine->nlev);
  else
    k_prolong_add<float><<<grid, bs, 0, c->stream>>>((float*)fine->d, (const float*)coarse->d, ig->parent, ig->nfine, ig->ncoarse, fine->nlev);
  after_launch(c, "prolong_add");
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
  } catch (...) {
    dfree(op->sub); dfree(op->diag); dfree(op->sup); dfree(op->h);
    delete op;
    throw;
  }
  return op;
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
    lfg_mesh m = new lfg_mesh_s;
    m->ctx = c;
    m->ncol = ncol;
    m->h_links.assign(links, links + (size_t)4 * ncol);
    try {
      m->links = (int*)dmalloc(soa.size() * sizeof(int));
      upload(m->links, soa.data(), soa.size() * sizeof(int));
    } catch (...) {
      dfree(m->links);
      delete m;
      throw;
    }
    *out = m;
  });
}

int lfg_mesh_destroy(lfg_mesh m) {
  if (!m) return LFG_OK;
  dfree(m->links);
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
  delete op;
  return LFG_OK;
}

int lfg_helm_apply(lfg_helm op, lfg_field y, lfg_field x) {
  if (!op) return LFG_ERR_ARG;
  return guard(op->ctx, [&] { helm_apply(op, y, x, nullptr, -1); });
}

int lfg_helm_smooth(lfg_helm op, double omega, lfg_field x_in, lfg_field b, lfg_field x_out) {
  if (!op) return LFG_ERR_ARG;
  return guard(op->ctx, [&] { helm_smooth(op, omega, x_in, b, x_out, nullptr, nullptr); });
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
      LFG_CUDA(cudaStreamSynchronize(c->stream));
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
      if (src->kind != kind) after_launch(c, "convert");
    }
    LFG_CUDA(cudaStreamSynchronize(c->stream));
    *out = d;
  });
}

}  // extern "C"

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
// into a deterministic reduction.  Grid-stride over all (level, column)
// elements: no recurrence, so every element is independent and the loads of
// many elements are in flight at once.
template <class T, bool RESID, bool DOT>
__global__ void __launch_bounds__(256) k_helm_apply(HelmArgs<T> A, const T* __restrict__ x,
                                                    const T* __restrict__ b, T* __restrict__ y,
                                                    const T* __restrict__ w, Red r) {
  const unsigned N = A.ncol;
  const unsigned total = N * (unsigned)A.nl;
  double acc = 0.0;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const unsigned k = i / N, c = i - k * N;
    T xn[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) xn[f] = x[(size_t)k * N + A.links[f * N + c]];
    const T xm = k > 0 ? x[i - N] : (T)0;
    const T xp = k + 1 < (unsigned)A.nl ? x[i + N] : (T)0;
    T v = helm_row(A, i, (int)k, xm, x[i], xp, xn);
    if (RESID) v = b[i] - v;
    y[i] = v;
    if (DOT) {
      const T ww = w ? w[i] : v;
      acc += (double)v * (double)ww;
    }
  }
  if (DOT) red_finish(r, acc);
}

// One block-Jacobi column sweep of A x = b:
//   x_out = omega T'^{-1} (b + H_off x_in) + (1 - omega) x_in,
// which equals x_in + omega T'^{-1} (b - A x_in).  XIN false: x_in = 0.
// PRO: x_in is the prolongation-corrected iterate x_in + P xc (P adds the
// parent's coarse value), formed on the fly and never stored.
//
// A block owns a tile of tc consecutive columns.  Phase 1: all threads load
// the tile's x, b and bands for every level into shared memory (coalesced
// rows of tc columns, many loads in flight) and form the right-hand side
// with the neighbour couplings.  Phase 2: one thread per column runs the
// Thomas recurrence of columnwise_op_appinv out of shared memory (c' over
// the super-diagonal, d' and then the solution over the right-hand side).
// Phase 3: coalesced write of the relaxed update.  Shared memory holds
// 5 * nl * tc values.
template <class T, bool XIN, bool PRO>
__global__ void __launch_bounds__(256) k_helm_smooth(HelmArgs<T> A, T omega,
                                                     const T* __restrict__ xin,
                                                     const T* __restrict__ b,
                                                     T* __restrict__ xout,
                                                     const int* __restrict__ parent,
                                                     const T* __restrict__ xc, int ncoarse,
                                                     int tc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nl = A.nl;
  const unsigned N = A.ncol;
  const size_t plane = (size_t)nl * N;
  const int tile = nl * tc;
  T* sx = reinterpret_cast<T*>(smem_raw);
  T* sr = sx + tile;
  T* ssub = sr + tile;
  T* sdg = ssub + tile;
  T* ssp = sdg + tile;
  const unsigned c0 = blockIdx.x * tc;
  auto X = [&](unsigned col, unsigned k) -> T {
    T v = xin[(size_t)k * N + col];
    if (PRO) v = v + xc[(size_t)k * ncoarse + parent[col]];
    return v;
  };
  // phase 1
#pragma unroll 4
  for (int e = threadIdx.x; e < tile; e += blockDim.x) {
    const int k = e / tc, j = e - k * tc;
    const unsigned c = c0 + j;
    if (c >= N) continue;
    const size_t i = (size_t)k * N + c;
    ssub[e] = A.sub[i];
    sdg[e] = A.diag[i];
    ssp[e] = A.sup[i];
    T rhs = b[i];
    if (XIN) {
      sx[e] = X(c, k);
      T hs = (T)0;
#pragma unroll
      for (int f = 0; f < 4; ++f) hs = hs + A.h[f * plane + i] * X(A.links[f * N + c], k);
      rhs = rhs + hs;
    }
    sr[e] = rhs;
  }
  __syncthreads();
  // phase 2: Thomas, column j of the tile
  for (int j = threadIdx.x; j < tc; j += blockDim.x) {
    if (c0 + j >= N) break;
    T cprev = (T)0, dprev = (T)0;
    for (int k = 0; k < nl; ++k) {
      const int e = k * tc + j;
      const T a1 = ssub[e], a2 = sdg[e], a3 = ssp[e];
      T inv, cpk, dpk;
      if (k == 0) {
        inv = (T)1 / a2;
        cpk = inv * a3;
        dpk = inv * sr[e];
      } else {
        inv = (T)1 / (a2 - a1 * cprev);
        cpk = (k < nl - 1) ? inv * a3 : (T)0;
        dpk = inv * (sr[e] - a1 * dprev);
      }
      ssp[e] = cpk;
      sr[e] = dpk;
      cprev = cpk;
      dprev = dpk;
    }
    T znext = (T)0;
    for (int k = nl - 1; k >= 0; --k) {
      const int e = k * tc + j;
      T z = sr[e];
      if (k < nl - 1) z = z - ssp[e] * znext;
      sr[e] = z;
      znext = z;
    }
  }
  __syncthreads();
  // phase 3
  const T om1 = (T)1 - omega;
  for (int e = threadIdx.x; e < tile; e += blockDim.x) {
    const int k = e / tc, j = e - k * tc;
    const unsigned c = c0 + j;
    if (c >= N) continue;
    T v = omega * sr[e];
    if (XIN) v = v + om1 * sx[e];
    xout[(size_t)k * N + c] = v;
  }
}

// bc(C,k) = sum over the children q (y outer, x inner) of (b - A x)(child,k):
// residual fused with restrict_mass_w3 (sci_restrict_mass_w3_kernel_mod.F90:126-179).
// One thread per coarse element (level, coarse column).
template <class T>
__global__ void __launch_bounds__(256) k_helm_resid_restrict(HelmArgs<T> A,
                                                             const T* __restrict__ x,
                                                             const T* __restrict__ b,
                                                             T* __restrict__ bc,
                                                             const int* __restrict__ child,
                                                             int ncoarse, int nq) {
  const unsigned NC = ncoarse, N = A.ncol;
  const unsigned total = NC * (unsigned)A.nl;
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const unsigned k = e / NC, C = e - k * NC;
    T acc = (T)0;
    for (int q = 0; q < nq; ++q) {
      const unsigned c = child[q * NC + C];
      const size_t i = (size_t)k * N + c;
      const T xm = k > 0 ? x[i - N] : (T)0;
      const T xp = k + 1 < (unsigned)A.nl ? x[i + N] : (T)0;
      T xn[4];
#pragma unroll
      for (int f = 0; f < 4; ++f) xn[f] = x[(size_t)k * N + A.links[f * N + c]];
      acc = acc + (b[i] - helm_row(A, i, (int)k, xm, x[i], xp, xn));
    }
    bc[e] = acc;
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

// Columns per smoother tile: as wide as shared memory allows (at most 64),
// narrowed on small meshes so that every SM receives blocks.
int smooth_tile(int ncol, int nl, size_t elem, int nsm) {
  int tc = 64;
  while (tc > 8 && (size_t)5 * nl * tc * elem > kSmemCap) tc /= 2;
  while (tc > 8 && (ncol + tc - 1) / tc < 2 * nsm) tc /= 2;
  return tc;
}

template <class T, bool XIN, bool PRO>
void launch_smooth_t(lfg_helm op, T omega, const T* xin, const T* b, T* xout,
                     const int* parent, const T* xc, int ncoarse) {
  lfg_ctx c = op->ctx;
  const int tc = smooth_tile(op->ncol, op->nl, sizeof(T), c->num_sms);
  const size_t smem = (size_t)5 * op->nl * tc * sizeof(T);
  if (smem > kSmemCap)
    throw Error(LFG_ERR_ARG, "helm_smooth: column too tall for the shared-memory tile");
  auto kern = k_helm_smooth<T, XIN, PRO>;
  static bool attr_set = false;
  if (!attr_set) {
    LFG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kSmemCap));
    attr_set = true;
  }
  const int grid = (op->ncol + tc - 1) / tc;
  kern<<<grid, 256, smem, c->stream>>>(args_of<T>(op), omega, xin, b, xout, parent, xc,
                                       ncoarse, tc);
  after_launch(c, "helm_smooth");
}

template <class T>
void smooth_t(lfg_helm op, double omega, lfg_field x_in, lfg_field b, lfg_field x_out,
              lfg_intergrid ig, lfg_field xc) {
  const T om = (T)omega;
  const T* xi = x_in ? (const T*)x_in->d : nullptr;
  if (!x_in)
    launch_smooth_t<T, false, false>(op, om, nullptr, (const T*)b->d, (T*)x_out->d, nullptr,
                                     nullptr, 0);
  else if (!ig)
    launch_smooth_t<T, true, false>(op, om, xi, (const T*)b->d, (T*)x_out->d, nullptr,
                                    nullptr, 0);
  else
    launch_smooth_t<T, true, true>(op, om, xi, (const T*)b->d, (T*)x_out->d, ig->parent,
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
  const int bs = 256, grid = c->stream_grid((size_t)op->ncol * op->nl, bs);
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
  const int bs = 256, grid = c->stream_grid((size_t)op->ncol * op->nl, bs);
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
  const int bs = 256, grid = c->stream_grid((size_t)ig->ncoarse * op->nl, bs);
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

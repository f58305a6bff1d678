// Locally-assembled (LMA) operators: element-matrix applies on continuous
// and discontinuous spaces, the transposed apply, the diagonal, and the
// per-cell bilinear form used by the adjoint.
//
// Drop-ins for components/science/source/kernel/algebra/
//   matrix_vector_kernel_mod.F90:107-140            (LFG_LMA_INC)
//   dg_matrix_vector_kernel_mod.F90:113-154         (LFG_LMA_WRITE)
//   transpose_matrix_vector_kernel_mod.F90:107-144  (LFG_LMA_TRANSPOSE)
//   sci_mm_diagonal_kernel_mod.F90:99-127           (lfg_lma_diagonal)
//
// The reference scatters each cell's y_e = A_e x_e into the shared dofs
// (GH_INC) inside a coloured OpenMP loop.  Here the applies run in two
// phases: k_lma_local streams the element matrices once, coalesced, and
// writes each cell-layer's local products; k_lma_gather_tab then has every
// output dof GATHER the products of its (cell, local dof) incidences, in
// cell order, through a padded incidence table, so the result is
// deterministic without atomics.  Operators whose incidence lists are wider
// than 16 keep the one-pass gathers (k_lma_apply, k_lma_apply_t), which
// walk the incidence lists directly.  Element matrices are stored
// [df_to][df_from][layer][cell]: at fixed (df, df2, layer) consecutive cells
// are contiguous.  Algorithmic traffic: w*ndf_to*ndf_from bytes per cell and
// layer for the matrix plus one read of x and one write of y.
#include "lfg_internal.cuh"

#include <algorithm>
#include <numeric>

using namespace lfg;

namespace {

template <class T>
struct LmaArgs {
  int ncell, nl, ndf_to, ndf_from;
  int nent_to, nlev_to, nent_from, nlev_from;
  const T* __restrict__ a;
  const int* __restrict__ ent_to;
  const int* __restrict__ off_to;
  const int* __restrict__ ent_from;
  const int* __restrict__ off_from;
};

template <class T>
LmaArgs<T> args_of(lfg_lma m) {
  return LmaArgs<T>{m->ncell, m->nl, m->ndf_to, m->ndf_from, m->nent_to, m->nlev_to,
                    m->nent_from, m->nlev_from, (const T*)m->a, m->ent_to, m->off_to,
                    m->ent_from, m->off_from};
}

template <class T>
__device__ __forceinline__ T amat(const LmaArgs<T>& L, int df, int df2, int layer, int cell) {
  return L.a[(((size_t)df * L.ndf_from + df2) * L.nl + layer) * L.ncell + cell];
}

// y(e,k) (+)= sum over incidences (cell, df) of e with layer = k - off(df):
//   sum_df2 A(df, df2, layer, cell) x(ent_from(df2,cell), layer + off_from(df2,cell))
template <class T, bool INC>
__global__ void k_lma_apply(LmaArgs<T> L, const int* __restrict__ ptr,
                            const int* __restrict__ inc, const T* __restrict__ x,
                            T* __restrict__ y) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (e >= L.nent_to) return;
  const size_t o = (size_t)k * L.nent_to + e;
  T acc = INC ? y[o] : (T)0;
  const int j0 = ptr[e], j1 = ptr[e + 1];
  int j = j0;
  while (j < j1) {
    const int cell = inc[j] / L.ndf_to;
    int jend = j + 1;
    while (jend < j1 && inc[jend] / L.ndf_to == cell) ++jend;
    for (int df2 = 0; df2 < L.ndf_from; ++df2) {
      const size_t fi = (size_t)df2 * L.ncell + cell;
      const int ef = L.ent_from[fi], of = L.off_from[fi];
      for (int g = j; g < jend; ++g) {
        const int df = inc[g] - cell * L.ndf_to;
        const int layer = k - L.off_to[(size_t)df * L.ncell + cell];
        if (layer < 0 || layer >= L.nl) continue;
        acc = acc + amat(L, df, df2, layer, cell) *
                        x[(size_t)(layer + of) * L.nent_from + ef];
      }
    }
    j = jend;
  }
  y[o] = acc;
}

// y_from(e,k) += sum over incidences (cell, df2) of the from-entity e, in
// increasing layer: sum_df A(df, df2, layer, cell) x_to(df), each cell-layer
// contribution summed from zero first (transpose_matrix_vector's lhs_e).
template <class T>
__global__ void k_lma_apply_t(LmaArgs<T> L, const int* __restrict__ ptr,
                              const int* __restrict__ inc, const T* __restrict__ x,
                              T* __restrict__ y) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (e >= L.nent_from) return;
  const size_t o = (size_t)k * L.nent_from + e;
  T acc = y[o];
  const int j0 = ptr[e], j1 = ptr[e + 1];
  int j = j0;
  while (j < j1) {
    const int cell = inc[j] / L.ndf_from;
    int jend = j + 1;
    while (jend < j1 && inc[jend] / L.ndf_from == cell) ++jend;
    // increasing layer = decreasing level offset = decreasing local dof
    for (int g = jend - 1; g >= j; --g) {
      const int df2 = inc[g] - cell * L.ndf_from;
      const int layer = k - L.off_from[(size_t)df2 * L.ncell + cell];
      if (layer < 0 || layer >= L.nl) continue;
      T le = (T)0;
      for (int df = 0; df < L.ndf_to; ++df) {
        const size_t ti = (size_t)df * L.ncell + cell;
        le = le + amat(L, df, df2, layer, cell) *
                      x[(size_t)(layer + L.off_to[ti]) * L.nent_to + L.ent_to[ti]];
      }
      acc = acc + le;
    }
    j = jend;
  }
  y[o] = acc;
}

// Two-phase applies.  Phase 1, one thread per (cell, layer) with cells
// fastest, streams the element matrix once (coalesced, evict-first loads so
// that the local products stay in L2) and writes the cell's local products
//   forward    (TR false): loc(df,  layer, cell) = sum_df2 A(df,df2) x(df2)
//   transposed (TR true):  loc(df2, layer, cell) = sum_df  A(df,df2) x(df)
// each summed from zero in ascending order.  Phase 2 is the gather: every
// output dof adds the local products of its incidences in the one-pass
// kernels' order.  The transposed form thus equals k_lma_apply_t bit for
// bit; the forward form adds one local product per incidence where the
// reference (and k_lma_apply) adds the ndf_from products one at a time, a
// rounding-level difference.
// NT/NF > 0 fix ndf_to/ndf_from at compile time (loops fully unrolled);
// 0 takes them at run time, up to kLocDf.
constexpr int kLocDf = 16;  // largest ndf handled by the two-phase form

// OS > 1 (fixed sizes only) splits a cell-layer's outputs over OS threads,
// each gathering the cell's x values and streaming COUT/OS matrix rows:
// fewer loads per thread, more threads with loads in flight.
template <class T, bool TR, int NT, int NF, int OS = 1>
__global__ void k_lma_local(LmaArgs<T> L, const T* __restrict__ x, T* __restrict__ loc) {
  grid_dep_wait();
  constexpr int CIN = TR ? NT : NF, COUT = TR ? NF : NT;
  static_assert(OS == 1 || (COUT > 0 && COUT % OS == 0), "output split needs fixed sizes");
  constexpr int MAXIN = CIN > 0 ? CIN : kLocDf;
  const int nin = CIN > 0 ? CIN : (TR ? L.ndf_to : L.ndf_from);
  const int nout = COUT > 0 ? COUT : (TR ? L.ndf_from : L.ndf_to);
  const int ndf_from = NF > 0 ? NF : L.ndf_from;
  const size_t plane = (size_t)L.ncell * L.nl;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < plane * OS;
       i += (size_t)gridDim.x * blockDim.x) {
    const int h = OS > 1 ? (int)(i / plane) : 0;  // which share of the outputs
    const size_t t = i - (size_t)h * plane;
    const int cell = (int)(t % L.ncell), layer = (int)(t / L.ncell);
    T xv[MAXIN];
#pragma unroll
    for (int d = 0; d < MAXIN; ++d)
      if (d < nin) {
        const size_t ti = (size_t)d * L.ncell + cell;
        xv[d] = TR ? x[(size_t)(layer + L.off_to[ti]) * L.nent_to + L.ent_to[ti]]
                   : x[(size_t)(layer + L.off_from[ti]) * L.nent_from + L.ent_from[ti]];
      }
    if constexpr (COUT == 0) {  // run-time sizes: one output at a time
      for (int o = 0; o < nout; ++o) {
        T acc = (T)0;
#pragma unroll
        for (int d = 0; d < MAXIN; ++d)
          if (d < nin) {
            const int df = TR ? d : o, df2 = TR ? o : d;
            acc = acc + __ldcs(L.a + (size_t)(df * ndf_from + df2) * plane + t) * xv[d];
          }
        loc[(size_t)o * plane + t] = acc;
      }
    } else {
      // fixed sizes: every output summed in registers before any store, so
      // that the stores do not hold back the matrix loads
      constexpr int CO = COUT / OS;
      T acc[CO];
#pragma unroll
      for (int oo = 0; oo < CO; ++oo) acc[oo] = (T)0;
#pragma unroll
      for (int d = 0; d < MAXIN; ++d)
#pragma unroll
        for (int oo = 0; oo < CO; ++oo) {
          const int o = h * CO + oo;
          const int df = TR ? d : o, df2 = TR ? o : d;
          acc[oo] = acc[oo] + __ldcs(L.a + (size_t)(df * ndf_from + df2) * plane + t) * xv[d];
        }
#pragma unroll
      for (int oo = 0; oo < CO; ++oo) loc[(size_t)(h * CO + oo) * plane + t] = acc[oo];
    }
  }
}

// Transposed 8 x 8 local products with the input dofs split over a lane
// pair: lane h = 0 sums df = 0..3 from zero for all eight outputs, hands
// the partial sums to lane h = 1 by shuffle, and that lane adds df = 4..7
// and stores, so each output is summed in ascending df as in the unsplit
// kernel (the same bits).  Each lane gathers 4 inputs and streams 32
// matrix values, the pair's loads of one plane are two 128-byte runs, and
// the loads of both halves are in flight at once (C48x30 W0 operator, 217
// MB of matrices: 47 -> 39 us under ncu; both phases of the apply 53 -> 45
// us between CUDA events).  Every lane runs the same trips (the bound is
// rounded up to the warp).
template <class T>
__global__ void __launch_bounds__(256) k_lma_local_tsplit(LmaArgs<T> L, const T* __restrict__ x,
                                                          T* __restrict__ loc) {
  grid_dep_wait();
  const size_t plane = (size_t)L.ncell * L.nl;
  const size_t total = 2 * plane, trips = (total + 31) & ~(size_t)31;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < trips;
       i += (size_t)gridDim.x * blockDim.x) {
    const bool on = i < total;
    const int h = (int)(i & 1);
    const size_t t = on ? i >> 1 : 0;
    const int cell = (int)(t % L.ncell), layer = (int)(t / L.ncell);
    T xv[4], a[4][8];
#pragma unroll
    for (int dd = 0; dd < 4; ++dd) {
      const size_t ti = (size_t)(4 * h + dd) * L.ncell + cell;
      xv[dd] = x[(size_t)(layer + L.off_to[ti]) * L.nent_to + L.ent_to[ti]];
#pragma unroll
      for (int o = 0; o < 8; ++o) a[dd][o] = __ldcs(L.a + (size_t)((4 * h + dd) * 8 + o) * plane + t);
    }
    T acc[8];
#pragma unroll
    for (int o = 0; o < 8; ++o) acc[o] = (T)0;
    if (h == 0) {
#pragma unroll
      for (int dd = 0; dd < 4; ++dd)
#pragma unroll
        for (int o = 0; o < 8; ++o) acc[o] = acc[o] + a[dd][o] * xv[dd];
    }
#pragma unroll
    for (int o = 0; o < 8; ++o) acc[o] = __shfl_up_sync(0xffffffffu, acc[o], 1);
    if (h == 1 && on) {
#pragma unroll
      for (int dd = 0; dd < 4; ++dd)
#pragma unroll
        for (int o = 0; o < 8; ++o) acc[o] = acc[o] + a[dd][o] * xv[dd];
#pragma unroll
      for (int o = 0; o < 8; ++o) loc[(size_t)o * plane + t] = acc[o];
    }
  }
}

// Padded incidence table: slot m of entity e, [m][e], holds its m-th
// incidence as (cell, o << 8 | df), o the level offset of local dof df in
// the cell; level k of e takes layer k - o of the cell when 0 <= k - o < nl.
// Empty slots carry an offset no level reaches.
__device__ __forceinline__ int slot_df(int2 s) { return s.y & 255; }
__device__ __forceinline__ int slot_off(int2 s) { return s.y >> 8; }

// gather through the padded table: y(e,k) (+)= sum over the slots of e
// whose layer is in range of loc(df, layer, cell); a thread covers KC
// levels of one entity and keeps its W slots in registers
template <class T, bool INC, int W, int KC>
__global__ void k_lma_gather_tab(const int2* __restrict__ tab, int nent, int nlev, int nl,
                                 int ncell, const T* __restrict__ loc, T* __restrict__ y) {
  grid_dep_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nent) return;
  int2 s[W];
#pragma unroll
  for (int m = 0; m < W; ++m) s[m] = tab[(size_t)m * nent + e];
  const int k0 = blockIdx.y * KC, k1 = min(k0 + KC, nlev);
  for (int k = k0; k < k1; ++k) {
    const size_t o = (size_t)k * nent + e;
    T acc = INC ? y[o] : (T)0;
#pragma unroll
    for (int m = 0; m < W; ++m) {
      const int layer = k - slot_off(s[m]);
      if (layer >= 0 && layer < nl)
        acc = acc + loc[((size_t)slot_df(s[m]) * nl + layer) * ncell + s[m].x];
    }
    y[o] = acc;
  }
}

// diag(e,k) += A(df, df, layer, cell) over incidences, increasing layer
template <class T>
__global__ void k_lma_diag(LmaArgs<T> L, const int* __restrict__ ptr,
                           const int* __restrict__ inc, T* __restrict__ d) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (e >= L.nent_to) return;
  const size_t o = (size_t)k * L.nent_to + e;
  T acc = d[o];
  const int j0 = ptr[e], j1 = ptr[e + 1];
  int j = j0;
  while (j < j1) {
    const int cell = inc[j] / L.ndf_to;
    int jend = j + 1;
    while (jend < j1 && inc[jend] / L.ndf_to == cell) ++jend;
    for (int g = jend - 1; g >= j; --g) {
      const int df = inc[g] - cell * L.ndf_to;
      const int layer = k - L.off_to[(size_t)df * L.ncell + cell];
      if (layer < 0 || layer >= L.nl) continue;
      acc = acc + amat(L, df, df, layer, cell);
    }
    j = jend;
  }
  d[o] = acc;
}

// out = m + kappa(cell, layer) * k, entry by entry
template <class T>
__global__ void k_lma_combine(T* __restrict__ out, const T* __restrict__ m,
                              const T* __restrict__ kk, const T* __restrict__ kappa, int ncell,
                              int nl, int nent) {
  const size_t plane = (size_t)nl * ncell;
  const size_t n = plane * nent;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = m[i] + kappa[i % plane] * kk[i];
}

// g(cell, layer) = scale * sum_df u(df) * (sum_df2 A(df,df2) v(df2))
template <class T>
__global__ void k_lma_bilinear(LmaArgs<T> L, const T* __restrict__ u, const T* __restrict__ v,
                               T scale, T* __restrict__ g) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  const int layer = blockIdx.y;
  if (cell >= L.ncell) return;
  T acc = (T)0;
  for (int df = 0; df < L.ndf_to; ++df) {
    const size_t ti = (size_t)df * L.ncell + cell;
    const T ud = u[(size_t)(layer + L.off_to[ti]) * L.nent_to + L.ent_to[ti]];
    T row = (T)0;
    for (int df2 = 0; df2 < L.ndf_from; ++df2) {
      const size_t fi = (size_t)df2 * L.ncell + cell;
      row = row + amat(L, df, df2, layer, cell) *
                      v[(size_t)(layer + L.off_from[fi]) * L.nent_from + L.ent_from[fi]];
    }
    acc = acc + ud * row;
  }
  g[(size_t)layer * L.ncell + cell] = scale * acc;
}

// host: entity / offset tables and incidence lists of one space
void build_space(const int* map, int ndf, int ncell, int nl, int nent, int nlev,
                 std::vector<int>& ent, std::vector<int>& off, std::vector<int>& ptr,
                 std::vector<int>& inc, int& maxinc) {
  ent.assign((size_t)ndf * ncell, 0);
  off.assign((size_t)ndf * ncell, 0);
  std::vector<int> count(nent, 0);
  for (int c = 0; c < ncell; ++c)
    for (int df = 0; df < ndf; ++df) {
      const long dof = map[(size_t)c * ndf + df];
      LFG_REQUIRE(dof >= 0 && dof < (long)nent * nlev, "lma_create: dof out of range");
      const int e = (int)(dof / nlev), o = (int)(dof % nlev);
      LFG_REQUIRE(o + nl <= nlev, "lma_create: a column's dofs run past its entity");
      ent[(size_t)df * ncell + c] = e;
      off[(size_t)df * ncell + c] = o;
      count[e]++;
    }
  ptr.assign(nent + 1, 0);
  for (int e = 0; e < nent; ++e) ptr[e + 1] = ptr[e] + count[e];
  maxinc = *std::max_element(count.begin(), count.end());
  inc.assign(ptr[nent], 0);
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int c = 0; c < ncell; ++c)       // cells ascending, then df ascending
    for (int df = 0; df < ndf; ++df) {
      const int e = ent[(size_t)df * ncell + c];
      inc[fill[e]++] = c * ndf + df;
    }
}

int* dcopy(const std::vector<int>& v) {
  int* p = (int*)dmalloc(v.size() * sizeof(int));
  upload(p, v.data(), v.size() * sizeof(int));
  return p;
}

// padded incidence table of one space (format at slot_df): incidences keep
// the lists' order (cells ascending); REV takes each cell's dfs in
// descending order (the transposed apply's).  Returns the width (a power
// of two), or 0 when the lists are wider than 16, ndf > 255 or the level
// offsets reach 2^22.
int build_tab(const std::vector<int>& off, const std::vector<int>& ptr,
              const std::vector<int>& inc, int ndf, int ncell, int nlev, int maxinc, bool rev,
              int2** out) {
  int w = 1;
  while (w < maxinc) w <<= 1;
  if (w > 16 || ndf > 255 || nlev >= (1 << 22)) return 0;
  const int nent = (int)ptr.size() - 1;
  std::vector<int2> tab((size_t)w * nent, make_int2(0, 1 << 30));
  for (int e = 0; e < nent; ++e) {
    int m = 0;
    for (int j = ptr[e]; j < ptr[e + 1];) {
      const int cell = inc[j] / ndf;
      int jend = j + 1;
      while (jend < ptr[e + 1] && inc[jend] / ndf == cell) ++jend;
      for (int q = 0; q < jend - j; ++q) {
        const int df = inc[rev ? jend - 1 - q : j + q] - cell * ndf;
        const int o = off[(size_t)df * ncell + cell];
        tab[(size_t)m++ * nent + e] = make_int2(cell, o << 8 | df);
      }
      j = jend;
    }
  }
  *out = (int2*)dmalloc(tab.size() * sizeof(int2));
  upload(*out, tab.data(), tab.size() * sizeof(int2));
  return w;
}

template <class T, bool TR>
void launch_local(lfg_ctx c, lfg_lma m, const T* x, T* loc) {
  const size_t ncl = (size_t)m->ncell * m->nl;
  auto go = [&](void (*k)(LmaArgs<T>, const T*, T*), int os) {
    launch_pdl(c, k, occ_grid(c, (const void*)k, 256, ncl * os), 256, 0, args_of<T>(m), x, loc);
  };
  // 8x8: forward outputs split over 2 threads (48.0 against 53.7 us on the
  // C48x30 W0 operator); the transposed products split their inputs over a
  // lane pair (splitting their outputs measured slower: 69 us)
  if (m->ndf_to == 8 && m->ndf_from == 8) {
    if (TR) go(k_lma_local_tsplit<T>, 2);
    else go(k_lma_local<T, TR, 8, 8, 2>, 2);
  }
  else if (m->ndf_to == 1 && m->ndf_from == 1) go(k_lma_local<T, TR, 1, 1>, 1);
  else go(k_lma_local<T, TR, 0, 0>, 1);
  // the element matrices and the input field; the local products are an
  // intermediate (kept in L2) and not counted
  const uint64_t nin = TR ? (uint64_t)m->nent_to * m->nlev_to
                          : (uint64_t)m->nent_from * m->nlev_from;
  after_launch(c, "lma_local", sizeof(T) * ((uint64_t)ncl * m->ndf_to * m->ndf_from + nin));
}

template <class T, bool INC>
void launch_gather_tab(lfg_ctx c, const int2* tab, int w, int nent, int nlev, int nl, int ncell,
                       const T* loc, T* y) {
  constexpr int KC = 4;
  const dim3 grid((nent + 127) / 128, (nlev + KC - 1) / KC);
  auto go = [&](void (*k)(const int2*, int, int, int, int, const T*, T*)) {
    launch_pdl(c, k, grid, dim3(128), 0, tab, nent, nlev, nl, ncell, loc, y);
  };
  switch (w) {
    case 1: go(k_lma_gather_tab<T, INC, 1, KC>); break;
    case 2: go(k_lma_gather_tab<T, INC, 2, KC>); break;
    case 4: go(k_lma_gather_tab<T, INC, 4, KC>); break;
    case 8: go(k_lma_gather_tab<T, INC, 8, KC>); break;
    default: go(k_lma_gather_tab<T, INC, 16, KC>); break;
  }
  // the output field written (and read with INC)
  after_launch(c, "lma_gather", sizeof(T) * (uint64_t)nent * nlev * (INC ? 2 : 1));
}

void upload_matrix(lfg_lma m, const double* ls) {
  const size_t n3 = (size_t)m->ncell * m->nl;
  const size_t n = n3 * m->ndf_to * m->ndf_from;
  std::vector<double> dev(n);
  for (int dt = 0; dt < m->ndf_to; ++dt)
    for (int dfm = 0; dfm < m->ndf_from; ++dfm)
      for (int c = 0; c < m->ncell; ++c)
        for (int l = 0; l < m->nl; ++l) {
          const size_t ik = (size_t)c * m->nl + l;
          dev[(((size_t)dt * m->ndf_from + dfm) * m->nl + l) * m->ncell + c] =
              ls[ik + n3 * (dt + (size_t)m->ndf_to * dfm)];
        }
  if (m->kind == LFG_R_DOUBLE) {
    upload(m->a, dev.data(), n * sizeof(double));
  } else {
    std::vector<float> f(dev.begin(), dev.end());
    upload(m->a, f.data(), n * sizeof(float));
  }
}

template <class F>
void dispatch(int kind, F&& f) {
  if (kind == LFG_R_DOUBLE) f(double{});
  else f(float{});
}

}  // namespace

extern "C" {

int lfg_lma_create(lfg_ctx c, int kind, int ncell, int nl, int ndf_to, int ndf_from,
                   const double* ls, const int* map_to, int nent_to, int nlev_to,
                   const int* map_from, int nent_from, int nlev_from, lfg_lma* out) {
  if (!c || !out) return LFG_ERR_ARG;
  return guard(c, [&] {
    LFG_REQUIRE(kind == LFG_R_DOUBLE || kind == LFG_R_SINGLE, "lma_create: bad kind");
    LFG_REQUIRE(ncell > 0 && nl > 0 && ndf_to > 0 && ndf_from > 0 && ls && map_to &&
                    map_from && nent_to > 0 && nent_from > 0 && nlev_to >= nl &&
                    nlev_from >= nl,
                "lma_create: bad arguments");
    lfg_lma m = new lfg_lma_s;
    m->ctx = c;
    m->kind = kind;
    m->ncell = ncell;
    m->nl = nl;
    m->ndf_to = ndf_to;
    m->ndf_from = ndf_from;
    m->nent_to = nent_to;
    m->nlev_to = nlev_to;
    m->nent_from = nent_from;
    m->nlev_from = nlev_from;
    try {
      std::vector<int> ent, off, ptr, inc;
      build_space(map_to, ndf_to, ncell, nl, nent_to, nlev_to, ent, off, ptr, inc, m->max_inc_to);
      m->ent_to = dcopy(ent);
      m->off_to = dcopy(off);
      m->inc_to_ptr = dcopy(ptr);
      m->inc_to = dcopy(inc);
      if (ndf_to <= kLocDf && ndf_from <= kLocDf)
        m->tab_to_w = build_tab(off, ptr, inc, ndf_to, ncell, nlev_to, m->max_inc_to, false,
                                &m->tab_to);
      build_space(map_from, ndf_from, ncell, nl, nent_from, nlev_from, ent, off, ptr, inc,
                  m->max_inc_from);
      m->ent_from = dcopy(ent);
      m->off_from = dcopy(off);
      m->inc_from_ptr = dcopy(ptr);
      m->inc_from = dcopy(inc);
      if (ndf_to <= kLocDf && ndf_from <= kLocDf)
        m->tab_from_w = build_tab(off, ptr, inc, ndf_from, ncell, nlev_from, m->max_inc_from,
                                  true, &m->tab_from);
      m->a = dmalloc((size_t)ncell * nl * ndf_to * ndf_from * kind);
      upload_matrix(m, ls);
    } catch (...) {
      lfg_lma_destroy(m);
      throw;
    }
    *out = m;
  });
}

int lfg_lma_destroy(lfg_lma m) {
  if (!m) return LFG_OK;
  for (void* p : {(void*)m->a, (void*)m->ent_to, (void*)m->off_to, (void*)m->ent_from,
                  (void*)m->off_from, (void*)m->inc_to_ptr, (void*)m->inc_to,
                  (void*)m->inc_from_ptr, (void*)m->inc_from, (void*)m->tab_to,
                  (void*)m->tab_from})
    dfree(p);
  delete m;
  return LFG_OK;
}

int lfg_lma_set_values(lfg_lma m, const double* ls) {
  if (!m || !ls) return LFG_ERR_ARG;
  return guard(m->ctx, [&] { upload_matrix(m, ls); });
}

int lfg_lma_apply(lfg_lma m, int mode, lfg_field lhs, lfg_field x) {
  if (!m) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(lhs && x && lhs->kind == m->kind && x->kind == m->kind,
                "lma_apply: field kinds must match the operator");
    if (mode == LFG_LMA_TRANSPOSE) {
      LFG_REQUIRE(lhs->ncol == m->nent_from && lhs->nlev == m->nlev_from &&
                      x->ncol == m->nent_to && x->nlev == m->nlev_to,
                  "lma_apply: transposed apply maps the to-space onto the from-space");
    } else {
      LFG_REQUIRE(mode == LFG_LMA_INC || mode == LFG_LMA_WRITE, "lma_apply: bad mode");
      LFG_REQUIRE(lhs->ncol == m->nent_to && lhs->nlev == m->nlev_to &&
                      x->ncol == m->nent_from && x->nlev == m->nlev_from,
                  "lma_apply: fields do not match the operator's spaces");
    }
    const bool tr = mode == LFG_LMA_TRANSPOSE;
    // two-phase form: local products, then the padded-table gather
    if (tr ? m->tab_from_w > 0 : m->tab_to_w > 0) {
      const size_t ncl = (size_t)m->ncell * m->nl;
      dispatch(m->kind, [&](auto tag) {
        using T = decltype(tag);
        T* loc = (T*)c->scratch(ncl * (tr ? m->ndf_from : m->ndf_to) * sizeof(T));
        if (tr) {
          launch_local<T, true>(c, m, (const T*)x->d, loc);
          launch_gather_tab<T, true>(c, m->tab_from, m->tab_from_w, m->nent_from, m->nlev_from,
                                     m->nl, m->ncell, loc, (T*)lhs->d);
        } else {
          launch_local<T, false>(c, m, (const T*)x->d, loc);
          if (mode == LFG_LMA_INC)
            launch_gather_tab<T, true>(c, m->tab_to, m->tab_to_w, m->nent_to, m->nlev_to, m->nl,
                                       m->ncell, loc, (T*)lhs->d);
          else
            launch_gather_tab<T, false>(c, m->tab_to, m->tab_to_w, m->nent_to, m->nlev_to, m->nl,
                                        m->ncell, loc, (T*)lhs->d);
        }
      });
      return;
    }
    dispatch(m->kind, [&](auto tag) {
      using T = decltype(tag);
      if (mode == LFG_LMA_TRANSPOSE) {
        dim3 grid((m->nent_from + 127) / 128, m->nlev_from);
        k_lma_apply_t<T><<<grid, 128, 0, c->stream>>>(args_of<T>(m), m->inc_from_ptr, m->inc_from,
                                                      (const T*)x->d, (T*)lhs->d);
      } else {
        dim3 grid((m->nent_to + 127) / 128, m->nlev_to);
        if (mode == LFG_LMA_INC)
          k_lma_apply<T, true><<<grid, 128, 0, c->stream>>>(args_of<T>(m), m->inc_to_ptr, m->inc_to, (const T*)x->d, (T*)lhs->d);
        else
          k_lma_apply<T, false><<<grid, 128, 0, c->stream>>>(args_of<T>(m), m->inc_to_ptr, m->inc_to, (const T*)x->d, (T*)lhs->d);
      }
    });
    // element matrices, x read; lhs read (INC, TRANSPOSE) and written
    const uint64_t nx = mode == LFG_LMA_TRANSPOSE ? (uint64_t)m->nent_to * m->nlev_to
                                                  : (uint64_t)m->nent_from * m->nlev_from;
    const uint64_t ny = mode == LFG_LMA_TRANSPOSE ? (uint64_t)m->nent_from * m->nlev_from
                                                  : (uint64_t)m->nent_to * m->nlev_to;
    after_launch(c, "lma_apply",
                 (uint64_t)m->kind * ((uint64_t)m->ncell * m->nl * m->ndf_to * m->ndf_from + nx +
                                      ny * (mode == LFG_LMA_WRITE ? 1 : 2)));
  });
}

int lfg_lma_diagonal(lfg_lma m, lfg_field diag) {
  if (!m) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(m->ndf_to == m->ndf_from, "lma_diagonal: operator must be square");
    LFG_REQUIRE(diag && diag->kind == m->kind && diag->ncol == m->nent_to &&
                    diag->nlev == m->nlev_to,
                "lma_diagonal: field does not match the operator");
    dispatch(m->kind, [&](auto tag) {
      using T = decltype(tag);
      dim3 grid((m->nent_to + 127) / 128, m->nlev_to);
      k_lma_diag<T><<<grid, 128, 0, c->stream>>>(args_of<T>(m), m->inc_to_ptr, m->inc_to, (T*)diag->d);
    });
    after_launch(c, "lma_diagonal");
  });
}

int lfg_lma_combine(lfg_lma out, lfg_lma mm, lfg_lma kk, lfg_field kappa) {
  if (!out || !mm || !kk) return LFG_ERR_ARG;
  lfg_ctx c = out->ctx;
  return guard(c, [&] {
    for (lfg_lma o : {mm, kk})
      LFG_REQUIRE(o->kind == out->kind && o->ncell == out->ncell && o->nl == out->nl &&
                      o->ndf_to == out->ndf_to && o->ndf_from == out->ndf_from,
                  "lma_combine: operators differ in shape or kind");
    LFG_REQUIRE(kappa && kappa->kind == out->kind && kappa->ncol == out->ncell &&
                    kappa->nlev == out->nl,
                "lma_combine: kappa must be a cell field with nlayers levels");
    const size_t n = (size_t)out->ncell * out->nl * out->ndf_to * out->ndf_from;
    dispatch(out->kind, [&](auto tag) {
      using T = decltype(tag);
      k_lma_combine<T><<<c->stream_grid(n), kThreads, 0, c->stream>>>(
          (T*)out->a, (const T*)mm->a, (const T*)kk->a, (const T*)kappa->d, out->ncell,
          out->nl, out->ndf_to * out->ndf_from);
    });
    after_launch(c, "lma_combine");
  });
}

int lfg_lma_bilinear(lfg_lma m, lfg_field u, lfg_field v, double scale, lfg_field g) {
  if (!m) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(u && v && g && u->kind == m->kind && v->kind == m->kind && g->kind == m->kind,
                "lma_bilinear: kinds must match");
    LFG_REQUIRE(u->ncol == m->nent_to && u->nlev == m->nlev_to && v->ncol == m->nent_from &&
                    v->nlev == m->nlev_from && g->ncol == m->ncell && g->nlev == m->nl,
                "lma_bilinear: fields do not match the operator");
    dispatch(m->kind, [&](auto tag) {
      using T = decltype(tag);
      dim3 grid((m->ncell + 127) / 128, m->nl);
      k_lma_bilinear<T><<<grid, 128, 0, c->stream>>>(args_of<T>(m), (const T*)u->d,
                                                     (const T*)v->d, (T)scale, (T*)g->d);
    });
    after_launch(c, "lma_bilinear");
  });
}

}  // extern "C"

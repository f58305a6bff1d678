// W2 intergrid transfers (components/science/source/kernel/inter_mesh/):
//   restrict_w2   sci_restrict_w2_kernel_mod.F90   W,S,E,N by face selectors, and B
//   restrict_w2h  sci_restrict_w2h_kernel_mod.F90  W,S,E,N by face selectors
//   restrict_w2v  sci_restrict_w2v_kernel_mod.F90  the vertical (B) column
//   weights_prolong_w2, prolong_w2 (sci_weights_prolong_w2_kernel_mod.F90,
//   sci_prolong_w2_kernel_mod.F90)
//
// W2 fields are flat arrays in the reference's dof order (the dof of level
// k of cell dof df at map(df, cell) + k); the face columns hold nlayers
// values, the vertical column nlayers + 1.  One thread per (coarse cell,
// level), levels fastest, so a warp reads consecutive dofs of a column.
// Restriction writes only the faces its coarse cell owns (the face
// selectors split the shared faces), so every coarse dof has one writer
// and the sums keep the reference's order (y outer, x inner).  The
// prolongation writes the fine faces on the coarse cell's boundary from
// both neighbouring coarse cells; both write the same value (the shared
// coarse face and the same fine weight), so the result is deterministic.
#include <cuda_runtime.h>

#include <vector>

#include "lfg_internal.cuh"

namespace {

using namespace lfg;

enum { DW = 0, DS = 1, DE = 2, DN = 3, DB = 4 };  // 0-based W2 dof numbers

struct W2Args {
  int ncoarse, nl, nx, ny, ndf;
  const int* child;  // [nx*ny][ncoarse], slot y*nx + x (0-based x, y)
  const int* mapc;   // [ncoarse][ndf]
  const int* mapf;   // [nfine][ndf]
  const int* sel_ew; // [ncoarse]
  const int* sel_ns;
  // 0: flat fields in the reference's dof order (the dof of level k is
  // map + k); else level-major columns (nent columns of nlayers+1 levels,
  // the maps hold column ids, the dof of level k is k*nent + map)
  int nent_c, nent_f;
};

__device__ __forceinline__ size_t dof_at(int map, int k, int nent) {
  return nent ? (size_t)k * nent + map : (size_t)map + k;
}

__device__ __forceinline__ int fcell(const W2Args& a, int C, int x, int y) {
  return a.child[(size_t)(y * a.nx + x) * a.ncoarse + C];
}

// fine-cell ranges (0-based, inclusive) of each horizontal face of a coarse cell
__device__ __forceinline__ void face_range(int df, int nx, int ny, int& x0, int& x1, int& y0,
                                           int& y1) {
  x0 = 0; x1 = nx - 1; y0 = 0; y1 = ny - 1;
  if (df == DN) y1 = 0;
  else if (df == DS) y0 = ny - 1;
  else if (df == DW) x1 = 0;
  else if (df == DE) x0 = nx - 1;
}

template <class T>
__global__ void k_w2_restrict(W2Args a, int mode, T* __restrict__ coarse,
                              const T* __restrict__ fine) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int nk = a.nl + 1;
  if (t >= (size_t)a.ncoarse * nk) return;
  const int C = (int)(t / nk), k = (int)(t % nk);
  if (mode == LFG_W2_V) {   // restrict_w2v: dof 1 of the W2V map
    T acc = (T)0;
    for (int y = 0; y < a.ny; ++y)
      for (int x = 0; x < a.nx; ++x)
        acc = acc + fine[dof_at(a.mapf[(size_t)fcell(a, C, x, y) * a.ndf], k, a.nent_f)];
    coarse[dof_at(a.mapc[(size_t)C * a.ndf], k, a.nent_c)] = acc;
    return;
  }
  if (k < a.nl) {
    const int ew = a.sel_ew[C], ns = a.sel_ns[C];
    for (int face = 1; face <= ew + ns; ++face) {
      int df = face - 1;
      if (face == 3 && ns == 2 && ew == 1) df = DN;
      int x0, x1, y0, y1;
      face_range(df, a.nx, a.ny, x0, x1, y0, y1);
      T acc = (T)0;
      for (int y = y0; y <= y1; ++y)
        for (int x = x0; x <= x1; ++x)
          acc = acc + fine[dof_at(a.mapf[(size_t)fcell(a, C, x, y) * a.ndf + df], k, a.nent_f)];
      coarse[dof_at(a.mapc[(size_t)C * a.ndf + df], k, a.nent_c)] = acc;
    }
  }
  if (mode == LFG_W2_FULL) {
    T acc = (T)0;
    for (int y = 0; y < a.ny; ++y)
      for (int x = 0; x < a.nx; ++x)
        acc = acc + fine[dof_at(a.mapf[(size_t)fcell(a, C, x, y) * a.ndf + DB], k, a.nent_f)];
    coarse[dof_at(a.mapc[(size_t)C * a.ndf + DB], k, a.nent_c)] = acc;
  }
}

__global__ void k_w2_weights(W2Args a, double* __restrict__ w) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int nk = a.nl + 1;
  if (t >= (size_t)a.ncoarse * nk) return;
  const int C = (int)(t / nk), k = (int)(t % nk);
  const int nx = a.nx, ny = a.ny;
  auto W = [&](int df, int x, int y) -> double& {
    return w[dof_at(a.mapf[(size_t)fcell(a, C, x, y) * a.ndf + df], k, a.nent_f)];
  };
  if (k < a.nl) {
    for (int x = 0; x < nx; ++x) {
      W(DN, x, 0) = 1.0 / (double)nx;
      W(DS, x, ny - 1) = 1.0 / (double)nx;
    }
    for (int y = 0; y < ny; ++y) {
      W(DW, 0, y) = 1.0 / (double)ny;
      W(DE, nx - 1, y) = 1.0 / (double)ny;
    }
    for (int y = 0; y < ny; ++y)
      for (int x = 1; x < nx; ++x) W(DW, x, y) = (double)(nx - x) / (double)nx;
    for (int x = 0; x < nx; ++x)
      for (int y = 1; y < ny; ++y) W(DN, x, y) = (double)(ny - y) / (double)ny;
  }
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) W(DB, x, y) = 1.0 / (double)(nx * ny);
}

__global__ void k_w2_prolong(W2Args a, double* __restrict__ fine,
                             const double* __restrict__ coarse,
                             const double* __restrict__ w) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int nk = a.nl + 1;
  if (t >= (size_t)a.ncoarse * nk) return;
  const int C = (int)(t / nk), k = (int)(t % nk);
  const int nx = a.nx, ny = a.ny;
  auto F = [&](int df, int x, int y) {
    return dof_at(a.mapf[(size_t)fcell(a, C, x, y) * a.ndf + df], k, a.nent_f);
  };
  auto CO = [&](int df) { return coarse[dof_at(a.mapc[(size_t)C * a.ndf + df], k, a.nent_c)]; };
  if (k < a.nl) {
    for (int x = 0; x < nx; ++x) {
      fine[F(DN, x, 0)] = w[F(DN, x, 0)] * CO(DN);
      fine[F(DS, x, ny - 1)] = w[F(DS, x, ny - 1)] * CO(DS);
    }
    for (int y = 0; y < ny; ++y) {
      fine[F(DW, 0, y)] = w[F(DW, 0, y)] * CO(DW);
      fine[F(DE, nx - 1, y)] = w[F(DE, nx - 1, y)] * CO(DE);
    }
    for (int y = 0; y < ny; ++y) {
      const double ew = w[F(DW, 0, y)];
      for (int x = 1; x < nx; ++x) {
        const double iw = w[F(DW, x, y)];
        fine[F(DW, x, y)] = ew * (iw * CO(DW) + (1.0 - iw) * CO(DE));
      }
    }
    for (int x = 0; x < nx; ++x) {
      const double ew = w[F(DN, x, 0)];
      for (int y = 1; y < ny; ++y) {
        const double iw = w[F(DN, x, y)];
        fine[F(DN, x, y)] = ew * (iw * CO(DN) + (1.0 - iw) * CO(DS));
      }
    }
  }
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) fine[F(DB, x, y)] = w[F(DB, x, y)] * CO(DB);
}

}  // namespace

namespace {

W2Args args_of(lfg_w2map m) {
  return W2Args{m->ig->ncoarse, m->nl, m->ig->nx, m->ig->ny, m->ndf, m->ig->child,
                m->mapc,        m->mapf, m->sel_ew, m->sel_ns, m->nent_c, m->nent_f};
}

void w2_release(lfg_w2map m) {
  dfree(m->mapc);
  dfree(m->mapf);
  dfree(m->sel_ew);
  dfree(m->sel_ns);
}

// Every dof a transfer touches must lie inside the field: face columns
// (dofs W, S, E, N) hold nlayers values, the vertical column (B, or dof 1
// of a W2V map) nlayers + 1.
void check_map(const int* map, int ncell, int ndf, int nl, int undf, const char* what) {
  for (int c = 0; c < ncell; ++c)
    for (int d = 0; d < ndf; ++d) {
      const int v = map[(size_t)c * ndf + d];
      const bool vertical = ndf == 2 ? d == 0 : d == DB;  // T is read through B's column
      const int top = vertical ? nl : nl - 1;
      LFG_REQUIRE(v >= 0 && (long)v + top < undf, std::string(what) + ": dofmap entry out of range");
    }
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// lfg_w2map_create (nent_c = nent_f = 0) and lfg_w2map_create_columns
int w2map_create(lfg_intergrid ig, int nlayers, int ndf, const int* map_coarse,
                 int undf_coarse, const int* map_fine, int undf_fine,
                 const int* face_selector_ew, const int* face_selector_ns, int nent_c,
                 int nent_f, lfg_w2map* out) {
  if (!ig || !out || !map_coarse || !map_fine) return LFG_ERR_ARG;
  lfg_ctx c = ig->ctx;
  lfg_w2map m = new lfg_w2map_s;
  const int rc = guard(c, [&] {
    LFG_REQUIRE(nlayers >= 1 && (ndf == 2 || ndf == 4 || ndf == 6),
                "w2map_create: ndf must be 6 (W2), 4 (W2H) or 2 (W2V)");
    LFG_REQUIRE(!face_selector_ew == !face_selector_ns,
                "w2map_create: give both face selectors or neither");
    m->ctx = c;
    m->ig = ig;
    m->nl = nlayers;
    m->ndf = ndf;
    m->undf_c = undf_coarse;
    m->undf_f = undf_fine;
    m->nent_c = nent_c;
    m->nent_f = nent_f;
    if (nent_c) {  // column ids of level-major fields with nlayers+1 levels
      for (size_t i = 0; i < (size_t)ig->ncoarse * ndf; ++i)
        LFG_REQUIRE(map_coarse[i] >= 0 && map_coarse[i] < nent_c,
                    "w2map_create_columns: coarse column id out of range");
      for (size_t i = 0; i < (size_t)ig->nfine * ndf; ++i)
        LFG_REQUIRE(map_fine[i] >= 0 && map_fine[i] < nent_f,
                    "w2map_create_columns: fine column id out of range");
    } else {
      check_map(map_coarse, ig->ncoarse, ndf, nlayers, undf_coarse, "w2map_create (coarse)");
      check_map(map_fine, ig->nfine, ndf, nlayers, undf_fine, "w2map_create (fine)");
    }
    m->mapc = (int*)dmalloc(sizeof(int) * (size_t)ig->ncoarse * ndf);
    m->mapf = (int*)dmalloc(sizeof(int) * (size_t)ig->nfine * ndf);
    upload(m->mapc, map_coarse, sizeof(int) * (size_t)ig->ncoarse * ndf);
    upload(m->mapf, map_fine, sizeof(int) * (size_t)ig->nfine * ndf);
    if (face_selector_ew) {
      for (int i = 0; i < ig->ncoarse; ++i)
        LFG_REQUIRE((face_selector_ew[i] == 1 || face_selector_ew[i] == 2) &&
                        (face_selector_ns[i] == 1 || face_selector_ns[i] == 2),
                    "w2map_create: face selectors must be 1 or 2");
      m->sel_ew = (int*)dmalloc(sizeof(int) * ig->ncoarse);
      m->sel_ns = (int*)dmalloc(sizeof(int) * ig->ncoarse);
      upload(m->sel_ew, face_selector_ew, sizeof(int) * ig->ncoarse);
      upload(m->sel_ns, face_selector_ns, sizeof(int) * ig->ncoarse);
      m->has_sel = true;
    }
  });
  if (rc != LFG_OK) {
    w2_release(m);
    delete m;
    return rc;
  }
  *out = m;
  return LFG_OK;
}

}  // namespace

extern "C" {

int lfg_w2map_create(lfg_intergrid ig, int nlayers, int ndf, const int* map_coarse,
                     int undf_coarse, const int* map_fine, int undf_fine,
                     const int* face_selector_ew, const int* face_selector_ns, lfg_w2map* out) {
  return w2map_create(ig, nlayers, ndf, map_coarse, undf_coarse, map_fine, undf_fine,
                      face_selector_ew, face_selector_ns, 0, 0, out);
}

int lfg_w2map_create_columns(lfg_intergrid ig, int nlayers, int ndf, const int* col_coarse,
                             int ncol_coarse, const int* col_fine, int ncol_fine,
                             const int* face_selector_ew, const int* face_selector_ns,
                             lfg_w2map* out) {
  if (ncol_coarse <= 0 || ncol_fine <= 0) return LFG_ERR_ARG;
  return w2map_create(ig, nlayers, ndf, col_coarse, ncol_coarse * (nlayers + 1), col_fine,
                      ncol_fine * (nlayers + 1), face_selector_ew, face_selector_ns,
                      ncol_coarse, ncol_fine, out);
}

int lfg_w2map_destroy(lfg_w2map m) {
  if (!m) return LFG_OK;
  w2_release(m);
  delete m;
  return LFG_OK;
}

int lfg_w2_restrict(lfg_w2map m, int mode, lfg_field coarse, lfg_field fine) {
  if (!m || !coarse || !fine) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(mode == LFG_W2_FULL || mode == LFG_W2_H || mode == LFG_W2_V,
                "w2_restrict: bad mode");
    LFG_REQUIRE(mode != LFG_W2_FULL || m->ndf == 6, "w2_restrict: W2 needs ndf 6");
    LFG_REQUIRE(mode != LFG_W2_H || m->ndf >= 4, "w2_restrict: W2H needs ndf 4 or 6");
    LFG_REQUIRE(mode != LFG_W2_V || m->ndf == 2, "w2_restrict: W2V needs ndf 2");
    LFG_REQUIRE(mode == LFG_W2_V || m->has_sel, "w2_restrict: face selectors required");
    LFG_REQUIRE(coarse->n() == (size_t)m->undf_c && fine->n() == (size_t)m->undf_f &&
                    coarse->kind == fine->kind,
                "w2_restrict: fields do not match the maps");
    const size_t n = (size_t)m->ig->ncoarse * (m->nl + 1);
    const int bs = 128;
    const unsigned grid = (unsigned)((n + bs - 1) / bs);
    if (coarse->kind == LFG_R_DOUBLE)
      k_w2_restrict<double><<<grid, bs, 0, c->stream>>>(args_of(m), mode, (double*)coarse->d,
                                                        (const double*)fine->d);
    else
      k_w2_restrict<float><<<grid, bs, 0, c->stream>>>(args_of(m), mode, (float*)coarse->d,
                                                       (const float*)fine->d);
    // fine field read, coarse field written (whole fields, an upper bound
    // for the partial restrictions)
    after_launch(c, "w2_restrict", (uint64_t)coarse->kind * (fine->n() + coarse->n()));
  });
}

int lfg_w2_prolong_weights(lfg_w2map m, lfg_field weights) {
  if (!m || !weights) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(m->ndf == 6 && weights->n() == (size_t)m->undf_f &&
                    weights->kind == LFG_R_DOUBLE,
                "w2_prolong_weights: needs a W2 (ndf 6) map and an r_double fine field");
    const size_t n = (size_t)m->ig->ncoarse * (m->nl + 1);
    k_w2_weights<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(args_of(m),
                                                                      (double*)weights->d);
    after_launch(c, "w2_weights", (uint64_t)8 * 2 * weights->n());
  });
}

int lfg_w2_prolong(lfg_w2map m, lfg_field fine, lfg_field coarse, lfg_field weights) {
  if (!m || !fine || !coarse || !weights) return LFG_ERR_ARG;
  lfg_ctx c = m->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(m->ndf == 6 && fine->n() == (size_t)m->undf_f &&
                    weights->n() == (size_t)m->undf_f && coarse->n() == (size_t)m->undf_c &&
                    fine->kind == LFG_R_DOUBLE && coarse->kind == LFG_R_DOUBLE &&
                    weights->kind == LFG_R_DOUBLE,
                "w2_prolong: needs a W2 (ndf 6) map and r_double fields of its sizes");
    const size_t n = (size_t)m->ig->ncoarse * (m->nl + 1);
    k_w2_prolong<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(
        args_of(m), (double*)fine->d, (const double*)coarse->d, (const double*)weights->d);
    // fine read and written, weights read, coarse read
    after_launch(c, "w2_prolong", (uint64_t)8 * (3 * fine->n() + coarse->n()));
  });
}

}  // extern "C"

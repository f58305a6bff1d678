// Batched independent W3 Helmholtz solves in ONE persistent launch.
//
// Every problem is solved by mixed-precision iterative refinement: the FP64
// residual r = b - A x, an FP32 preconditioned conjugate gradient on
// A e = r (cg_solve, components/science/source/solver/
// sci_iterative_solver_mod.f90:495-592, with monitor_convergence and
// a_tol = 0) whose preconditioner is the exact column solve T'^{-1}
// (columnwise_op_appinv, sci_columnwise_op_appinv_kernel_mod.F90:77-145,
// on the Thomas factors of the operator), and x += e in FP64.
//
// Execution.  A cooperative grid of G CTAs (all resident) walks a list of
// column tiles: tile = (problem, TC consecutive columns), thread = column,
// a loop over the column's levels.  In every phase the CTAs take tiles from
// a shared counter, heaviest first (tiles sorted by level count), so the
// work of a phase is balanced whatever subset of problems is still active.
// Data written in one phase and read in a later one is read through L2
// (ld.global.cg), since the tile may run on another SM.
//
// The grid advances in phases separated by a grid barrier.  In each phase
// each unfinished problem does one step of its own state machine:
//   RESID    r64 = b - A x (FP64), r = float(r64), e = 0, z = T'^{-1} r
//   APPLY    p = beta p + z (p = z on the first inner step), q = A p, <p, q>
//   UPDATE   e += alpha p, r -= alpha q, |r|^2, z = T'^{-1} r, <r, z>
//   CORRECT  x += double(e)
// so an inner CG iteration takes two phases.  The direction p is double
// buffered: APPLY reads the previous p from one buffer and writes the new
// one to the other, forming the new p of the four horizontal neighbours on
// the fly from their previous p and z (the same arithmetic as their owner).
// Scalars are reduced without atomics on floating point: each tile writes
// its partial sums to its own slot; the CTA that finishes a problem's last
// tile of the phase (an integer counter per problem) adds the slots in tile
// order and computes the problem's next state, so every reduction is
// deterministic and no CTA waits for it.  The grid stops when every
// problem is done (an integer count) or after a phase limit.
//
// Every wait is bounded: the barrier spins at most spin_limit times, then
// records an error and returns, and the whole grid leaves at the next
// barrier check; the host reports LFG_ERR_STATE.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <map>
#include <set>

#include "lfg_internal.cuh"

namespace lfg {
namespace {

enum BMode : int { BM_RESID = 0, BM_APPLY, BM_UPDATE, BM_CORRECT, BM_DONE };
enum BErr : unsigned { BE_NONE = 0, BE_BARRIER = 1, BE_PHASES = 2 };
// ctrl words
// C_SNAP, C_SNAP + 1: done counts per barrier parity; C_WORK..C_WORK + 3:
// tile counters of phases 0..3 mod 4
enum : int { C_ARRIVE = 0, C_GEN = 1, C_DONE = 2, C_ERR = 3, C_PHASES = 4, C_SNAP = 5,
             C_WORK = 8, C_NCTRL = 16 };

struct BProb {
  int ncol, nl, tile0, ntiles;
  const double *sub64, *diag64, *sup64, *h64;  // FP64 operator [nl][ncol], h [4][nl][ncol]
  const float *sub, *diag, *sup, *h, *inv, *cp;  // FP32 operator and Thomas factors
  const int* links;                              // [4][ncol]
  const double* b;
  double* x;
  float *e, *r, *z, *q;
  float* p[2];  // direction, double buffered
};

struct BState {
  int mode, status, outer, it, inner_total;
  int pb;  // bits 0: buffer of the current p; 1: next APPLY starts a CG (p = z)
  double rz, alpha, beta, rnrm0, bnorm, res, inner_err;
};

struct BArgs {
  const BProb* probs;
  BState* st;
  const int2* tiles;  // (problem, first column), heaviest first
  int ntiles, nprob;
  int nslots;         // partial-sum slots: one per tile, problem p's from tile0
  double* part;       // [3][nslots]
  unsigned* cnt;      // [nprob]
  unsigned* ctrl;     // C_NCTRL words
  double tol, inner_tol;
  int max_outer, max_inner, max_phases;
  unsigned barrier_extra;  // test hook: arrivals the barrier waits for beyond the grid
  long long spin_limit;
};

template <class T>
__device__ __forceinline__ T ldcg(const T* p) { return __ldcg(p); }

// Grid barrier for a cooperative (co-resident) grid.  Returns the number of
// finished problems as it stood when the last CTA arrived (a snapshot kept
// per barrier parity, so a CTA that leaves late does not see the count move
// on under work that faster CTAs have started), or -1 when the wait ran out
// of spins or another CTA recorded an error.
__device__ int grid_barrier(const BArgs& a) {
  __shared__ int res;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = a.ctrl + C_GEN;
    const unsigned g = *gen;
    int ok = 1;
    __threadfence();
    const unsigned arrived = atomicAdd(a.ctrl + C_ARRIVE, 1u) + 1;
    if (arrived == gridDim.x + a.barrier_extra) {
      atomicExch(a.ctrl + C_SNAP + (g & 1u), atomicAdd(a.ctrl + C_DONE, 0u));
      // barrier g ends phase g: phase g + 2 reuses the counter of phase g - 2
      atomicExch(a.ctrl + C_WORK + ((g + 2u) & 3u), 0u);
      atomicExch(a.ctrl + C_ARRIVE, 0u);
      __threadfence();
      atomicAdd(a.ctrl + C_GEN, 1u);
    } else {
      long long spins = 0;
      while (*gen == g) {
        if (++spins > a.spin_limit) {
          atomicCAS(a.ctrl + C_ERR, (unsigned)BE_NONE, (unsigned)BE_BARRIER);
          ok = 0;
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
    res = (ok && ldcg(a.ctrl + C_ERR) == BE_NONE) ? (int)ldcg(a.ctrl + C_SNAP + (g & 1u)) : -1;
  }
  __syncthreads();
  return res;
}

// The finishing CTA's warp 0: add the tiles' partial sums in tile order and
// advance the problem's state.
__device__ void finish_problem(const BArgs& a, int pi, const BProb& P, int mode) {
  const int lane = threadIdx.x;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int i = lane; i < P.ntiles; i += 32) {
    const int t = P.tile0 + i;
    s0 += ldcg(a.part + t);
    s1 += ldcg(a.part + a.nslots + t);
    s2 += ldcg(a.part + 2 * (size_t)a.nslots + t);
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  if (lane != 0) return;
  BState* sp = a.st + pi;
  BState s;
  s.mode = mode;
  s.status = ldcg(&sp->status);
  s.outer = ldcg(&sp->outer);
  s.it = ldcg(&sp->it);
  s.inner_total = ldcg(&sp->inner_total);
  s.pb = ldcg(&sp->pb);
  s.rz = ldcg(&sp->rz);
  s.alpha = ldcg(&sp->alpha);
  s.beta = ldcg(&sp->beta);
  s.rnrm0 = ldcg(&sp->rnrm0);
  s.bnorm = ldcg(&sp->bnorm);
  s.res = ldcg(&sp->res);
  s.inner_err = ldcg(&sp->inner_err);
  switch (mode) {
    case BM_RESID: {
      const double rn = sqrt(s0);
      if (s.outer == 0) s.bnorm = rn;
      if (s.outer == 0 && rn < DBL_EPSILON) {  // zero right-hand side: x = 0
        s.res = 0.0;
        s.status = LFG_OK;
        s.mode = BM_DONE;
        break;
      }
      s.res = rn / s.bnorm;
      if (isnan(s.res)) {
        s.status = LFG_NAN;
        s.mode = BM_DONE;
      } else if (s.res <= a.tol) {
        s.status = LFG_OK;
        s.mode = BM_DONE;
      } else if (s.outer >= a.max_outer) {
        s.status = LFG_NOT_CONVERGED;
        s.mode = BM_DONE;
      } else {
        s.rnrm0 = sqrt(s2);
        s.rz = s1;
        s.it = 0;
        s.pb |= 2;
        // cg_solve returns at once when |r0| < EPS (e stays 0)
        s.mode = s.rnrm0 < DBL_EPSILON ? BM_CORRECT : BM_APPLY;
      }
      break;
    }
    case BM_APPLY:
      s.alpha = s.rz / s0;
      s.pb = (s.pb & 1) ^ 1;  // the p just written is current; first step done
      s.mode = BM_UPDATE;
      break;
    case BM_UPDATE: {
      s.it += 1;
      s.inner_total += 1;
      s.inner_err = sqrt(s2) / s.rnrm0;
      if (s.inner_err <= a.inner_tol || s.it >= a.max_inner || isnan(s.inner_err)) {
        s.mode = BM_CORRECT;
      } else {
        s.beta = s1 / s.rz;
        s.rz = s1;
        s.mode = BM_APPLY;
      }
      break;
    }
    case BM_CORRECT:
      s.outer += 1;
      s.mode = BM_RESID;
      break;
    default:
      break;
  }
  *sp = s;
  atomicExch(a.cnt + pi, 0u);
  if (s.mode == BM_DONE) atomicAdd(a.ctrl + C_DONE, 1u);
}

// One column of one tile in the problem's current mode; partial sums into
// s0 (|r64|^2 or <p,q>), s1 (<r,z>), s2 (|r|^2).  dps: this thread's
// forward-substitution values, stride TC.  Levels go in chunks of U whose
// loads are all issued before any arithmetic (indices clamped into the
// column, so no load waits behind a branch).
constexpr int kU = 8;    // FP32 phases (6 loads a level)
constexpr int kUB = 16;  // the backward substitutions (2 loads a level)
constexpr int kUA = 2;   // the apply phase (17 loads a level)
constexpr int kU64 = 2;  // the FP64 residual phase

template <int TC>
__device__ __forceinline__ void column_step(const BProb& P, const BState* st, int mode, int c,
                                            float* dps, double& s0, double& s1, double& s2) {
  const int N = P.ncol, nl = P.nl;
  const size_t plane = (size_t)nl * N;
  int nb[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) nb[f] = __ldg(P.links + (size_t)f * N + c);
  float* __restrict__ e = P.e;
  float* __restrict__ r = P.r;
  float* __restrict__ z = P.z;
  float* __restrict__ q = P.q;
  const float* __restrict__ sub = P.sub;
  const float* __restrict__ inv = P.inv;
  const float* __restrict__ cp = P.cp;
  switch (mode) {
    case BM_RESID: {
      // r64 = b - A x in FP64 (T' row then minus the four couplings)
      double* __restrict__ x = P.x;
      double xm = 0.0, x0 = ldcg(x + c);
      float dprev = 0.f;
      for (int k0 = 0; k0 < nl; k0 += kU64) {
        double vs[kU64], vd[kU64], vu[kU64], vh[4][kU64], vx[kU64], vn[4][kU64], vb[kU64];
        float fs[kU64], fi[kU64];
#pragma unroll
        for (int u = 0; u < kU64; ++u) {
          const int kk = min(k0 + u, nl - 1);
          const size_t i = (size_t)kk * N + c;
          vs[u] = __ldg(P.sub64 + i);
          vd[u] = __ldg(P.diag64 + i);
          vu[u] = __ldg(P.sup64 + i);
#pragma unroll
          for (int f = 0; f < 4; ++f) {
            vh[f][u] = __ldg(P.h64 + f * plane + i);
            vn[f][u] = ldcg(x + (size_t)kk * N + nb[f]);
          }
          vx[u] = ldcg(x + (size_t)min(kk + 1, nl - 1) * N + c);
          vb[u] = __ldg(P.b + i);
          fs[u] = __ldg(sub + i);
          fi[u] = __ldg(inv + i);
        }
#pragma unroll
        for (int u = 0; u < kU64; ++u) {
          const int k = k0 + u;
          if (k < nl) {
            const size_t i = (size_t)k * N + c;
            const double xp = k + 1 < nl ? vx[u] : 0.0;
            double ax = k > 0 ? vs[u] * xm : 0.0;
            ax = ax + vd[u] * x0;
            if (k + 1 < nl) ax = ax + vu[u] * xp;
#pragma unroll
            for (int f = 0; f < 4; ++f) ax = ax - vh[f][u] * vn[f][u];
            const double r64 = vb[u] - ax;
            s0 += r64 * r64;
            const float rv = (float)r64;
            r[i] = rv;
            e[i] = 0.f;
            s2 += (double)rv * (double)rv;
            const float d = (k > 0 ? rv - fs[u] * dprev : rv) * fi[u];
            dps[k * TC] = d;
            dprev = d;
            xm = x0;
            x0 = xp;
          }
        }
      }
      float zn = 0.f;
      for (int k1 = nl - 1; k1 >= 0; k1 -= kUB) {
        float vc[kUB], vr[kUB];
#pragma unroll
        for (int u = 0; u < kUB; ++u) {
          const size_t i = (size_t)max(k1 - u, 0) * N + c;
          vc[u] = __ldg(cp + i);
          vr[u] = r[i];
        }
#pragma unroll
        for (int u = 0; u < kUB; ++u) {
          const int k = k1 - u;
          if (k >= 0) {
            const size_t i = (size_t)k * N + c;
            const float zv = dps[k * TC] - vc[u] * zn;
            z[i] = zv;
            s1 += (double)vr[u] * (double)zv;
            zn = zv;
          }
        }
      }
      break;
    }
    case BM_APPLY: {
      const float* __restrict__ dg = P.diag;
      const float* __restrict__ sp = P.sup;
      const float* __restrict__ h = P.h;
      const int pb = ldcg(&st->pb);
      const bool first = pb & 2;
      const float* __restrict__ pold = P.p[pb & 1];
      float* __restrict__ pnew = P.p[(pb & 1) ^ 1];
      const float be = first ? 0.f : (float)ldcg(&st->beta);
      // p = beta p + z, or z on a CG's first step: the same expression for
      // this column and its neighbours
      auto dirn = [&](float po, float zv) { return first ? zv : be * po + zv; };
      float pm = 0.f, p0 = dirn(first ? 0.f : ldcg(pold + c), ldcg(z + c));
      for (int k0 = 0; k0 < nl; k0 += kUA) {
        float vs[kUA], vd[kUA], vu[kUA], vh[4][kUA], vp[kUA], vz[kUA], vnp[4][kUA], vnz[4][kUA];
#pragma unroll
        for (int u = 0; u < kUA; ++u) {
          const int kk = min(k0 + u, nl - 1);
          const size_t i = (size_t)kk * N + c;
          const size_t i1 = (size_t)min(kk + 1, nl - 1) * N + c;
          vs[u] = __ldg(sub + i);
          vd[u] = __ldg(dg + i);
          vu[u] = __ldg(sp + i);
#pragma unroll
          for (int f = 0; f < 4; ++f) {
            vh[f][u] = __ldg(h + f * plane + i);
            vnz[f][u] = ldcg(z + (size_t)kk * N + nb[f]);
            vnp[f][u] = first ? 0.f : ldcg(pold + (size_t)kk * N + nb[f]);
          }
          vz[u] = ldcg(z + i1);
          vp[u] = first ? 0.f : ldcg(pold + i1);
        }
#pragma unroll
        for (int u = 0; u < kUA; ++u) {
          const int k = k0 + u;
          if (k < nl) {
            const float pp = k + 1 < nl ? dirn(vp[u], vz[u]) : 0.f;
            float ax = k > 0 ? vs[u] * pm : 0.f;
            ax = ax + vd[u] * p0;
            if (k + 1 < nl) ax = ax + vu[u] * pp;
#pragma unroll
            for (int f = 0; f < 4; ++f) ax = ax - vh[f][u] * dirn(vnp[f][u], vnz[f][u]);
            const size_t i = (size_t)k * N + c;
            pnew[i] = p0;
            q[i] = ax;
            s0 += (double)p0 * (double)ax;
            pm = p0;
            p0 = pp;
          }
        }
      }
      break;
    }
    case BM_UPDATE: {
      const float* __restrict__ p = P.p[ldcg(&st->pb) & 1];
      const double alpha = ldcg(&st->alpha);
      const float al = (float)alpha, mal = (float)(-alpha);
      float dprev = 0.f;
      for (int k0 = 0; k0 < nl; k0 += kU) {
        float vp[kU], vq[kU], ve[kU], vr[kU], vs[kU], vi[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const size_t i = (size_t)min(k0 + u, nl - 1) * N + c;
          vp[u] = ldcg(p + i);
          vq[u] = ldcg(q + i);
          ve[u] = ldcg(e + i);
          vr[u] = ldcg(r + i);
          vs[u] = __ldg(sub + i);
          vi[u] = __ldg(inv + i);
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const int k = k0 + u;
          if (k < nl) {
            const size_t i = (size_t)k * N + c;
            e[i] = ve[u] + al * vp[u];
            const float rv = vr[u] + mal * vq[u];
            r[i] = rv;
            s2 += (double)rv * (double)rv;
            const float d = (k > 0 ? rv - vs[u] * dprev : rv) * vi[u];
            dps[k * TC] = d;
            dprev = d;
          }
        }
      }
      float zn = 0.f;
      for (int k1 = nl - 1; k1 >= 0; k1 -= kUB) {
        float vc[kUB], vr[kUB];
#pragma unroll
        for (int u = 0; u < kUB; ++u) {
          const size_t i = (size_t)max(k1 - u, 0) * N + c;
          vc[u] = __ldg(cp + i);
          vr[u] = r[i];
        }
#pragma unroll
        for (int u = 0; u < kUB; ++u) {
          const int k = k1 - u;
          if (k >= 0) {
            const float zv = dps[k * TC] - vc[u] * zn;
            z[(size_t)k * N + c] = zv;
            s1 += (double)vr[u] * (double)zv;
            zn = zv;
          }
        }
      }
      break;
    }
    case BM_CORRECT: {
      double* __restrict__ x = P.x;
      for (int k0 = 0; k0 < nl; k0 += kU) {
        double vx[kU];
        float ve[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const size_t i = (size_t)min(k0 + u, nl - 1) * N + c;
          vx[u] = ldcg(x + i);
          ve[u] = ldcg(e + i);
        }
#pragma unroll
        for (int u = 0; u < kU; ++u)
          if (k0 + u < nl) x[(size_t)(k0 + u) * N + c] = vx[u] + (double)ve[u];
      }
      break;
    }
    default:
      break;
  }
}

template <int TC>
__global__ void __launch_bounds__(TC, 512 / TC) k_batch(BArgs a) {
  extern __shared__ float dps[];  // [nl_max][TC]
  __shared__ double red[3][TC / 32];
  __shared__ int last;
  __shared__ int s_next;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int phase = 0;; ++phase) {
    unsigned* work = a.ctrl + C_WORK + (phase & 3);
    if (tid == 0) s_next = (int)atomicAdd(work, 1u);
    __syncthreads();
    int t = s_next;
    while (t < a.ntiles) {
      __syncthreads();  // every thread has read s_next
      int nxt = 0;
      if (tid == 0) nxt = (int)atomicAdd(work, 1u);  // in flight while this tile runs
      const int2 tl = a.tiles[t];
      const BProb& P = a.probs[tl.x];
      const int mode = ldcg(&a.st[tl.x].mode);
      if (mode != BM_DONE) {
        const int slot = P.tile0 + tl.y / TC;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        const int c = tl.y + tid;
        if (c < P.ncol) column_step<TC>(P, a.st + tl.x, mode, c, dps + tid, s0, s1, s2);
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        s2 = warp_sum(s2);
        if (lane == 0) {
          red[0][warp] = s0;
          red[1][warp] = s1;
          red[2][warp] = s2;
        }
        __syncthreads();
        if (tid == 0) {
          double t0 = 0.0, t1 = 0.0, t2 = 0.0;
          for (int w = 0; w < TC / 32; ++w) {
            t0 += red[0][w];
            t1 += red[1][w];
            t2 += red[2][w];
          }
          a.part[slot] = t0;
          a.part[a.nslots + slot] = t1;
          a.part[2 * (size_t)a.nslots + slot] = t2;
          __threadfence();
          last = atomicAdd(a.cnt + tl.x, 1u) + 1 == (unsigned)P.ntiles;
        }
        __syncthreads();
        if (last && warp == 0) {
          __threadfence();
          finish_problem(a, tl.x, P, mode);
        }
      }
      if (tid == 0) s_next = nxt;
      __syncthreads();
      t = s_next;
    }
    const int ndone = grid_barrier(a);
    if (ndone < 0) return;
    if (ndone >= a.nprob) break;
    if (phase + 1 >= a.max_phases) {
      if (blockIdx.x == 0 && tid == 0)
        atomicCAS(a.ctrl + C_ERR, (unsigned)BE_NONE, (unsigned)BE_PHASES);
      break;
    }
  }
  if (blockIdx.x == 0 && tid == 0) {
    unsigned ph = 0;
    // phases run = number of completed barriers
    ph = ldcg(a.ctrl + C_GEN);
    a.ctrl[C_PHASES] = ph;
  }
}

constexpr int kTileChoices[3] = {64, 128, 256};
constexpr size_t kMaxBatchSmem = 200 * 1024;
constexpr long long kDefaultSpinLimit = 1ll << 24;  // x 128 ns sleeps: a few seconds

template <int TC>
void* kernel_of() { return (void*)&k_batch<TC>; }

void* batch_kernel(int tc) {
  switch (tc) {
    case 64: return kernel_of<64>();
    case 128: return kernel_of<128>();
    case 256: return kernel_of<256>();
  }
  throw Error(LFG_ERR_ARG, "batch: tile_cols must be 64, 128 or 256");
}

}  // namespace
}  // namespace lfg

using namespace lfg;

struct lfg_batch_s {
  lfg_ctx ctx = nullptr;
  int nprob = 0, nl_max = 0;
  size_t total = 0;
  lfg_batch_cfg cfg{};
  std::vector<lfg_helm> ops;           // FP64 operator of each problem (borrowed)
  std::map<lfg_helm, lfg_helm> op32;   // FP32 copies, owned
  std::vector<size_t> off;             // dof offset of each problem
  // device buffers
  double* b64 = nullptr;
  double* x64 = nullptr;
  float* v32 = nullptr;                // e, r, z, q, p (two buffers)
  BState* st = nullptr;
  BState* st0 = nullptr;
  double* part = nullptr;
  unsigned* cnt = nullptr;
  unsigned* ctrl = nullptr;
  // per tile width: descriptors and tile list
  std::map<int, BProb*> probs;
  std::map<int, int2*> tiles;
  std::map<int, int> ntiles;
  std::vector<lfg_field> rhs, sol;
  // launch shape
  int tc = 0, bpsm = 0, grid = 0;
  bool tuned = false;
  cudaGraphExec_t gexec = nullptr;
  unsigned barrier_extra = 0;
  std::vector<BState> h_st;
  unsigned h_ctrl[C_NCTRL] = {};
  int max_phases = 0;
};

namespace {

void build_tiles(lfg_batch b, int tc) {
  std::vector<BProb> hp(b->nprob);
  std::vector<int2> ht;
  const size_t T = b->total;
  for (int p = 0; p < b->nprob; ++p) {
    lfg_helm o = b->ops[p], f = b->op32.at(o);
    BProb& d = hp[p];
    d.ncol = o->ncol;
    d.nl = o->nl;
    d.tile0 = (int)ht.size();
    d.ntiles = (o->ncol + tc - 1) / tc;
    for (int i = 0; i < d.ntiles; ++i) ht.push_back(make_int2(p, i * tc));
    d.sub64 = (const double*)o->sub;
    d.diag64 = (const double*)o->diag;
    d.sup64 = (const double*)o->sup;
    d.h64 = (const double*)o->h;
    d.sub = (const float*)f->sub;
    d.diag = (const float*)f->diag;
    d.sup = (const float*)f->sup;
    d.h = (const float*)f->h;
    d.inv = (const float*)f->inv;
    d.cp = (const float*)f->cp;
    d.links = o->mesh->links;
    d.b = b->b64 + b->off[p];
    d.x = b->x64 + b->off[p];
    d.e = b->v32 + b->off[p];
    d.r = b->v32 + T + b->off[p];
    d.z = b->v32 + 2 * T + b->off[p];
    d.q = b->v32 + 3 * T + b->off[p];
    d.p[0] = b->v32 + 4 * T + b->off[p];
    d.p[1] = b->v32 + 5 * T + b->off[p];
  }
  // heaviest tiles first (levels x columns), then by problem and column
  std::stable_sort(ht.begin(), ht.end(), [&](const int2& u, const int2& v) {
    const long cu = (long)hp[u.x].nl * std::min(tc, hp[u.x].ncol - u.y);
    const long cv = (long)hp[v.x].nl * std::min(tc, hp[v.x].ncol - v.y);
    return cu > cv;
  });
  BProb* dp = (BProb*)dmalloc(sizeof(BProb) * hp.size());
  int2* dt = (int2*)dmalloc(sizeof(int2) * ht.size());
  LFG_CUDA(cudaMemcpy(dp, hp.data(), sizeof(BProb) * hp.size(), cudaMemcpyHostToDevice));
  LFG_CUDA(cudaMemcpy(dt, ht.data(), sizeof(int2) * ht.size(), cudaMemcpyHostToDevice));
  b->probs[tc] = dp;
  b->tiles[tc] = dt;
  b->ntiles[tc] = (int)ht.size();
}

size_t smem_of(lfg_batch b, int tc) { return (size_t)b->nl_max * tc * sizeof(float); }

// Largest co-resident CTAs per SM for tile width tc (0 when it does not fit).
int max_blocks_per_sm(lfg_batch b, int tc) {
  const size_t smem = smem_of(b, tc);
  if (smem > kMaxBatchSmem) return 0;
  void* k = batch_kernel(tc);
  LFG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int nb = 0;
  LFG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, tc, smem));
  return nb;
}

// Enqueue one whole batched solve: reset the state and launch the grid.
void enqueue(lfg_batch b, int tc, int bpsm) {
  lfg_ctx c = b->ctx;
  const int nb = max_blocks_per_sm(b, tc);
  LFG_REQUIRE(nb > 0 && bpsm >= 1 && bpsm <= nb, "batch: launch shape does not fit on an SM");
  LFG_CUDA(cudaMemsetAsync(b->x64, 0, sizeof(double) * b->total, c->stream));
  LFG_CUDA(cudaMemcpyAsync(b->st, b->st0, sizeof(BState) * b->nprob, cudaMemcpyDeviceToDevice,
                           c->stream));
  LFG_CUDA(cudaMemsetAsync(b->cnt, 0, sizeof(unsigned) * b->nprob, c->stream));
  LFG_CUDA(cudaMemsetAsync(b->ctrl, 0, sizeof(unsigned) * C_NCTRL, c->stream));
  BArgs a{};
  a.probs = b->probs.at(tc);
  a.st = b->st;
  a.tiles = b->tiles.at(tc);
  a.ntiles = b->ntiles.at(tc);
  a.nslots = a.ntiles;
  a.nprob = b->nprob;
  a.part = b->part;
  a.cnt = b->cnt;
  a.ctrl = b->ctrl;
  a.tol = b->cfg.tol;
  a.inner_tol = b->cfg.inner_tol;
  a.max_outer = b->cfg.max_outer;
  a.max_inner = b->cfg.max_inner;
  a.max_phases = b->max_phases;
  a.barrier_extra = b->barrier_extra;
  a.spin_limit = b->cfg.spin_limit > 0 ? b->cfg.spin_limit : kDefaultSpinLimit;
  cudaLaunchConfig_t lc{};
  lc.gridDim = dim3((unsigned)(bpsm * c->num_sms));
  lc.blockDim = dim3((unsigned)tc);
  lc.dynamicSmemBytes = smem_of(b, tc);
  lc.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  void* args[] = {&a};
  LFG_CUDA(cudaLaunchKernelExC(&lc, batch_kernel(tc), args));
  after_launch(c, "batch");
}

void check_done(lfg_batch b) {
  lfg_ctx c = b->ctx;
  LFG_CUDA(cudaMemcpyAsync(b->h_st.data(), b->st, sizeof(BState) * b->nprob,
                           cudaMemcpyDeviceToHost, c->stream));
  LFG_CUDA(cudaMemcpyAsync(b->h_ctrl, b->ctrl, sizeof(b->h_ctrl), cudaMemcpyDeviceToHost,
                           c->stream));
  LFG_CUDA(cudaStreamSynchronize(c->stream));
  if (b->h_ctrl[C_ERR] == BE_BARRIER)
    throw Error(LFG_ERR_STATE, "batch: a grid barrier wait ran out (spin limit reached)");
  if (b->h_ctrl[C_ERR] == BE_PHASES)
    throw Error(LFG_ERR_STATE, "batch: phase limit reached before every problem finished");
}

// Time every launch shape that fits once (after one untimed run) and keep
// the fastest; ties go to the earlier (narrower) candidate.
void autotune(lfg_batch b) {
  lfg_ctx c = b->ctx;
  std::vector<std::pair<int, int>> cands;
  for (int tc : kTileChoices) {
    if (b->cfg.tile_cols && tc != b->cfg.tile_cols) continue;
    const int nb = max_blocks_per_sm(b, tc);
    for (int bp = 1; bp <= nb; bp = bp * 2 > nb && bp < nb ? nb : bp * 2) {
      if (b->cfg.blocks_per_sm && bp != b->cfg.blocks_per_sm) continue;
      cands.push_back({tc, bp});
    }
    if (b->cfg.blocks_per_sm && b->cfg.blocks_per_sm <= nb &&
        std::find(cands.begin(), cands.end(), std::make_pair(tc, b->cfg.blocks_per_sm)) ==
            cands.end())
      cands.push_back({tc, b->cfg.blocks_per_sm});
  }
  LFG_REQUIRE(!cands.empty(), "batch: no launch shape fits (too many levels for shared memory?)");
  if (cands.size() == 1) {
    b->tc = cands[0].first;
    b->bpsm = cands[0].second;
  } else {
    cudaEvent_t e0, e1;
    LFG_CUDA(cudaEventCreate(&e0));
    LFG_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    for (auto& cd : cands) {
      enqueue(b, cd.first, cd.second);
      LFG_CUDA(cudaEventRecord(e0, c->stream));
      enqueue(b, cd.first, cd.second);
      LFG_CUDA(cudaEventRecord(e1, c->stream));
      LFG_CUDA(cudaEventSynchronize(e1));
      check_done(b);
      float ms = 0.f;
      LFG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) {
        best = ms;
        b->tc = cd.first;
        b->bpsm = cd.second;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  b->grid = b->bpsm * c->num_sms;
  b->tuned = true;
  if (b->cfg.use_graph) {
    cudaGraph_t g = nullptr;
    LFG_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue(b, b->tc, b->bpsm);
    } catch (...) {
      cudaStreamEndCapture(c->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    LFG_CUDA(cudaStreamEndCapture(c->stream, &g));
    const cudaError_t e = cudaGraphInstantiate(&b->gexec, g, 0);
    cudaGraphDestroy(g);
    LFG_CUDA(e);
  }
}

void release(lfg_batch b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  for (lfg_field f : b->rhs) lfg_field_destroy(f);
  for (lfg_field f : b->sol) lfg_field_destroy(f);
  for (auto& kv : b->probs) dfree(kv.second);
  for (auto& kv : b->tiles) dfree(kv.second);
  for (auto& kv : b->op32) lfg_helm_destroy(kv.second);
  dfree(b->b64);
  dfree(b->x64);
  dfree(b->v32);
  dfree(b->st);
  dfree(b->st0);
  dfree(b->part);
  dfree(b->cnt);
  dfree(b->ctrl);
}

}  // namespace

extern "C" {

int lfg_batch_create(lfg_ctx c, int nproblems, const lfg_helm* ops, const lfg_batch_cfg* cfg,
                     lfg_batch* out) {
  if (!c || !out || nproblems <= 0 || !ops) return LFG_ERR_ARG;
  lfg_batch b = new lfg_batch_s;
  b->ctx = c;
  const int rc = guard(c, [&] {
    b->nprob = nproblems;
    if (cfg) {
      b->cfg = *cfg;
    } else {
      b->cfg.tol = 1e-8;
      b->cfg.inner_tol = 1e-5;
      b->cfg.max_outer = 10;
      b->cfg.max_inner = 200;
      b->cfg.use_graph = 1;
    }
    LFG_REQUIRE(b->cfg.tol > 0 && b->cfg.inner_tol > 0 && b->cfg.max_outer >= 1 &&
                    b->cfg.max_inner >= 1,
                "batch_create: tolerances and iteration limits must be positive");
    LFG_REQUIRE(b->cfg.tile_cols == 0 || b->cfg.tile_cols == 64 || b->cfg.tile_cols == 128 ||
                    b->cfg.tile_cols == 256,
                "batch_create: tile_cols must be 0 (autotune), 64, 128 or 256");
    LFG_REQUIRE(b->cfg.blocks_per_sm >= 0, "batch_create: blocks_per_sm must be >= 0");
    for (int p = 0; p < nproblems; ++p) {
      lfg_helm o = ops[p];
      LFG_REQUIRE(o && o->ctx == c, "batch_create: operator of another context or NULL");
      LFG_REQUIRE(o->kind == LFG_R_DOUBLE, "batch_create: operators must be r_double");
      b->ops.push_back(o);
      b->off.push_back(b->total);
      b->total += (size_t)o->ncol * o->nl;
      b->nl_max = std::max(b->nl_max, o->nl);
      if (!b->op32.count(o)) {
        lfg_helm f = nullptr;
        const int r = lfg_helm_copy_kind(o, LFG_R_SINGLE, &f);
        if (r != LFG_OK) throw Error(r, "batch_create: FP32 copy of an operator failed");
        b->op32[o] = f;
      }
    }
    // phases: 2 per outer iteration (RESID, CORRECT) + 2 per inner one
    b->max_phases = (b->cfg.max_outer + 1) * (2 * b->cfg.max_inner + 2) + 4;
    const size_t T = b->total;
    b->b64 = (double*)dmalloc(sizeof(double) * T);
    b->x64 = (double*)dmalloc(sizeof(double) * T);
    b->v32 = (float*)dmalloc(sizeof(float) * 6 * T);
    LFG_CUDA(cudaMemset(b->b64, 0, sizeof(double) * T));
    LFG_CUDA(cudaMemset(b->x64, 0, sizeof(double) * T));
    b->st = (BState*)dmalloc(sizeof(BState) * nproblems);
    b->st0 = (BState*)dmalloc(sizeof(BState) * nproblems);
    std::vector<BState> s0(nproblems);
    for (auto& s : s0) {
      s = BState{};
      s.mode = BM_RESID;
      s.status = LFG_NOT_CONVERGED;
    }
    LFG_CUDA(cudaMemcpy(b->st0, s0.data(), sizeof(BState) * nproblems, cudaMemcpyHostToDevice));
    LFG_CUDA(cudaMemcpy(b->st, s0.data(), sizeof(BState) * nproblems, cudaMemcpyHostToDevice));
    b->h_st.resize(nproblems);
    int maxt = 0;
    for (int tc : kTileChoices) {
      build_tiles(b, tc);
      maxt = std::max(maxt, b->ntiles[tc]);
    }
    b->part = (double*)dmalloc(sizeof(double) * 3 * (size_t)maxt);
    b->cnt = (unsigned*)dmalloc(sizeof(unsigned) * nproblems);
    b->ctrl = (unsigned*)dmalloc(sizeof(unsigned) * C_NCTRL);
    for (int p = 0; p < nproblems; ++p) {
      lfg_field fr = nullptr, fx = nullptr;
      const int nl = b->ops[p]->nl, ncol = b->ops[p]->ncol;
      int r = lfg_field_wrap(c, LFG_R_DOUBLE, ncol, nl, b->b64 + b->off[p], &fr);
      if (r != LFG_OK) throw Error(r, "batch_create: field view");
      b->rhs.push_back(fr);
      r = lfg_field_wrap(c, LFG_R_DOUBLE, ncol, nl, b->x64 + b->off[p], &fx);
      if (r != LFG_OK) throw Error(r, "batch_create: field view");
      b->sol.push_back(fx);
    }
    if (b->cfg.tile_cols && b->cfg.blocks_per_sm) {
      b->tc = b->cfg.tile_cols;
      b->bpsm = b->cfg.blocks_per_sm;
      LFG_REQUIRE(max_blocks_per_sm(b, b->tc) >= b->bpsm,
                  "batch_create: blocks_per_sm exceeds what fits on an SM");
    }
  });
  if (rc != LFG_OK) {
    release(b);
    delete b;
    return rc;
  }
  *out = b;
  return LFG_OK;
}

int lfg_batch_destroy(lfg_batch b) {
  if (!b) return LFG_ERR_ARG;
  lfg_ctx c = b->ctx;
  const int rc = guard(c, [&] {
    LFG_CUDA(cudaStreamSynchronize(c->stream));
  });
  release(b);
  delete b;
  return rc;
}

int lfg_batch_rhs(lfg_batch b, int problem, lfg_field* rhs) {
  if (!b || !rhs || problem < 0 || problem >= b->nprob) return LFG_ERR_ARG;
  *rhs = b->rhs[problem];
  return LFG_OK;
}

int lfg_batch_solution(lfg_batch b, int problem, lfg_field* x) {
  if (!b || !x || problem < 0 || problem >= b->nprob) return LFG_ERR_ARG;
  *x = b->sol[problem];
  return LFG_OK;
}

int lfg_batch_launch(lfg_batch b) {
  if (!b) return LFG_ERR_ARG;
  return guard(b->ctx, [&] {
    if (!b->tuned) autotune(b);
    if (b->gexec) {
      LFG_CUDA(cudaGraphLaunch(b->gexec, b->ctx->stream));
      b->ctx->launches++;
    } else {
      enqueue(b, b->tc, b->bpsm);
    }
  });
}

int lfg_batch_wait(lfg_batch b, int* nfailed) {
  if (!b) return LFG_ERR_ARG;
  return guard(b->ctx, [&] {
    check_done(b);
    int nf = 0;
    for (const BState& s : b->h_st) nf += s.mode != BM_DONE || s.status != LFG_OK;
    if (nfailed) *nfailed = nf;
  });
}

int lfg_batch_solve(lfg_batch b, int* nfailed) {
  const int rc = lfg_batch_launch(b);
  if (rc != LFG_OK) return rc;
  return lfg_batch_wait(b, nfailed);
}

int lfg_batch_result(lfg_batch b, int problem, int* status, int* outer_iterations,
                     int* inner_iterations, double* rel_residual) {
  if (!b || problem < 0 || problem >= b->nprob) return LFG_ERR_ARG;
  const BState& s = b->h_st[problem];
  if (status) *status = s.mode == BM_DONE ? s.status : LFG_NOT_CONVERGED;
  if (outer_iterations) *outer_iterations = s.outer;
  if (inner_iterations) *inner_iterations = s.inner_total;
  if (rel_residual) *rel_residual = s.res;
  return LFG_OK;
}

int lfg_batch_tuning(lfg_batch b, int* tile_cols, int* blocks_per_sm, int* grid_blocks,
                     int* phases) {
  if (!b) return LFG_ERR_ARG;
  if (tile_cols) *tile_cols = b->tc;
  if (blocks_per_sm) *blocks_per_sm = b->bpsm;
  if (grid_blocks) *grid_blocks = b->tc ? b->bpsm * b->ctx->num_sms : 0;
  if (phases) *phases = (int)b->h_ctrl[C_PHASES];
  return LFG_OK;
}

int lfg_batch_test_stall(lfg_batch b, int extra_arrivals) {
  if (!b || extra_arrivals < 0) return LFG_ERR_ARG;
  return guard(b->ctx, [&] {
    b->barrier_extra = (unsigned)extra_arrivals;
    if (b->gexec) {  // the captured launch holds the old value
      LFG_CUDA(cudaGraphExecDestroy(b->gexec));
      b->gexec = nullptr;
      b->tuned = false;
    }
  });
}

}  // extern "C"

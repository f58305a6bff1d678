// The column substitutions of the block-Jacobi sweep with TMA staging
// (fine meshes; FP32, and FP64 in the register form):
//   d'_k = inv_k (r_k - sub_k d'_{k-1}),  z_k = d'_k - c'_k z_{k+1},
//   x_out = omega z + (1 - omega) x_in            (x_in optional)
//
// A persistent grid walks tiles of TC columns.  Every tile is a sequence of
// jobs: the forward chunks (KCH levels of r, inv, sub) bottom-up, then the
// backward chunks (KCH levels of c' and x_in) top-down.  One elected thread
// issues each job as 2-D TMA tile loads (cp.async.bulk.tensor) into a ring
// of NST shared-memory stages, completed on an mbarrier with an expected
// byte count; all threads (one per column) wait on the stage's barrier,
// compute, and leave the stage to the next job after a block barrier.  The
// bytes in flight are held by the TMA engine, not by registers, so the
// loads of the next NST-1 chunks overlap the recurrence of the current one.
// Between the passes d' stays in registers (k_subst_tma_reg, columns of up
// to 80 levels: the chunk count is a template parameter and the loops are
// fully unrolled; FP32 tiles of 128 columns, FP64 tiles of 64) or, for
// taller FP32 columns, in shared memory (k_subst_tma).
//
// Rules kept: every tile's first column is a multiple of the tile width,
// so the TMA's innermost coordinate times the element size is a multiple of
// 16 bytes; rows of the level-major arrays are N elements apart, so N must
// be a multiple of 4 (FP32) or 2 (FP64) (the host falls back to the
// per-column kernel otherwise); loads only (no TMA
// store), so out-of-range columns and levels of the last tile read zeros.
// Every wait is bounded: a barrier that does not complete within the spin
// limit sets the context's device error word, the block waits (bounded) for
// the loads it has issued and returns.  The stage-wait limit is a kernel
// argument, so a test can make the waits run out
// (lfg_ctx_test_tma_spin_limit); the drain keeps the built-in limit.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>

#include "lfg_internal.cuh"

namespace lfg {
namespace {

constexpr int TC = 128;     // columns per tile (box inner extent: 512 bytes)
constexpr int KCH = 16;     // levels per chunk
constexpr int NST = 3;      // ring stages
constexpr int NARR = 3;     // arrays per stage (forward: r, inv, sub; backward: c', x_in)
constexpr int kMaxLevels = 128;
constexpr long long kSpinLimit = 1ll << 22;
constexpr unsigned kErrTmaWait = 0x7101u;

struct TmaMaps {
  CUtensorMap r, inv, sub, cp, xin;
};

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// true when phase `parity` of the barrier has completed
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  long long spins = kSpinLimit) {
  for (long long i = 0; i < spins; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

template <bool XIN>
__global__ void __launch_bounds__(TC) k_subst_tma(const __grid_constant__ TmaMaps maps, int ncol,
                                                  int nl, float omega, float* __restrict__ xout,
                                                  unsigned* err, long long stage_spins) {
  grid_dep_wait();
  extern __shared__ __align__(128) unsigned char smem[];
  float* stage = reinterpret_cast<float*>(smem);                       // [NST][NARR][KCH][TC]
  float* sd = stage + NST * NARR * KCH * TC;                           // [nl][TC]
  __shared__ __align__(8) unsigned long long full[NST];
  __shared__ int s_abort;
  const int t = threadIdx.x;
  const int nch = (nl + KCH - 1) / KCH;
  const int ntile = (ncol + TC - 1) / TC;
  const int my_tiles = blockIdx.x < ntile ? (ntile - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int njobs = my_tiles * 2 * nch;
  if (t == 0) {
    for (int s = 0; s < NST; ++s) mbar_init(&full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  __syncthreads();
  // job j: tile blockIdx.x + (j / (2 nch)) * gridDim.x; forward chunk q for
  // q < nch, else backward chunk 2 nch - 1 - q
  auto issue = [&](int j) {
    const int s = j % NST;
    const int tile = blockIdx.x + (j / (2 * nch)) * gridDim.x;
    const int q = j % (2 * nch);
    const bool fwd = q < nch;
    const int chunk = fwd ? q : 2 * nch - 1 - q;
    const int c0 = tile * TC, k0 = chunk * KCH;
    float* dst = stage + (size_t)s * NARR * KCH * TC;
    const int narr = fwd ? 3 : (XIN ? 2 : 1);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&full[s], (unsigned)(narr * KCH * TC * sizeof(float)));
    if (fwd) {
      tma_load_2d(dst, &maps.r, c0, k0, &full[s]);
      tma_load_2d(dst + KCH * TC, &maps.inv, c0, k0, &full[s]);
      tma_load_2d(dst + 2 * KCH * TC, &maps.sub, c0, k0, &full[s]);
    } else {
      tma_load_2d(dst, &maps.cp, c0, k0, &full[s]);
      if (XIN) tma_load_2d(dst + KCH * TC, &maps.xin, c0, k0, &full[s]);
    }
  };
  if (t == 0)
    for (int j = 0; j < NST && j < njobs; ++j) issue(j);
  float d = 0.f, z = 0.f;
  const float om1 = 1.f - omega;
  int j = 0;
  for (; j < njobs; ++j) {
    const int s = j % NST;
    const unsigned parity = (unsigned)((j / NST) & 1);
    if (!mbar_wait_bounded(&full[s], parity, stage_spins)) {
      atomicCAS(err, 0u, kErrTmaWait);
      s_abort = 1;
    }
    __syncthreads();
    if (s_abort) break;
    const int tile = blockIdx.x + (j / (2 * nch)) * gridDim.x;
    const int q = j % (2 * nch);
    const float* st = stage + (size_t)s * NARR * KCH * TC;
    const int c = tile * TC + t;
    if (q < nch) {
      const int k0 = q * KCH;
#pragma unroll
      for (int u = 0; u < KCH; ++u) {
        const int k = k0 + u;
        const float rv = st[u * TC + t], iv = st[(KCH + u) * TC + t],
                    sb = st[(2 * KCH + u) * TC + t];
        if (k < nl) {
          d = k == 0 ? iv * rv : iv * (rv - sb * d);
          sd[k * TC + t] = d;
        }
      }
    } else {
      const int k0 = (2 * nch - 1 - q) * KCH;
#pragma unroll
      for (int u = KCH - 1; u >= 0; --u) {
        const int k = k0 + u;
        if (k < nl) {
          const float dk = sd[k * TC + t];
          z = (k == nl - 1) ? dk : dk - st[u * TC + t] * z;
          float v = omega * z;
          if (XIN) v = v + om1 * st[(KCH + u) * TC + t];
          if (c < ncol) xout[(size_t)k * ncol + c] = v;
        }
      }
    }
    __syncthreads();  // the stage has been read by every thread
    if (t == 0 && j + NST < njobs) issue(j + NST);
  }
  if (s_abort && t == 0) {
    // drain the loads this block has issued (bounded) before leaving
    for (int i = j; i < njobs && i < j + NST; ++i) {
      if (i >= njobs) break;
      mbar_wait_bounded(&full[i % NST], (unsigned)((i / NST) & 1));
    }
  }
}

// The same sweep with d' in registers: NCH = ceil(nl / KCH) is fixed at
// compile time, so each thread keeps its column's NCH*KCH values of d' in
// a fully unrolled register array instead of shared memory.  The stages
// are then all the shared memory a block needs, 3 blocks fit on an SM
// instead of 2, and half as many bytes again are in flight.  The job
// sequence, ring and bounded waits are those of k_subst_tma.  T is float
// (tiles of 128 columns) or double (tiles of 64): a box row is 512 bytes
// and a stage 24 KB either way.
constexpr int kRegChunks = 5;  // register form up to kRegChunks * KCH levels
template <class T>
__host__ __device__ constexpr int tile_cols() { return 512 / (int)sizeof(T); }

template <class T, bool XIN, int NCH>
__global__ void __launch_bounds__(tile_cols<T>(), 3)
    k_subst_tma_reg(const __grid_constant__ TmaMaps maps, int ncol, int nl, T omega,
                    T* __restrict__ xout, unsigned* err, long long stage_spins) {
  grid_dep_wait();
  constexpr int TCT = tile_cols<T>();
  extern __shared__ __align__(128) unsigned char smem[];
  T* stage = reinterpret_cast<T*>(smem);  // [NST][NARR][KCH][TCT]
  __shared__ __align__(8) unsigned long long full[NST];
  __shared__ int s_abort;
  const int t = threadIdx.x;
  constexpr int nch = NCH;
  const int ntile = (ncol + TCT - 1) / TCT;
  const int my_tiles = blockIdx.x < ntile ? (ntile - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int njobs = my_tiles * 2 * nch;
  if (t == 0) {
    for (int s = 0; s < NST; ++s) mbar_init(&full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  __syncthreads();
  auto issue = [&](int j) {
    const int s = j % NST;
    const int tile = blockIdx.x + (j / (2 * nch)) * gridDim.x;
    const int q = j % (2 * nch);
    const bool fwd = q < nch;
    const int chunk = fwd ? q : 2 * nch - 1 - q;
    const int c0 = tile * TCT, k0 = chunk * KCH;
    T* dst = stage + (size_t)s * NARR * KCH * TCT;
    const int narr = fwd ? 3 : (XIN ? 2 : 1);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&full[s], (unsigned)(narr * KCH * TCT * sizeof(T)));
    if (fwd) {
      tma_load_2d(dst, &maps.r, c0, k0, &full[s]);
      tma_load_2d(dst + KCH * TCT, &maps.inv, c0, k0, &full[s]);
      tma_load_2d(dst + 2 * KCH * TCT, &maps.sub, c0, k0, &full[s]);
    } else {
      tma_load_2d(dst, &maps.cp, c0, k0, &full[s]);
      if (XIN) tma_load_2d(dst + KCH * TCT, &maps.xin, c0, k0, &full[s]);
    }
  };
  // wait for job j's stage; false (for the whole block) when a wait ran out
  auto acquire = [&](int j) {
    if (!mbar_wait_bounded(&full[j % NST], (unsigned)((j / NST) & 1), stage_spins)) {
      atomicCAS(err, 0u, kErrTmaWait);
      s_abort = 1;
    }
    __syncthreads();
    return s_abort == 0;
  };
  auto release = [&](int j) {
    __syncthreads();  // the stage has been read by every thread
    if (t == 0 && j + NST < njobs) issue(j + NST);
  };
  if (t == 0)
    for (int j = 0; j < NST && j < njobs; ++j) issue(j);
  const T om1 = (T)1 - omega;
  int j = 0;
  bool ok = true;
  for (int it = 0; it < my_tiles && ok; ++it) {
    const int c = (blockIdx.x + it * gridDim.x) * TCT + t;
    T dreg[NCH * KCH];
    T d = (T)0;
#pragma unroll
    for (int q = 0; q < NCH; ++q) {
      if (!(ok = acquire(j))) break;
      const T* st = stage + (size_t)(j % NST) * NARR * KCH * TCT;
#pragma unroll
      for (int u = 0; u < KCH; ++u) {
        const int k = q * KCH + u;
        const T rv = st[u * TCT + t], iv = st[(KCH + u) * TCT + t],
                sb = st[(2 * KCH + u) * TCT + t];
        if (k < nl) d = k == 0 ? iv * rv : iv * (rv - sb * d);
        dreg[k] = d;
      }
      release(j++);
    }
    if (!ok) break;
    T z = (T)0;
#pragma unroll
    for (int q = NCH - 1; q >= 0; --q) {
      if (!(ok = acquire(j))) break;
      const T* st = stage + (size_t)(j % NST) * NARR * KCH * TCT;
#pragma unroll
      for (int u = KCH - 1; u >= 0; --u) {
        const int k = q * KCH + u;
        if (k < nl) {
          z = (k == nl - 1) ? dreg[k] : dreg[k] - st[u * TCT + t] * z;
          T v = omega * z;
          if (XIN) v = v + om1 * st[(KCH + u) * TCT + t];
          if (c < ncol) xout[(size_t)k * ncol + c] = v;
        }
      }
      release(j++);
    }
  }
  if (!ok && t == 0) {
    // drain the loads this block has issued (bounded) before leaving
    for (int i = j; i < njobs && i < j + NST; ++i)
      mbar_wait_bounded(&full[i % NST], (unsigned)((i / NST) & 1));
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 2-D tensor map over a level-major array [nl][ncol] of T, box KCH levels
// x tile_cols<T>() columns (512 bytes).
template <class T>
CUtensorMap make_map(const T* base, int ncol, int nl) {
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  const cuuint64_t dims[2] = {(cuuint64_t)ncol, (cuuint64_t)nl};
  const cuuint64_t strides[1] = {(cuuint64_t)ncol * sizeof(T)};
  const cuuint32_t box[2] = {(cuuint32_t)tile_cols<T>(), (cuuint32_t)KCH};
  const cuuint32_t estr[2] = {1, 1};
  const CUtensorMapDataType dt =
      sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const CUresult r = encode_fn()(&m, dt, 2, (void*)base, dims,
                                 strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(LFG_ERR_CUDA, "tensor map encode failed");
  return m;
}

// Stage-wait limit of a launch: the context's test setting, else the
// built-in one.  The drain after a wait ran out always uses the built-in
// limit, so every load a block issued has landed before it returns.
long long stage_spins(lfg_ctx c) {
  return c->tma_stage_spins >= 0 ? c->tma_stage_spins : kSpinLimit;
}

size_t smem_bytes(int nl) {
  return sizeof(float) * ((size_t)NST * NARR * KCH * TC + (size_t)nl * TC);
}

}  // namespace

bool subst_tma_applicable(lfg_ctx c, int ncol, int nl, const void* const* ptrs, int nptr,
                          int elem_bytes) {
  if (!c->dev_err || nl < 1 || nl > kMaxLevels) return false;
  if (elem_bytes == 4) {
    if (ncol % 4 != 0 || ncol < 2 * TC) return false;
  } else {  // FP64: the register form only
    if (elem_bytes != 8 || ncol % 2 != 0 || ncol < 2 * tile_cols<double>() ||
        nl > kRegChunks * KCH)
      return false;
  }
  for (int i = 0; i < nptr; ++i)
    if (ptrs[i] && reinterpret_cast<uintptr_t>(ptrs[i]) % 16 != 0) return false;
  return encode_fn() != nullptr;
}

namespace {

// f(n, kernel) for the register kernels of n = N, N-1, ..., 1 chunks
template <class T, bool X, int N, class F>
void for_reg_kernels(F&& f) {
  f(N, (const void*)k_subst_tma_reg<T, X, N>);
  if constexpr (N > 1) for_reg_kernels<T, X, N - 1>(f);
}

template <class T>
void launch_reg(lfg_ctx c, const TmaMaps& maps, int ncol, int nl, bool xin, T omega, T* xout) {
  constexpr int TCT = tile_cols<T>();
  const int nch = (nl + KCH - 1) / KCH;
  const size_t smem = sizeof(T) * (size_t)NST * NARR * KCH * TCT;
  const void* kern = nullptr;
  auto pick = [&](int n, const void* k) {
    if (n == nch) kern = k;
  };
  if (xin) for_reg_kernels<T, true, kRegChunks>(pick);
  else for_reg_kernels<T, false, kRegChunks>(pick);
  if (!kern) throw Error(LFG_ERR_ARG, "subst_tma: column taller than the register form");
  ensure_smem_attr(kern, (int)smem);
  int per_sm = 0;
  LFG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TCT, smem));
  const int ntile = (ncol + TCT - 1) / TCT;
  const int grid = std::max(1, std::min(ntile, c->num_sms * std::max(per_sm, 1)));
  TmaMaps m = maps;
  int nc = ncol, nlv = nl;
  T om = omega;
  T* xo = xout;
  unsigned* err = c->dev_err;
  long long spins = stage_spins(c);
  void* args[] = {&m, &nc, &nlv, &om, &xo, &err, &spins};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(TCT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = c->pdl ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  LFG_CUDA(cudaLaunchKernelExC(&cfg, kern, args));
  // r, inv, sub, c' read and x written, x_in read when given
  after_launch(c, "helm_subst_tma", sizeof(T) * (uint64_t)ncol * nl * (xin ? 6 : 5));
}

template <class T>
TmaMaps maps_of(int ncol, int nl, const T* r, const T* sub, const T* inv, const T* cp,
                const T* xin) {
  TmaMaps maps;
  maps.r = make_map(r, ncol, nl);
  maps.inv = make_map(inv, ncol, nl);
  maps.sub = make_map(sub, ncol, nl);
  maps.cp = make_map(cp, ncol, nl);
  maps.xin = make_map(xin ? xin : cp, ncol, nl);
  return maps;
}

}  // namespace

// Launches the TMA substitution; xin may be null (zero start).  The caller
// checked subst_tma_applicable.
void subst_tma(lfg_ctx c, int ncol, int nl, const float* r, const float* sub, const float* inv,
               const float* cp, const float* xin, float omega, float* xout) {
  const TmaMaps maps = maps_of(ncol, nl, r, sub, inv, cp, xin);
  if ((nl + KCH - 1) / KCH <= kRegChunks) {
    launch_reg<float>(c, maps, ncol, nl, xin != nullptr, omega, xout);
    return;
  }
  const size_t smem = smem_bytes(nl);
  const void* kern = xin ? (const void*)k_subst_tma<true> : (const void*)k_subst_tma<false>;
  ensure_smem_attr(kern, (int)smem_bytes(kMaxLevels));
  int per_sm = 0;
  LFG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TC, smem));
  const int ntile = (ncol + TC - 1) / TC;
  const int grid = std::max(1, std::min(ntile, c->num_sms * std::max(per_sm, 1)));
  if (xin)
    launch_pdl(c, k_subst_tma<true>, grid, TC, smem, maps, ncol, nl, omega, xout, c->dev_err,
               stage_spins(c));
  else
    launch_pdl(c, k_subst_tma<false>, grid, TC, smem, maps, ncol, nl, omega, xout, c->dev_err,
               stage_spins(c));
  after_launch(c, "helm_subst_tma", sizeof(float) * (uint64_t)ncol * nl * (xin ? 6 : 5));
}

void subst_tma(lfg_ctx c, int ncol, int nl, const double* r, const double* sub,
               const double* inv, const double* cp, const double* xin, double omega,
               double* xout) {
  launch_reg<double>(c, maps_of(ncol, nl, r, sub, inv, cp, xin), ncol, nl, xin != nullptr,
                     omega, xout);
}

}  // namespace lfg

// Context, fields, host<->device transfers and the vector-algebra built-ins.
//
// The built-ins replace the PSyclone built-ins invoked by the reference's
// field vectors (components/science/source/algorithm/solver/
// sci_field_vector_mod.x90:132-286, sci_r_solver_field_vector_mod.x90:119-296)
// and the FP64-accumulated inner products of the hand-written PSy layer
// (components/science/source/psy/sci_psykal_light_mod.f90:72-214).  Every
// inner product is a deterministic two-level reduction: fixed grid-stride
// partition, fixed-order block tree, and the last block to finish sums the
// per-block partials in index order -- no floating-point atomics, so repeated
// runs are bit-identical.
#include "lfg_internal.cuh"

#include <map>
#include <utility>

#include <cstdlib>
#include <cstring>

using namespace lfg;

namespace lfg {

void* dmalloc(size_t bytes) {
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess)
    throw Error(LFG_ERR_NOMEM, std::string("cudaMalloc(") + std::to_string(bytes) +
                                   "): " + cudaGetErrorString(e));
  return p;
}
void dfree(void* p) {
  if (p) cudaFree(p);
}
void upload(void* d, const void* h, size_t bytes) {
  LFG_CUDA(cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice));
}

// ------------------------------------------------------------ kernels
// The vector algebra streams its arrays in 16-byte packs (4 floats or 2
// doubles per load) when every pointer is 16-byte aligned, so each load
// instruction moves four times the bytes of a scalar FP32 load; a scalar
// tail (and the scalar path for unaligned views) covers the rest.  Each
// kernel is an element operation applied to W consecutive elements; the
// scalars (Sc) are evaluated once per thread.
template <class T, int W>
struct Pack {
  T e[W];
  __device__ __forceinline__ static Pack load(const T* p) {
    Pack r;
    if constexpr (W * sizeof(T) == 16) {
      const uint4 q = *reinterpret_cast<const uint4*>(p);
      memcpy(r.e, &q, 16);
    } else {
#pragma unroll
      for (int i = 0; i < W; ++i) r.e[i] = p[i];
    }
    return r;
  }
  __device__ __forceinline__ void store(T* p) const {
    if constexpr (W * sizeof(T) == 16) {
      uint4 q;
      memcpy(&q, e, 16);
      *reinterpret_cast<uint4*>(p) = q;
    } else {
#pragma unroll
      for (int i = 0; i < W; ++i) p[i] = e[i];
    }
  }
};

template <class T>
constexpr int kVec = 16 / (int)sizeof(T);

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Applies op over [0, n): packs of W = 16 / sizeof(T) elements, then the tail.
template <class T, class Op>
__device__ __forceinline__ void for_each_pack(const Op& op, size_t n, bool vec, double& acc) {
  const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t st = (size_t)gridDim.x * blockDim.x;
  size_t i0 = 0;
  if (vec) {
    constexpr int W = kVec<T>;
    const size_t nv = n / W;
    for (size_t j = tid; j < nv; j += st) op.template run<W>(j * W, acc);
    i0 = nv * W;
  }
  for (size_t i = i0 + tid; i < n; i += st) op.template run<1>(i, acc);
}

template <class T, class Op>
__global__ void k_ew(Op op, size_t n, bool vec) {
  grid_dep_wait();
  double acc = 0.0;
  const auto b = op.bind();
  for_each_pack<T>(b, n, vec, acc);
}

template <class T, class Op>
__global__ void k_ewr(Op op, size_t n, bool vec, Red r) {
  grid_dep_wait();
  double acc = 0.0;
  const auto b = op.bind();
  for_each_pack<T>(b, n, vec, acc);
  red_finish(r, acc);
}

#define LFG_PACK(T, W, name, ptr, i) const Pack<T, W> name = Pack<T, W>::load((ptr) + (i))

// X = c
template <class T>
struct SetOp {
  T* x;
  Sc a;
  struct B {
    T* x;
    T v;
    template <int W> __device__ void run(size_t i, double&) const {
      Pack<T, W> o;
#pragma unroll
      for (int q = 0; q < W; ++q) o.e[q] = v;
      o.store(x + i);
    }
  };
  __device__ B bind() const { return B{x, (T)sc_eval(a)}; }
};

template <class TO, class TI>
__global__ void k_copy(TO* __restrict__ y, const TI* __restrict__ x, size_t n) {
  grid_dep_wait();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = (TO)x[i];
}

// Y = X, same kind
template <class T>
struct CopyOp {
  T* y;
  const T* x;
  struct B {
    T* y;
    const T* x;
    template <int W> __device__ void run(size_t i, double&) const {
      Pack<T, W>::load(x + i).store(y + i);
    }
  };
  __device__ B bind() const { return B{y, x}; }
};

// X = X + b Y   (inc_X_plus_bY); Y may be of another kind (r_def += r_solver,
// sci_psykal_light_mod.f90:218-265), the product is then formed in X's kind.
template <class T, class TY>
__global__ void k_axpy(T* __restrict__ x, const TY* __restrict__ y, size_t n, Sc b) {
  grid_dep_wait();
  const T bv = (T)sc_eval(b);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    x[i] = x[i] + bv * (T)y[i];
}

template <class T>
struct AxpyOp {  // X = X + b Y, same kind
  T* x;
  const T* y;
  Sc b;
  struct B {
    T* x;
    const T* y;
    T bv;
    template <int W> __device__ void run(size_t i, double&) const {
      LFG_PACK(T, W, xv, x, i);
      LFG_PACK(T, W, yv, y, i);
      Pack<T, W> o;
#pragma unroll
      for (int q = 0; q < W; ++q) o.e[q] = xv.e[q] + bv * yv.e[q];
      o.store(x + i);
    }
  };
  __device__ B bind() const { return B{x, y, (T)sc_eval(b)}; }
};

// X = a X + Y   (inc_aX_plus_Y)
template <class T>
struct AypxOp {
  T* x;
  const T* y;
  Sc a;
  struct B {
    T* x;
    const T* y;
    T av;
    template <int W> __device__ void run(size_t i, double&) const {
      LFG_PACK(T, W, xv, x, i);
      LFG_PACK(T, W, yv, y, i);
      Pack<T, W> o;
#pragma unroll
      for (int q = 0; q < W; ++q) o.e[q] = av * xv.e[q] + yv.e[q];
      o.store(x + i);
    }
  };
  __device__ B bind() const { return B{x, y, (T)sc_eval(a)}; }
};

// Z = a X + b Y   (aX_plus_bY)
template <class T>
struct AxpbyOp {
  T* z;
  const T* x;
  const T* y;
  Sc a, b;
  struct B {
    T* z;
    const T* x;
    const T* y;
    T av, bv;
    template <int W> __device__ void run(size_t i, double&) const {
      LFG_PACK(T, W, xv, x, i);
      LFG_PACK(T, W, yv, y, i);
      Pack<T, W> o;
#pragma unroll
      for (int q = 0; q < W; ++q) o.e[q] = av * xv.e[q] + bv * yv.e[q];
      o.store(z + i);
    }
  };
  __device__ B bind() const { return B{z, x, y, (T)sc_eval(a), (T)sc_eval(b)}; }
};

// X = a X   (inc_a_times_X)
template <class T>
struct ScaleOp {
  T* x;
  Sc a;
  struct B {
    T* x;
    T av;
    template <int W> __device__ void run(size_t i, double&) const {
      LFG_PACK(T, W, xv, x, i);
      Pack<T, W> o;
#pragma unroll
      for (int q = 0; q < W; ++q) o.e[q] = av * xv.e[q];
      o.store(x + i);
    }
  };
  __device__ B bind() const { return B{x, (T)sc_eval(a)}; }
};

// Z = X / Y   (X_divideby_Y)
template <class T>
__global__ void k_divide(T* __restrict__ z, const T* __restrict__ x, const T* __restrict__ y,
                         size_t n) {
  grid_dep_wait();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    z[i] = x[i] / y[i];
}

// <X, Y> accumulated in double
template <class T>
struct DotOp {
  const T* x;
  const T* y;
  struct B {
    const T* x;
    const T* y;
    template <int W> __device__ void run(size_t i, double& acc) const {
      LFG_PACK(T, W, xv, x, i);
      LFG_PACK(T, W, yv, y, i);
#pragma unroll
      for (int q = 0; q < W; ++q) acc += (double)xv.e[q] * (double)yv.e[q];
    }
  };
  __device__ B bind() const { return B{x, y}; }
};

// Modified Gram-Schmidt step of gcr_solve (sci_iterative_solver_mod.f90:1358-1362)
// fused with the next inner product: v -= a vj; pv -= a pvj; acc <v, next>
// (next == null: <v, v>, the norm that follows the loop).
template <class T>
struct MgsOp {
  T* v;
  T* pv;
  const T* vj;
  const T* pvj;
  const T* next;
  Sc a;
  struct B {
    T* v;
    T* pv;
    const T* vj;
    const T* pvj;
    const T* next;
    T av;
    template <int W> __device__ void run(size_t i, double& acc) const {
      LFG_PACK(T, W, vv, v, i);
      LFG_PACK(T, W, vjv, vj, i);
      LFG_PACK(T, W, pvv, pv, i);
      LFG_PACK(T, W, pvjv, pvj, i);
      Pack<T, W> nv, np, w;
#pragma unroll
      for (int q = 0; q < W; ++q) {
        nv.e[q] = vv.e[q] + av * vjv.e[q];
        np.e[q] = pvv.e[q] + av * pvjv.e[q];
      }
      if (next) w = Pack<T, W>::load(next + i);
      else w = nv;
#pragma unroll
      for (int q = 0; q < W; ++q) acc += (double)nv.e[q] * (double)w.e[q];
      nv.store(v + i);
      np.store(pv + i);
    }
  };
  __device__ B bind() const { return B{v, pv, vj, pvj, next, (T)sc_eval(a)}; }
};

// v *= b; pv *= b; acc <res, v>   (gcr_solve :1363-1367)
template <class T>
struct Scale2DotOp {
  T* v;
  T* pv;
  const T* res;
  Sc b;
  struct B {
    T* v;
    T* pv;
    const T* res;
    T bv;
    template <int W> __device__ void run(size_t i, double& acc) const {
      LFG_PACK(T, W, vv, v, i);
      LFG_PACK(T, W, pvv, pv, i);
      LFG_PACK(T, W, rv, res, i);
      Pack<T, W> nv, np;
#pragma unroll
      for (int q = 0; q < W; ++q) {
        nv.e[q] = bv * vv.e[q];
        np.e[q] = bv * pvv.e[q];
        acc += (double)rv.e[q] * (double)nv.e[q];
      }
      nv.store(v + i);
      np.store(pv + i);
    }
  };
  __device__ B bind() const { return B{v, pv, res, (T)sc_eval(b)}; }
};

// dx += a pv; res -= a v; acc <res, res>   (gcr_solve :1368-1374)
template <class T>
struct Update2NormOp {
  T* dx;
  const T* pv;
  T* res;
  const T* v;
  Sc a;
  struct B {
    T* dx;
    const T* pv;
    T* res;
    const T* v;
    T ap, am;
    template <int W> __device__ void run(size_t i, double& acc) const {
      LFG_PACK(T, W, dv, dx, i);
      LFG_PACK(T, W, pvv, pv, i);
      LFG_PACK(T, W, rv, res, i);
      LFG_PACK(T, W, vv, v, i);
      Pack<T, W> nd, nr;
#pragma unroll
      for (int q = 0; q < W; ++q) {
        nd.e[q] = dv.e[q] + ap * pvv.e[q];
        nr.e[q] = rv.e[q] + am * vv.e[q];
        acc += (double)nr.e[q] * (double)nr.e[q];
      }
      nd.store(dx + i);
      nr.store(res + i);
    }
  };
  __device__ B bind() const {
    const double ad = sc_eval(a);
    return B{dx, pv, res, v, (T)ad, (T)(-ad)};
  }
};

// The CG update of one iteration in one pass (cg_solve,
// sci_iterative_solver_mod.f90:560-575): x += a p, r -= a q, acc <r, r>, and
// the new x also written to snap when given.  Each value is formed as the
// separate axpy kernels form it.
template <class T>
struct CgUpdateOp {
  T* x;
  const T* p;
  T* r;
  const T* q;
  T* snap;
  Sc a;
  struct B {
    T* x;
    const T* p;
    T* r;
    const T* q;
    T* snap;
    T ap, am;
    template <int W> __device__ void run(size_t i, double& acc) const {
      LFG_PACK(T, W, xv, x, i);
      LFG_PACK(T, W, pv, p, i);
      LFG_PACK(T, W, rv, r, i);
      LFG_PACK(T, W, qv, q, i);
      Pack<T, W> nx, nr;
#pragma unroll
      for (int k = 0; k < W; ++k) {
        nx.e[k] = xv.e[k] + ap * pv.e[k];
        nr.e[k] = rv.e[k] + am * qv.e[k];
        acc += (double)nr.e[k] * (double)nr.e[k];
      }
      nx.store(x + i);
      if (snap) nx.store(snap + i);
      nr.store(r + i);
    }
  };
  __device__ B bind() const {
    const double ad = sc_eval(a);
    return B{x, p, r, q, snap, (T)ad, (T)(-ad)};
  }
};

// z = x / d and acc <x, z> in one pass: the diagonal preconditioner's apply
// (X_divideby_Y) with the inner product that follows it in cg_solve.
template <class T>
struct DivideDotOp {
  T* z;
  const T* x;
  const T* d;
  struct B {
    T* z;
    const T* x;
    const T* d;
    template <int W> __device__ void run(size_t i, double& acc) const {
      LFG_PACK(T, W, xv, x, i);
      LFG_PACK(T, W, dv, d, i);
      Pack<T, W> o;
#pragma unroll
      for (int k = 0; k < W; ++k) {
        o.e[k] = xv.e[k] / dv.e[k];
        acc += (double)xv.e[k] * (double)o.e[k];
      }
      o.store(z + i);
    }
  };
  __device__ B bind() const { return B{z, x, d}; }
};

// x += b y; acc <x, next> (next null: <x, x>)  (gmres/fgmres Arnoldi, and
// the monitored residual update of bicgstab / jacobi)
template <class T>
struct AxpyDotOp {
  T* x;
  const T* y;
  const T* next;
  Sc b;
  struct B {
    T* x;
    const T* y;
    const T* next;
    T bv;
    template <int W> __device__ void run(size_t i, double& acc) const {
      LFG_PACK(T, W, xv, x, i);
      LFG_PACK(T, W, yv, y, i);
      Pack<T, W> o, w;
#pragma unroll
      for (int q = 0; q < W; ++q) o.e[q] = xv.e[q] + bv * yv.e[q];
      if (next) w = Pack<T, W>::load(next + i);
      else w = o;
#pragma unroll
      for (int q = 0; q < W; ++q) acc += (double)o.e[q] * (double)w.e[q];
      o.store(x + i);
    }
  };
  __device__ B bind() const { return B{x, y, next, (T)sc_eval(b)}; }
};

// dst = a src   (copy followed by inc_a_times_X)
template <class T>
struct ScaleCopyOp {
  T* dst;
  const T* src;
  Sc a;
  struct B {
    T* dst;
    const T* src;
    T av;
    template <int W> __device__ void run(size_t i, double&) const {
      LFG_PACK(T, W, sv, src, i);
      Pack<T, W> o;
#pragma unroll
      for (int q = 0; q < W; ++q) o.e[q] = av * sv.e[q];
      o.store(dst + i);
    }
  };
  __device__ B bind() const { return B{dst, src, (T)sc_eval(a)}; }
};

// Column-contiguous (e*nlev + k) <-> level-major (k*ncol + e) with kind
// conversion, through 32x32 shared-memory tiles.
template <class TO, class TI>
__global__ void k_to_level_major(TO* __restrict__ out, const TI* __restrict__ in, int ncol,
                                 int nlev) {
  __shared__ TI tile[32][33];
  const int e0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    int e = e0 + j, k = k0 + threadIdx.x;
    if (e < ncol && k < nlev) tile[j][threadIdx.x] = in[(size_t)e * nlev + k];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    int k = k0 + j, e = e0 + threadIdx.x;
    if (e < ncol && k < nlev) out[(size_t)k * ncol + e] = (TO)tile[threadIdx.x][j];
  }
}

template <class TO, class TI>
__global__ void k_to_column(TO* __restrict__ out, const TI* __restrict__ in, int ncol,
                            int nlev) {
  __shared__ TI tile[32][33];
  const int e0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    int k = k0 + j, e = e0 + threadIdx.x;
    if (e < ncol && k < nlev) tile[j][threadIdx.x] = in[(size_t)k * ncol + e];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    int e = e0 + j, k = k0 + threadIdx.x;
    if (e < ncol && k < nlev) out[(size_t)e * nlev + k] = (TO)tile[threadIdx.x][j];
  }
}

// ------------------------------------------------------------ launchers
#define DISPATCH_KIND(kind, T, ...)                         \
  do {                                                      \
    if ((kind) == LFG_R_DOUBLE) {                           \
      using T = double;                                     \
      __VA_ARGS__;                                          \
    } else {                                                \
      using T = float;                                      \
      __VA_ARGS__;                                          \
    }                                                       \
  } while (0)

static void same_shape(lfg_field a, lfg_field b, const char* what) {
  LFG_REQUIRE(a && b, std::string(what) + ": null field");
  LFG_REQUIRE(a->ncol == b->ncol && a->nlev == b->nlev,
              std::string(what) + ": fields differ in shape");
}
static void same_kind(lfg_field a, lfg_field b, const char* what) {
  same_shape(a, b, what);
  LFG_REQUIRE(a->kind == b->kind, std::string(what) + ": fields differ in kind");
}

// words: arrays the operation reads plus arrays it writes (n values each)
template <class T, class Op>
void launch_ew(lfg_ctx c, const Op& op, size_t n, bool vec, const char* what, int words) {
  const size_t work = vec ? n / kVec<T> + n % kVec<T> : n;
  launch_pdl(c, k_ew<T, Op>, occ_grid(c, (const void*)k_ew<T, Op>, kThreads, work), kThreads, 0,
             op, n, vec);
  after_launch(c, what, (uint64_t)words * n * sizeof(T));
}

// out: where the reduction's result goes (null: the slot's result word)
template <class T, class Op>
void launch_ewr(lfg_ctx c, const Op& op, size_t n, bool vec, int slot, const char* what,
                int words, double* out = nullptr) {
  const size_t work = vec ? n / kVec<T> + n % kVec<T> : n;
  // the reduction's partials live in kMaxRedBlocks slots per reduction
  const int g = std::min(occ_grid(c, (const void*)k_ewr<T, Op>, kThreads, work), kMaxRedBlocks);
  Red r = c->red(slot);
  if (out) r.result = out;
  launch_pdl(c, k_ewr<T, Op>, g, kThreads, 0, op, n, vec, r);
  after_launch(c, what, (uint64_t)words * n * sizeof(T));
}

template <class... P>
bool all_aligned(const P*... p) {
  return (... && (p == nullptr || aligned16(p)));
}

void vec_set(lfg_field x, Sc a) {
  lfg_ctx c = x->ctx;
  DISPATCH_KIND(x->kind, T, launch_ew<T>(c, SetOp<T>{(T*)x->d, a}, x->n(), all_aligned(x->d), "set", 1));
}

void vec_copy(lfg_field dst, lfg_field src) {
  same_shape(dst, src, "copy");
  lfg_ctx c = dst->ctx;
  if (dst->kind == src->kind) {
    DISPATCH_KIND(dst->kind, T,
                  launch_ew<T>(c, CopyOp<T>{(T*)dst->d, (const T*)src->d}, dst->n(),
                               all_aligned(dst->d, src->d), "copy", 2));
    return;
  }
  const int g = c->stream_grid(dst->n());
  if (dst->kind == LFG_R_DOUBLE)
    launch_pdl(c, k_copy<double, float>, g, kThreads, 0, (double*)dst->d, (const float*)src->d,
               dst->n());
  else
    launch_pdl(c, k_copy<float, double>, g, kThreads, 0, (float*)dst->d, (const double*)src->d,
               dst->n());
  after_launch(c, "copy", (uint64_t)dst->n() * (dst->kind + src->kind));
}

void vec_axpy(lfg_field x, Sc b, lfg_field y) {
  same_shape(x, y, "inc_X_plus_bY");
  lfg_ctx c = x->ctx;
  if (x->kind == y->kind) {
    DISPATCH_KIND(x->kind, T,
                  launch_ew<T>(c, AxpyOp<T>{(T*)x->d, (const T*)y->d, b}, x->n(),
                               all_aligned(x->d, y->d), "axpy", 3));
    return;
  }
  const int g = c->stream_grid(x->n());
  if (x->kind == LFG_R_DOUBLE)
    launch_pdl(c, k_axpy<double, float>, g, kThreads, 0, (double*)x->d, (const float*)y->d,
               x->n(), b);
  else
    launch_pdl(c, k_axpy<float, double>, g, kThreads, 0, (float*)x->d, (const double*)y->d,
               x->n(), b);
  after_launch(c, "axpy", (uint64_t)x->n() * (2 * x->kind + y->kind));
}

void vec_aypx(lfg_field x, Sc a, lfg_field y) {
  same_kind(x, y, "inc_aX_plus_Y");
  lfg_ctx c = x->ctx;
  DISPATCH_KIND(x->kind, T,
                launch_ew<T>(c, AypxOp<T>{(T*)x->d, (const T*)y->d, a}, x->n(),
                             all_aligned(x->d, y->d), "aypx", 3));
}

void vec_axpby(lfg_field z, Sc a, lfg_field x, Sc b, lfg_field y) {
  same_kind(z, x, "aX_plus_bY");
  same_kind(z, y, "aX_plus_bY");
  lfg_ctx c = z->ctx;
  DISPATCH_KIND(z->kind, T,
                launch_ew<T>(c, AxpbyOp<T>{(T*)z->d, (const T*)x->d, (const T*)y->d, a, b},
                             z->n(), all_aligned(z->d, x->d, y->d), "axpby", 3));
}

void vec_scale(lfg_field x, Sc a) {
  lfg_ctx c = x->ctx;
  DISPATCH_KIND(x->kind, T,
                launch_ew<T>(c, ScaleOp<T>{(T*)x->d, a}, x->n(), all_aligned(x->d), "scale", 2));
}

void vec_divide(lfg_field z, lfg_field x, lfg_field y) {
  same_kind(z, x, "X_divideby_Y");
  same_kind(z, y, "X_divideby_Y");
  lfg_ctx c = z->ctx;
  DISPATCH_KIND(z->kind, T,
                launch_pdl(c, k_divide<T>, c->stream_grid(z->n()), kThreads, 0, (T*)z->d,
                           (const T*)x->d, (const T*)y->d, z->n()));
  after_launch(c, "divide", (uint64_t)3 * z->n() * z->kind);
}

void vec_dot(lfg_field x, lfg_field y, int slot) {
  same_kind(x, y, "X_innerproduct_Y");
  lfg_ctx c = x->ctx;
  DISPATCH_KIND(x->kind, T,
                launch_ewr<T>(c, DotOp<T>{(const T*)x->d, (const T*)y->d}, x->n(),
                              all_aligned(x->d, y->d), slot, "dot", 2));
}

static void vec_dot_to(lfg_field x, lfg_field y, double* out) {
  same_kind(x, y, "X_innerproduct_Y");
  lfg_ctx c = x->ctx;
  DISPATCH_KIND(x->kind, T,
                launch_ewr<T>(c, DotOp<T>{(const T*)x->d, (const T*)y->d}, x->n(),
                              all_aligned(x->d, y->d), 0, "dot", 2, out));
}

void vec_mgs_step(lfg_field v, lfg_field pv, lfg_field vj, lfg_field pvj, Sc alpha,
                  lfg_field next, int slot) {
  same_kind(v, pv, "mgs");
  same_kind(v, vj, "mgs");
  same_kind(v, pvj, "mgs");
  if (next) same_kind(v, next, "mgs");
  lfg_ctx c = v->ctx;
  const void* nx = next ? next->d : nullptr;
  DISPATCH_KIND(v->kind, T,
                launch_ewr<T>(c, MgsOp<T>{(T*)v->d, (T*)pv->d, (const T*)vj->d,
                                          (const T*)pvj->d, (const T*)nx, alpha},
                              v->n(), all_aligned(v->d, pv->d, vj->d, pvj->d, nx), slot,
                              "mgs", nx ? 7 : 6));
}

void vec_scale2_dot(lfg_field v, lfg_field pv, Sc beta, lfg_field res, int slot) {
  same_kind(v, pv, "scale2_dot");
  same_kind(v, res, "scale2_dot");
  lfg_ctx c = v->ctx;
  DISPATCH_KIND(v->kind, T,
                launch_ewr<T>(c, Scale2DotOp<T>{(T*)v->d, (T*)pv->d, (const T*)res->d, beta},
                              v->n(), all_aligned(v->d, pv->d, res->d), slot, "scale2_dot", 5));
}

void vec_update2_norm(lfg_field dx, lfg_field pv, lfg_field res, lfg_field v, Sc alpha,
                      int slot) {
  same_kind(dx, pv, "update2_norm");
  same_kind(dx, res, "update2_norm");
  same_kind(dx, v, "update2_norm");
  lfg_ctx c = dx->ctx;
  DISPATCH_KIND(dx->kind, T,
                launch_ewr<T>(c, Update2NormOp<T>{(T*)dx->d, (const T*)pv->d, (T*)res->d,
                                                  (const T*)v->d, alpha},
                              dx->n(), all_aligned(dx->d, pv->d, res->d, v->d), slot,
                              "update2_norm", 6));
}

void vec_cg_update(lfg_field x, lfg_field p, lfg_field r, lfg_field q, lfg_field snap, Sc alpha,
                   int slot) {
  same_kind(x, p, "cg_update");
  same_kind(x, r, "cg_update");
  same_kind(x, q, "cg_update");
  if (snap) same_kind(x, snap, "cg_update");
  lfg_ctx c = x->ctx;
  void* sn = snap ? snap->d : nullptr;
  DISPATCH_KIND(x->kind, T,
                launch_ewr<T>(c, CgUpdateOp<T>{(T*)x->d, (const T*)p->d, (T*)r->d,
                                               (const T*)q->d, (T*)sn, alpha},
                              x->n(), all_aligned(x->d, p->d, r->d, q->d, sn), slot,
                              "cg_update", sn ? 7 : 6));
}

void vec_divide_dot(lfg_field z, lfg_field x, lfg_field d, int slot) {
  same_kind(z, x, "divide_dot");
  same_kind(z, d, "divide_dot");
  lfg_ctx c = z->ctx;
  DISPATCH_KIND(z->kind, T,
                launch_ewr<T>(c, DivideDotOp<T>{(T*)z->d, (const T*)x->d, (const T*)d->d},
                              z->n(), all_aligned(z->d, x->d, d->d), slot, "divide_dot", 3));
}

void vec_axpy_norm(lfg_field x, Sc b, lfg_field y, int slot) {
  same_kind(x, y, "axpy_norm");
  lfg_ctx c = x->ctx;
  DISPATCH_KIND(x->kind, T,
                launch_ewr<T>(c, AxpyDotOp<T>{(T*)x->d, (const T*)y->d, nullptr, b}, x->n(),
                              all_aligned(x->d, y->d), slot, "axpy_norm", 3));
}

void vec_axpy_dot(lfg_field x, Sc b, lfg_field y, lfg_field next, int slot) {
  same_kind(x, y, "axpy_dot");
  if (next) same_kind(x, next, "axpy_dot");
  lfg_ctx c = x->ctx;
  const void* nx = next ? next->d : nullptr;
  DISPATCH_KIND(x->kind, T,
                launch_ewr<T>(c, AxpyDotOp<T>{(T*)x->d, (const T*)y->d, (const T*)nx, b},
                              x->n(), all_aligned(x->d, y->d, nx), slot, "axpy_dot", nx ? 4 : 3));
}

void vec_scale_copy(lfg_field dst, Sc a, lfg_field src) {
  same_kind(dst, src, "scale_copy");
  lfg_ctx c = dst->ctx;
  DISPATCH_KIND(dst->kind, T,
                launch_ew<T>(c, ScaleCopyOp<T>{(T*)dst->d, (const T*)src->d, a}, dst->n(),
                             all_aligned(dst->d, src->d), "scale_copy", 2));
}

}  // namespace lfg

namespace lfg {
void ensure_smem_attr(const void* kern, int bytes) {
  int dev = 0;
  LFG_CUDA(cudaGetDevice(&dev));
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> done;
  std::lock_guard<std::mutex> lock(mu);
  int& have = done[std::make_pair(kern, dev)];
  if (have >= bytes) return;
  LFG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  have = bytes;
}

void check_device_error(lfg_ctx c) {
  if (!c->dev_err) return;
  unsigned e = 0;
  LFG_CUDA(cudaMemcpyAsync(&e, c->dev_err, sizeof(e), cudaMemcpyDeviceToHost, c->stream));
  LFG_CUDA(cudaStreamSynchronize(c->stream));
  if (e) {
    LFG_CUDA(cudaMemsetAsync(c->dev_err, 0, sizeof(unsigned), c->stream));
    char buf[96];
    snprintf(buf, sizeof(buf), "a kernel's bounded wait ran out (device error 0x%x)", e);
    throw Error(LFG_ERR_STATE, buf);
  }
}
}  // namespace lfg

// ------------------------------------------------------------ ctx methods
void* lfg_ctx_s::staging(size_t bytes) {
  if (bytes > stage_bytes) {
    dfree(stage);
    stage = nullptr;
    stage_bytes = 0;
    stage = dmalloc(bytes);
    stage_bytes = bytes;
  }
  return stage;
}

void* lfg_ctx_s::scratch(size_t bytes) {
  if (bytes > scratch_bytes) {
    LFG_CUDA(cudaStreamSynchronize(stream));
    dfree(scratch_buf);
    scratch_buf = nullptr;
    scratch_bytes = 0;
    scratch_buf = dmalloc(bytes);
    scratch_bytes = bytes;
    ++scratch_gen;
  }
  return scratch_buf;
}

double lfg_ctx_s::read_result(int slot) {
  LFG_CUDA(cudaMemcpyAsync(host_results + slot, red_results + slot, sizeof(double),
                           cudaMemcpyDeviceToHost, stream));
  LFG_CUDA(cudaStreamSynchronize(stream));
  return host_results[slot];
}

void lfg_ctx_s::read_results(int slot, int n, double* out) {
  LFG_CUDA(cudaMemcpyAsync(host_results + slot, red_results + slot, sizeof(double) * n,
                           cudaMemcpyDeviceToHost, stream));
  LFG_CUDA(cudaStreamSynchronize(stream));
  for (int i = 0; i < n; ++i) out[i] = host_results[slot + i];
}

// ================================================================ C ABI
extern "C" {

const char* lfg_version(void) { return "lfric_core_b200 1.0 (sm_100a)"; }

int lfg_ctx_create(int device, lfg_ctx* out) {
  if (!out) return LFG_ERR_ARG;
  *out = nullptr;
  lfg_ctx c = new (std::nothrow) lfg_ctx_s;
  if (!c) return LFG_ERR_NOMEM;
  int st = guard(c, [&] {
    LFG_CUDA(cudaSetDevice(device));
    c->device = device;
    c->pdl = std::getenv("LFG_NO_PDL") == nullptr;
    LFG_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
    LFG_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    c->red_partials = (double*)dmalloc(sizeof(double) * kRedSlots * kMaxRedBlocks);
    c->red_counters = (unsigned*)dmalloc(sizeof(unsigned) * kRedSlots);
    c->red_results = (double*)dmalloc(sizeof(double) * kRedSlots);
    LFG_CUDA(cudaMemset(c->red_counters, 0, sizeof(unsigned) * kRedSlots));
    LFG_CUDA(cudaMemset(c->red_results, 0, sizeof(double) * kRedSlots));
    LFG_CUDA(cudaMallocHost(&c->host_results, sizeof(double) * kRedSlots));
    c->dev_err = (unsigned*)dmalloc(sizeof(unsigned));
    LFG_CUDA(cudaMemset(c->dev_err, 0, sizeof(unsigned)));
    // lfg_tri_solve_noalloc's set-up on this device, done here while
    // memory can still be had
    LFG_CUDA(noalloc_prepare(device));
  });
  if (st != LFG_OK) {
    fprintf(stderr, "lfg_ctx_create: %s\n", c->last_error.c_str());
    lfg_ctx_destroy(c);
    return st;
  }
  *out = c;
  return LFG_OK;
}

int lfg_ctx_destroy(lfg_ctx c) {
  if (!c) return LFG_OK;
  if (c->own_stream) cudaStreamSynchronize(c->own_stream);
  dfree(c->red_partials);
  dfree(c->red_counters);
  dfree(c->red_results);
  dfree(c->stage);
  dfree(c->scratch_buf);
  dfree(c->dev_err);
  if (c->host_results) cudaFreeHost(c->host_results);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return LFG_OK;
}

int lfg_ctx_set_stream(lfg_ctx c, void* stream) {
  if (!c) return LFG_ERR_ARG;
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return LFG_OK;
}

int lfg_ctx_test_tma_spin_limit(lfg_ctx c, long long spins) {
  if (!c) return LFG_ERR_ARG;
  c->tma_stage_spins = spins < 0 ? -1 : spins;
  return LFG_OK;
}

int lfg_ctx_synchronize(lfg_ctx c) {
  if (!c) return LFG_ERR_ARG;
  return guard(c, [&] {
    LFG_CUDA(cudaStreamSynchronize(c->stream));
    check_device_error(c);
  });
}

int lfg_ctx_kernel_launches(lfg_ctx c, uint64_t* count) {
  if (!c || !count) return LFG_ERR_ARG;
  *count = c->launches;
  return LFG_OK;
}

int lfg_ctx_algorithmic_bytes(lfg_ctx c, uint64_t* bytes) {
  if (!c || !bytes) return LFG_ERR_ARG;
  *bytes = c->bytes;
  return LFG_OK;
}

const char* lfg_last_error(lfg_ctx c) {
  if (!c) return "null context";
  return c->last_error.c_str();
}

// ------------------------------------------------------------ fields
int lfg_field_create(lfg_ctx c, int kind, int ncol, int nlev, lfg_field* out) {
  if (!c || !out) return LFG_ERR_ARG;
  return guard(c, [&] {
    LFG_REQUIRE(kind == LFG_R_DOUBLE || kind == LFG_R_SINGLE, "field_create: bad kind");
    LFG_REQUIRE(ncol > 0 && nlev > 0, "field_create: sizes must be positive");
    lfg_field f = new lfg_field_s;
    f->ctx = c;
    f->kind = kind;
    f->ncol = ncol;
    f->nlev = nlev;
    try {
      f->d = dmalloc(f->bytes());
      f->owned = true;
      LFG_CUDA(cudaMemsetAsync(f->d, 0, f->bytes(), c->stream));
    } catch (...) {
      delete f;
      throw;
    }
    *out = f;
  });
}

int lfg_field_wrap(lfg_ctx c, int kind, int ncol, int nlev, void* dptr, lfg_field* out) {
  if (!c || !out) return LFG_ERR_ARG;
  return guard(c, [&] {
    LFG_REQUIRE(kind == LFG_R_DOUBLE || kind == LFG_R_SINGLE, "field_wrap: bad kind");
    LFG_REQUIRE(ncol > 0 && nlev > 0 && dptr, "field_wrap: bad arguments");
    lfg_field f = new lfg_field_s;
    f->ctx = c;
    f->kind = kind;
    f->ncol = ncol;
    f->nlev = nlev;
    f->d = dptr;
    f->owned = false;
    *out = f;
  });
}

int lfg_field_destroy(lfg_field f) {
  if (!f) return LFG_OK;
  if (f->owned) dfree(f->d);
  delete f;
  return LFG_OK;
}

int lfg_field_device_ptr(lfg_field f, void** p) {
  if (!f || !p) return LFG_ERR_ARG;
  *p = f->d;
  return LFG_OK;
}

}  // extern "C"

namespace {

// buf[k*ncols + i] = field(cols[i], k) for every level k (PACK), or the
// reverse (unpack): the halo columns of a partitioned field moved through
// one contiguous buffer per neighbouring rank.
template <class T, bool PACK>
__global__ void k_columns(T* __restrict__ f, int ncol, int nlev, const int* __restrict__ cols,
                          int ncols, T* __restrict__ buf) {
  const size_t n = (size_t)ncols * nlev;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(t / ncols), i = (int)(t - (size_t)k * ncols);
    const size_t o = (size_t)k * ncol + cols[i];
    if (PACK) buf[t] = f[o];
    else f[o] = buf[t];
  }
}

template <bool PACK>
int columns_op(lfg_field f, const int* cols, int ncols, void* buf) {
  if (!f || (ncols > 0 && (!cols || !buf)) || ncols < 0) return LFG_ERR_ARG;
  lfg_ctx c = f->ctx;
  return guard(c, [&] {
    if (ncols == 0) return;
    const size_t n = (size_t)ncols * f->nlev;
    if (f->kind == LFG_R_DOUBLE)
      k_columns<double, PACK><<<c->stream_grid(n), kThreads, 0, c->stream>>>(
          (double*)f->d, f->ncol, f->nlev, cols, ncols, (double*)buf);
    else
      k_columns<float, PACK><<<c->stream_grid(n), kThreads, 0, c->stream>>>(
          (float*)f->d, f->ncol, f->nlev, cols, ncols, (float*)buf);
    after_launch(c, PACK ? "pack_columns" : "unpack_columns", (uint64_t)2 * f->kind * n);
  });
}

}  // namespace

extern "C" {

int lfg_field_pack_columns(lfg_field f, const int* device_cols, int ncols, void* device_buf) {
  return columns_op<true>(f, device_cols, ncols, device_buf);
}

int lfg_field_unpack_columns(lfg_field f, const int* device_cols, int ncols,
                             const void* device_buf) {
  return columns_op<false>(f, device_cols, ncols, const_cast<void*>(device_buf));
}

int lfg_field_zero_columns(lfg_field f, int first, int count) {
  if (!f || first < 0 || count < 0 || first + count > f->ncol) return LFG_ERR_ARG;
  lfg_ctx c = f->ctx;
  return guard(c, [&] {
    if (count == 0) return;
    LFG_CUDA(cudaMemset2DAsync((char*)f->d + (size_t)first * f->kind, (size_t)f->ncol * f->kind,
                               0, (size_t)count * f->kind, f->nlev, c->stream));
  });
}

int lfg_field_import(lfg_field f, const void* host, int host_kind) {
  if (!f) return LFG_ERR_ARG;
  lfg_ctx c = f->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(host, "field_import: null host array");
    LFG_REQUIRE(host_kind == LFG_R_DOUBLE || host_kind == LFG_R_SINGLE,
                "field_import: bad host kind");
    const size_t bytes = f->n() * host_kind;
    void* st = c->staging(bytes);
    LFG_CUDA(cudaMemcpyAsync(st, host, bytes, cudaMemcpyHostToDevice, c->stream));
    dim3 grid((f->ncol + 31) / 32, (f->nlev + 31) / 32), block(32, 8);
    if (f->kind == LFG_R_DOUBLE && host_kind == LFG_R_DOUBLE)
      k_to_level_major<double, double><<<grid, block, 0, c->stream>>>((double*)f->d, (const double*)st, f->ncol, f->nlev);
    else if (f->kind == LFG_R_DOUBLE)
      k_to_level_major<double, float><<<grid, block, 0, c->stream>>>((double*)f->d, (const float*)st, f->ncol, f->nlev);
    else if (host_kind == LFG_R_DOUBLE)
      k_to_level_major<float, double><<<grid, block, 0, c->stream>>>((float*)f->d, (const double*)st, f->ncol, f->nlev);
    else
      k_to_level_major<float, float><<<grid, block, 0, c->stream>>>((float*)f->d, (const float*)st, f->ncol, f->nlev);
    after_launch(c, "to_level_major", (uint64_t)bytes + f->bytes());
    LFG_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int lfg_field_export(lfg_field f, void* host, int host_kind) {
  if (!f) return LFG_ERR_ARG;
  lfg_ctx c = f->ctx;
  return guard(c, [&] {
    LFG_REQUIRE(host, "field_export: null host array");
    LFG_REQUIRE(host_kind == LFG_R_DOUBLE || host_kind == LFG_R_SINGLE,
                "field_export: bad host kind");
    const size_t bytes = f->n() * host_kind;
    void* st = c->staging(bytes);
    dim3 grid((f->ncol + 31) / 32, (f->nlev + 31) / 32), block(32, 8);
    if (f->kind == LFG_R_DOUBLE && host_kind == LFG_R_DOUBLE)
      k_to_column<double, double><<<grid, block, 0, c->stream>>>((double*)st, (const double*)f->d, f->ncol, f->nlev);
    else if (f->kind == LFG_R_DOUBLE)
      k_to_column<float, double><<<grid, block, 0, c->stream>>>((float*)st, (const double*)f->d, f->ncol, f->nlev);
    else if (host_kind == LFG_R_DOUBLE)
      k_to_column<double, float><<<grid, block, 0, c->stream>>>((double*)st, (const float*)f->d, f->ncol, f->nlev);
    else
      k_to_column<float, float><<<grid, block, 0, c->stream>>>((float*)st, (const float*)f->d, f->ncol, f->nlev);
    after_launch(c, "to_column", (uint64_t)bytes + f->bytes());
    LFG_CUDA(cudaMemcpyAsync(host, st, bytes, cudaMemcpyDeviceToHost, c->stream));
    LFG_CUDA(cudaStreamSynchronize(c->stream));
  });
}

// ------------------------------------------------------------ built-ins
#define FIELD_CTX(f) ((f) ? (f)->ctx : nullptr)

int lfg_setval_c(lfg_field x, double v) {
  if (!x) return LFG_ERR_ARG;
  return guard(x->ctx, [&] { vec_set(x, sc_const(v)); });
}
int lfg_setval_X(lfg_field dst, lfg_field src) {
  if (!dst || !src) return LFG_ERR_ARG;
  return guard(dst->ctx, [&] { vec_copy(dst, src); });
}
int lfg_inc_X_plus_bY(lfg_field x, double b, lfg_field y) {
  if (!x || !y) return LFG_ERR_ARG;
  return guard(x->ctx, [&] { vec_axpy(x, sc_const(b), y); });
}
int lfg_inc_aX_plus_Y(double a, lfg_field x, lfg_field y) {
  if (!x || !y) return LFG_ERR_ARG;
  return guard(x->ctx, [&] { vec_aypx(x, sc_const(a), y); });
}
int lfg_aX_plus_bY(lfg_field z, double a, lfg_field x, double b, lfg_field y) {
  if (!z || !x || !y) return LFG_ERR_ARG;
  return guard(z->ctx, [&] { vec_axpby(z, sc_const(a), x, sc_const(b), y); });
}
int lfg_inc_a_times_X(double a, lfg_field x) {
  if (!x) return LFG_ERR_ARG;
  return guard(x->ctx, [&] { vec_scale(x, sc_const(a)); });
}
int lfg_X_divideby_Y(lfg_field z, lfg_field x, lfg_field y) {
  if (!z || !x || !y) return LFG_ERR_ARG;
  return guard(z->ctx, [&] { vec_divide(z, x, y); });
}
int lfg_X_innerproduct_Y(lfg_field x, lfg_field y, double* result) {
  if (!x || !y || !result) return LFG_ERR_ARG;
  return guard(x->ctx, [&] {
    vec_dot(x, y, 0);
    *result = x->ctx->read_result(0);
  });
}
int lfg_X_innerproduct_X(lfg_field x, double* result) {
  return lfg_X_innerproduct_Y(x, x, result);
}
int lfg_X_innerproduct_Y_device(lfg_field x, lfg_field y, void* device_result) {
  if (!x || !y || !device_result) return LFG_ERR_ARG;
  return guard(x->ctx, [&] {
    LFG_REQUIRE(x->n() == y->n(), "X_innerproduct_Y: fields differ in size");
    vec_dot_to(x, y, (double*)device_result);
  });
}

}  // extern "C"

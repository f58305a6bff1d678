// Internal definitions of the B200 LFRic solver library.
//
// Device layout: a field of ncol horizontal entities with nlev dofs each is
// stored level-major, element (k, c) at k*ncol + c, so that a warp of
// threads handling consecutive columns reads consecutive addresses at every
// level.  Operators use the same layout for their coefficient arrays.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <unordered_map>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/lfg.h"

namespace lfg {

// Blocks per SM used for streaming grids (grid = SMs * this, grid-stride).
constexpr int kStreamBlocksPerSM = 8;
constexpr int kThreads = 256;
// Reduction slots available per context and the partial buffer per slot.
constexpr int kRedSlots = 512;
constexpr int kMaxRedBlocks = 4096;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define LFG_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      throw ::lfg::Error(LFG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define LFG_REQUIRE(cond, msg)                                             \
  do {                                                                     \
    if (!(cond)) throw ::lfg::Error(LFG_ERR_ARG, std::string(msg));        \
  } while (0)

// A scalar operand evaluated on the device: lets Krylov scalars stay in
// device memory (no host round trip) while keeping the reference's order of
// operations.  value = c, c*a, c*a/b or c/sqrt(a).
enum ScOp : int { SC_CONST = 0, SC_MUL = 1, SC_DIV = 2, SC_RSQRT = 3 };
struct Sc {
  int op;
  double c;
  const double* a;
  const double* b;
};
inline Sc sc_const(double c) { return Sc{SC_CONST, c, nullptr, nullptr}; }
inline Sc sc_mul(double c, const double* a) { return Sc{SC_MUL, c, a, nullptr}; }
inline Sc sc_div(double c, const double* a, const double* b) { return Sc{SC_DIV, c, a, b}; }
inline Sc sc_rsqrt(double c, const double* a) { return Sc{SC_RSQRT, c, a, nullptr}; }

__device__ __forceinline__ double sc_eval(const Sc& s) {
  switch (s.op) {
    case SC_MUL: return s.c * *s.a;
    case SC_DIV: return s.c * *s.a / *s.b;
    case SC_RSQRT: return s.c / sqrt(*s.a);
    default: return s.c;
  }
}

// One deterministic reduction: per-block partial sums, then the last block
// to finish adds the partials in index order and writes the result.
struct Red {
  double* partials;   // [kMaxRedBlocks]
  unsigned* counter;  // zero between reductions
  double* result;
};

// ------------------------------------------------------------ reductions
// Deterministic block sum (fixed shuffle tree) and the last-block finish.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block; the result is valid in thread 0.  Fixed tree.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double s[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  v = warp_sum(v);
  if (lane == 0) s[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < (int)(blockDim.x >> 5) ? s[lane] : 0.0;
    v = warp_sum(v);
  }
  return v;
}

__device__ __forceinline__ void red_finish(const Red& r, double v) {
  __shared__ bool is_last;
  v = block_sum(v);
  if (threadIdx.x == 0) {
    r.partials[blockIdx.x] = v;
    __threadfence();
    unsigned t = atomicAdd(r.counter, 1u);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (is_last) {
    __threadfence();
    double acc = 0.0;
    const volatile double* p = r.partials;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) acc += p[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) {
      *r.result = acc;
      *r.counter = 0u;
    }
  }
}

}  // namespace lfg

// ------------------------------------------------------------------ objects
struct lfg_ctx_s {
  int device = 0;
  int num_sms = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::string last_error;
  uint64_t launches = 0;
  // algorithmic bytes of the launched kernels: each array a kernel reads
  // counted once, each array it writes counted once, at stored precision
  uint64_t bytes = 0;
  // reduction slots
  double* red_partials = nullptr;  // [kRedSlots][kMaxRedBlocks]
  unsigned* red_counters = nullptr;
  double* red_results = nullptr;   // [kRedSlots]
  double* host_results = nullptr;  // pinned [kRedSlots]
  // host<->device staging for import/export
  void* stage = nullptr;
  size_t stage_bytes = 0;
  // device scratch of the kernels that need one (grown on demand)
  void* scratch_buf = nullptr;
  size_t scratch_bytes = 0;
  // counts reallocations of scratch_buf: a captured CUDA graph whose kernels
  // use the scratch buffer is replayed only under the generation it was
  // captured in
  uint64_t scratch_gen = 0;
  // device error word: kernels whose bounded waits ran out record a code
  // here (0 = none); read by check_device_error
  unsigned* dev_err = nullptr;
  // polls of a TMA stage wait before the substitution kernels give up
  // (< 0: their built-in limit); lfg_ctx_test_tma_spin_limit sets it
  long long tma_stage_spins = -1;
  // launch the multigrid and Helmholtz kernels with programmatic dependent
  // launch (off when LFG_NO_PDL is set in the environment: a debugging aid)
  bool pdl = true;

  lfg::Red red(int slot) {
    return lfg::Red{red_partials + (size_t)slot * lfg::kMaxRedBlocks, red_counters + slot,
                    red_results + slot};
  }
  int stream_grid(size_t n, int threads = lfg::kThreads) const {
    size_t need = (n + threads - 1) / threads;
    size_t cap = (size_t)num_sms * lfg::kStreamBlocksPerSM;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
  }
  void* staging(size_t bytes);
  void* scratch(size_t bytes);
  double read_result(int slot);   // synchronises the stream
  // n consecutive slots' results into out[] (one copy; synchronises)
  void read_results(int slot, int n, double* out);
};

struct lfg_field_s {
  lfg_ctx ctx = nullptr;
  int kind = LFG_R_DOUBLE;
  int ncol = 0, nlev = 0;
  void* d = nullptr;
  bool owned = false;
  size_t n() const { return (size_t)ncol * nlev; }
  size_t bytes() const { return n() * kind; }
};

struct lfg_mesh_s {
  lfg_ctx ctx = nullptr;
  int ncol = 0;
  int* links = nullptr;  // device, SoA [4][ncol]
  std::vector<int> h_links;  // host copy, [ncol][4]
  // For each side f of column c, the side whose coupling stands for its face:
  // hsrc[f][c] = g << 29 | d reads side g of column d.  Of a face's two sides
  // the one with the larger side index (N > E > S > W; then the smaller
  // column) is read for both, so inside a panel a column reads its own E and
  // N couplings and its W and S neighbours' E and N ones.  Null when the
  // links do not pair up.
  int* hsrc = nullptr;  // device [4][ncol]
  // Structured cubed-sphere numbering, detected at creation (pn = 0: none):
  // 6 panels of pn x pn cells, numbered row-major inside each panel, and
  // every cell off a panel's border has its side-f neighbour at
  // c + base[(f + roll_p) & 3], base = {-1, +pn, +1, -pn},
  // roll_p = (proll >> 2p) & 3.  pcf: the interior cells' hsrc codes follow
  // from it (a side f >= 2 is its own face's designated side, a side f < 2
  // reads its neighbour's side f + 2).
  int pn = 0;
  unsigned proll = 0;
  bool pcf = false;
  // First columns of the kPanelMargin-wide border groups of the
  // element-parallel panel kernels (every group of rows 0 and pn-1, the
  // first and last group of every other row); built when
  // pn % kPanelMargin == 0 and pn >= 3 kPanelMargin, else null.
  int* pedge = nullptr;  // device
  int npedge = 0;
};

struct lfg_intergrid_s {
  lfg_ctx ctx = nullptr;
  int ncoarse = 0, nfine = 0, nx = 0, ny = 0;
  int* child = nullptr;    // device [nx*ny][ncoarse], slot q = y*nx + x
  int* parent = nullptr;   // device [nfine]
  int* ccorner = nullptr;  // device [4][ncoarse] W0 coarse corner vertices (or null)
  int* w0_inj = nullptr;   // device [nvert_coarse] coinciding fine vertex
  int* w0_src = nullptr;   // device [nvert_fine] coarse cell of the last write (-1: none)
  double* w0_w = nullptr;  // device [nvert_fine][5] weights NE,SE,SW,NW and term count
  int nvert_coarse = 0, nvert_fine = 0;
  std::vector<int> h_child;  // [ncoarse][ny][nx]
  // 2x2 maps between structured meshes (pnc = coarse panel side, 0: none):
  // child slot q of coarse cell (panel P, column I, row J) is the fine cell
  // P nf^2 + (2J + dy) nf + 2I + dx, nf = 2 pnc, with
  // 2 dy + dx = (qpos >> (8P + 2q)) & 3.  cedge: the coarse cells on a
  // panel's border (I or J in {0, pnc-1}).
  int pnc = 0;
  unsigned long long qpos = 0;
  int* cedge = nullptr;  // device
  int ncedge = 0;
};

// W2 intergrid maps (lfg_w2.cu)
struct lfg_w2map_s {
  lfg_ctx ctx = nullptr;
  lfg_intergrid ig = nullptr;
  int nl = 0, ndf = 0, undf_c = 0, undf_f = 0;
  int nent_c = 0, nent_f = 0;  // level-major columns (0: flat fields)
  bool has_sel = false;
  int* mapc = nullptr;
  int* mapf = nullptr;
  int* sel_ew = nullptr;
  int* sel_ns = nullptr;
};

struct lfg_cma_s {
  lfg_ctx ctx = nullptr;
  int kind = LFG_R_DOUBLE;
  int ncol = 0, nrow = 0, ncolumn = 0, bw = 0, alpha = 0, beta = 0, gm = 0, gp = 0;
  void* bands = nullptr;      // [bw][nrow][ncol]
  int* ind_to = nullptr;      // device, 0-based column offsets [nrow]
  int* ind_from = nullptr;    // [ncolumn]
  int* jminus = nullptr;      // [nrow] first band column of each row (0-based)
  int* jplus = nullptr;       // [nrow] last band column of each row
  int max_ind_to = 0, max_ind_from = 0;  // largest 1-based column offsets
  bool ind_identity = false;       // ind_to(i) = i for every row (W3 -> W3 style maps)
  bool ind_from_identity = false;  // ind_from(j) = j for every column
  int* tptr = nullptr;        // [ncolumn+1] rows reaching each column (transpose)
  int* trow = nullptr;
  // Thomas factors of a square tridiagonal operator (columnwise_op_appinv's
  // inverse denominators and c'), [nrow][ncol]; computed on the first
  // lfg_cma_apply_inverse after the bands change
  void* finv = nullptr;
  void* fcp = nullptr;
  bool fvalid = false;
  // The row lists of the last assembly (lfg_cma_assemble: per row, the
  // element-matrix planes and bands it sums), kept with the dofmaps they
  // came from: re-assembling with new element matrices and the same
  // dofmaps, as every timestep does, reuses them and stays asynchronous.
  std::vector<int> asm_key;
  int* asm_rowptr = nullptr;  // device [nrow+1]
  int* asm_list = nullptr;    // device int2 [rowptr[nrow]]
  int asm_maxq = 0;           // most contributions of one row
  // shapes of the last product C = C + A B into this operator, and the
  // widest spans of A's and C's rows
  std::vector<int> mul_key;
  int mul_span_a = 0, mul_span_c = 0;
};

struct lfg_lma_s {
  lfg_ctx ctx = nullptr;
  int kind = LFG_R_DOUBLE;
  int ncell = 0, nl = 0, ndf_to = 0, ndf_from = 0;
  int nent_to = 0, nlev_to = 0, nent_from = 0, nlev_from = 0;
  void* a = nullptr;        // [ndf_to][ndf_from][nl][ncell]
  int* ent_to = nullptr;    // [ndf_to][ncell] entity of each cell dof
  int* off_to = nullptr;    // [ndf_to][ncell] level offset
  int* ent_from = nullptr;  // [ndf_from][ncell]
  int* off_from = nullptr;
  // gather lists: for each output entity its (cell, df) incidences
  int* inc_to_ptr = nullptr;   // [nent_to+1]
  int* inc_to = nullptr;       // packed cell*ndf_to + df
  int* inc_from_ptr = nullptr;
  int* inc_from = nullptr;
  int max_inc_to = 0, max_inc_from = 0;
  // the same lists padded to a fixed width, [slot][entity], each slot the
  // pair (loc offset of layer 0, level offset); empty slots never match a
  // level.  tab_to keeps the forward order, tab_from the transposed one.
  int2* tab_to = nullptr;
  int2* tab_from = nullptr;
  int tab_to_w = 0, tab_from_w = 0;  // 0: no padded table (wider lists)
};

struct lfg_helm_s {
  lfg_ctx ctx = nullptr;
  lfg_mesh mesh = nullptr;
  int kind = LFG_R_DOUBLE;
  int ncol = 0, nl = 0;
  void* sub = nullptr;   // [nl][ncol]
  void* diag = nullptr;
  void* sup = nullptr;
  void* h = nullptr;     // [4][nl][ncol]
  // every face's two sides carry the same coupling bit for bit, so the
  // kernels read each face through mesh->hsrc (half the coupling traffic)
  bool hsym = false;
  // Thomas factors of T' (columnwise_op_appinv's inverse denominators and
  // c'), functions of the matrix alone: computed once per operator
  void* inv = nullptr;   // [nl][ncol]
  void* cp = nullptr;    // [nl][ncol]
};

namespace lfg {

// Launch bookkeeping and error checks shared by all translation units.
inline void after_launch(lfg_ctx ctx, const char* what, uint64_t bytes = 0) {
  ctx->launches++;
  ctx->bytes += bytes;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    throw Error(LFG_ERR_CUDA, std::string("launch of ") + what + ": " + cudaGetErrorString(e));
}

void* dmalloc(size_t bytes);
// Raises kern's dynamic shared-memory limit to `bytes` on the current
// device; once per (kernel, device), thread-safe (the attribute belongs to
// the kernel's module in each device's context).
void ensure_smem_attr(const void* kern, int bytes);
void dfree(void* p);
void upload(void* d, const void* h, size_t bytes);

// entry-point wrapper: converts exceptions into status codes
template <class F>
int guard(lfg_ctx ctx, F&& f) {
  // the context's device is current for the call, the caller's afterwards
  struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(lfg_ctx c) {
      int cur = 0;
      if (c && cudaGetDevice(&cur) == cudaSuccess && cur != c->device &&
          cudaSetDevice(c->device) == cudaSuccess)
        prev = cur;
    }
    ~DeviceScope() {
      if (prev >= 0) cudaSetDevice(prev);
    }
  } scope(ctx);
  try {
    f();
    return LFG_OK;
  } catch (const Error& e) {
    if (ctx) ctx->last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    if (ctx) ctx->last_error = "host allocation failed";
    return LFG_ERR_NOMEM;
  } catch (const std::exception& e) {
    if (ctx) ctx->last_error = e.what();
    return LFG_ERR_ARG;
  }
}

// Grid for a grid-stride kernel: enough blocks for `work` threads, capped
// at one full wave (the blocks of `kern` that fit on every SM at once, from
// the occupancy calculator; cached per kernel).  A cap above one wave would
// leave a partial second wave whose blocks each walk the grid-stride loop
// on their own.
inline int occ_grid(lfg_ctx c, const void* kern, int threads, size_t work, size_t smem = 0) {
  static std::mutex mu;
  static std::unordered_map<const void*, int> per_sm;
  int nb;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = per_sm.find(kern);
    if (it == per_sm.end()) {
      int v = 0;
      LFG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kern, threads, smem));
      it = per_sm.emplace(kern, v > 0 ? v : 1).first;
    }
    nb = it->second;
  }
  const size_t need = (work + threads - 1) / threads;
  const size_t cap = (size_t)c->num_sms * nb;
  return (int)std::max<size_t>(1, std::min(need, cap));
}

// ------------------------------------------------------- vector accesses
// V consecutive values of a V*sizeof(T)-aligned address moved by one load
// or store instruction (8 or 16 bytes).
template <class T, int V>
struct Vec {
  T e[V];
};

// V consecutive values from a V*sizeof(T)-aligned address (8 or 16 bytes:
// one load); STREAM: evict-first, for arrays read once.  FP32 vectors
// ignore STREAM: the FP32 panel kernels measured faster with plain loads
// (C192x70: sweep right-hand side 76 against 83 us, apply 104 against 107
// us, residual + restriction 114 against 127 us).
template <bool STREAM, class T, int V>
__device__ __forceinline__ Vec<T, V> vld(const T* p) {
  Vec<T, V> r;
  if constexpr (std::is_same_v<T, float> && V == 4) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    r.e[0] = q.x; r.e[1] = q.y; r.e[2] = q.z; r.e[3] = q.w;
  } else if constexpr (std::is_same_v<T, float> && V == 2) {
    const float2 q = *reinterpret_cast<const float2*>(p);
    r.e[0] = q.x; r.e[1] = q.y;
  } else if constexpr (std::is_same_v<T, double> && V == 2) {
    const double2 q = STREAM ? __ldcs(reinterpret_cast<const double2*>(p))
                             : *reinterpret_cast<const double2*>(p);
    r.e[0] = q.x; r.e[1] = q.y;
  } else if constexpr (std::is_same_v<T, int> && V == 4) {
    const int4 q = *reinterpret_cast<const int4*>(p);
    r.e[0] = q.x; r.e[1] = q.y; r.e[2] = q.z; r.e[3] = q.w;
  } else if constexpr (std::is_same_v<T, int> && V == 2) {
    const int2 q = *reinterpret_cast<const int2*>(p);
    r.e[0] = q.x; r.e[1] = q.y;
  } else {
    static_assert(V == 1, "vld: unsupported width");
    r.e[0] = STREAM ? __ldcs(p) : *p;
  }
  return r;
}

template <class T, int V>
__device__ __forceinline__ void vst(T* p, const Vec<T, V>& v) {
  if constexpr (std::is_same_v<T, float> && V == 4)
    *reinterpret_cast<float4*>(p) = make_float4(v.e[0], v.e[1], v.e[2], v.e[3]);
  else if constexpr (std::is_same_v<T, float> && V == 2)
    *reinterpret_cast<float2*>(p) = make_float2(v.e[0], v.e[1]);
  else if constexpr (std::is_same_v<T, double> && V == 2)
    *reinterpret_cast<double2*>(p) = make_double2(v.e[0], v.e[1]);
  else
    p[0] = v.e[0];
}

// ------------------------------------------- programmatic dependent launch
// A kernel launched by launch_pdl may begin launching as soon as every block
// of the kernel before it in the stream has exited, before that kernel's
// completion has been signalled; it must call grid_dep_wait() before its
// first access to global memory, which returns once the earlier kernel has
// finished and its writes are visible.  Only kernels that call
// grid_dep_wait() at their top are launched this way.  (No kernel here
// signals its dependents early: letting a kernel's successor launch while
// the kernel itself still waited on its own predecessor filled the SMs with
// waiting blocks and halved the solve rate.)
__device__ __forceinline__ void grid_dep_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <class... KArgs, class... Args>
void launch_pdl(lfg_ctx c, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = c->pdl ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  LFG_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
}

// Columns at each end of a panel row that the element-parallel panel
// kernels leave to their per-column edge path (a multiple of every vector
// width they use).
constexpr int kPanelMargin = 4;

// Throws LFG_ERR_STATE when a kernel recorded a device error (synchronises).
void check_device_error(lfg_ctx c);

// Looks up lfg_tri_solve_noalloc's device array on device `dev` (current)
// and loads its kernels there (lfg_cma.cu); called by lfg_ctx_create.
cudaError_t noalloc_prepare(int dev);

// TMA-staged column substitution (lfg_subst_tma.cu), fine meshes; FP64
// for columns of at most 80 levels.
bool subst_tma_applicable(lfg_ctx c, int ncol, int nl, const void* const* ptrs, int nptr,
                          int elem_bytes);
void subst_tma(lfg_ctx c, int ncol, int nl, const float* r, const float* sub, const float* inv,
               const float* cp, const float* xin, float omega, float* xout);
void subst_tma(lfg_ctx c, int ncol, int nl, const double* r, const double* sub,
               const double* inv, const double* cp, const double* xin, double omega,
               double* xout);

// vector algebra launchers (lfg_core.cu)
void vec_set(lfg_field x, Sc a);
void vec_copy(lfg_field dst, lfg_field src);
void vec_axpy(lfg_field x, Sc b, lfg_field y);                 // x = x + b y
void vec_aypx(lfg_field x, Sc a, lfg_field y);                 // x = a x + y
void vec_axpby(lfg_field z, Sc a, lfg_field x, Sc b, lfg_field y);
void vec_scale(lfg_field x, Sc a);
void vec_divide(lfg_field z, lfg_field x, lfg_field y);
void vec_dot(lfg_field x, lfg_field y, int slot);               // result in slot
// fused Krylov steps
void vec_mgs_step(lfg_field v, lfg_field pv, lfg_field vj, lfg_field pvj, Sc alpha,
                  lfg_field next, int slot);  // v -= a vj; pv -= a pvj; slot = <v, next or v>
void vec_scale2_dot(lfg_field v, lfg_field pv, Sc beta, lfg_field res, int slot);
void vec_update2_norm(lfg_field dx, lfg_field pv, lfg_field res, lfg_field v, Sc alpha,
                      int slot);             // dx += a pv; res -= a v; slot = <res,res>
// x += a p; r -= a q; slot = <r, r>; snap = x (snap may be null)
void vec_cg_update(lfg_field x, lfg_field p, lfg_field r, lfg_field q, lfg_field snap, Sc alpha,
                   int slot);
void vec_divide_dot(lfg_field z, lfg_field x, lfg_field d, int slot);  // z = x / d; slot = <x, z>
void vec_axpy_norm(lfg_field x, Sc b, lfg_field y, int slot);   // x += b y; slot = <x,x>
// x += b y; slot = <x, next> (next null: <x, x>)
void vec_axpy_dot(lfg_field x, Sc b, lfg_field y, lfg_field next, int slot);
void vec_scale_copy(lfg_field dst, Sc a, lfg_field src);        // dst = a src

// Helmholtz launchers (lfg_helm.cu)
void helm_apply(lfg_helm op, lfg_field y, lfg_field x, lfg_field dot_with, int slot);
void helm_residual(lfg_helm op, lfg_field r, lfg_field x, lfg_field b, int norm_slot);
// r = b - A x formed in FP64 by an r_double operator and stored in the
// r_single field r; norm_slot = <b - A x, b - A x> in FP64
void helm_residual_lower(lfg_helm op, lfg_field r, lfg_field x, lfg_field b, int norm_slot);
// x_out = sweep(x_in); x_in null: zero guess.  rbuf: workspace of ncol*nl
// values of the operator's kind for the right-hand side (null: the
// context's scratch).
void helm_smooth(lfg_helm op, double omega, lfg_field x_in, lfg_field b, lfg_field x_out,
                 void* rbuf);
void helm_residual_restrict(lfg_helm op, lfg_intergrid ig, lfg_field x, lfg_field b,
                            lfg_field bc);
void prolong_add(lfg_intergrid ig, lfg_field fine, lfg_field coarse);

}  // namespace lfg

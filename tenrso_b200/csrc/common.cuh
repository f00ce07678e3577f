// Shared definitions for the tenrso_b200 CUDA library: the context object,
// error reporting in tenrso's wording, device workspace slots and small
// device helpers. All kernels target sm_100a only.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <list>
#include <string>
#include <utility>
#include <vector>

#include "../../include/tenrso_b200.h"

namespace tsr {

// ---------------------------------------------------------------------------
// error handling
// ---------------------------------------------------------------------------
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

#define TSR_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e__ = (call);                                                            \
    if (e__ != cudaSuccess)                                                              \
      return ::tsr::fail(TSR_E_CUDA, "CUDA error %s at %s:%d: %s", cudaGetErrorName(e__), \
                         __FILE__, __LINE__, cudaGetErrorString(e__));                   \
  } while (0)

#define TSR_TRY(expr)        \
  do {                       \
    int rc__ = (expr);       \
    if (rc__ != TSR_OK) return rc__; \
  } while (0)

// Device-side status word bits (written by kernels, read by the host after a
// synchronize; no kernel raises an error any other way).
enum DevStatus : unsigned {
  DS_OK = 0,
  DS_NOT_SPD = 1u << 0,      // Gram not positive definite even after the ridge
  DS_RIDGE_USED = 1u << 1,   // ridge fallback engaged (informational)
  DS_TIMEOUT = 1u << 2,      // a bounded wait gave up
  DS_BAD_INDEX = 1u << 3,    // an input index was out of range
};

// ---------------------------------------------------------------------------
// context and workspace
// ---------------------------------------------------------------------------
struct Buffer {
  void* ptr = nullptr;
  size_t bytes = 0;
};

enum Slot {
  SLOT_UNFOLD0 = 0,   // per-mode unfolded copies (fp32 or bf16 hi)
  SLOT_UNFOLD_LO = 8,  // per-mode bf16 lo copies
  SLOT_FACTORS = 16,  // factor matrices (fp32)
  SLOT_PARTIALS,      // split-K partial MTTKRP results
  SLOT_GRAMS,         // FP64 Grams / Hadamards / inverses
  SLOT_STATE,         // ALS state (fit history, flags)
  SLOT_TENSOR,        // staged input tensor
  SLOT_OUT,           // staged output
  SLOT_MISC0,
  SLOT_MISC1,
  SLOT_MISC2,
  SLOT_MISC3,
  SLOT_D3_HI,         // 3-way single-layout path: bf16 hi half of X
  SLOT_D3_LO,         //   bf16 lo half of X
  SLOT_D3_IMG,        //   B images of the contracted factors
  SLOT_SPARSE0,
  SLOT_SPARSE1 = SLOT_SPARSE0 + 16,
  SLOT_COUNT = SLOT_SPARSE1 + 16
};

}  // namespace tsr

namespace tsr {
// Kernel timeline tracing of the CP-ALS sweep (off unless enabled on the
// context): each traced launch owns one slot; every CTA's thread 0 folds the
// %globaltimer value at entry into start (min) and at exit into end (max).
struct TraceSlot {
  unsigned long long* start;
  unsigned long long* end;
};
__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void trace_begin(const TraceSlot& tr) {
  if (tr.start && threadIdx.x == 0) atomicMin(tr.start, globaltimer_ns());
}
__device__ __forceinline__ void trace_end(const TraceSlot& tr) {
  if (tr.end && threadIdx.x == 0) atomicMax(tr.end, globaltimer_ns());
}
enum TraceKind { TRACE_MTTKRP = 0, TRACE_INVERSE = 1, TRACE_SOLVE = 2 };
}  // namespace tsr

struct tsr_ctx {
  int device = 0;
  int sm_count = 148;
  size_t l2_bytes = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  tsr::Buffer slots[tsr::SLOT_COUNT];
  void* pinned = nullptr;  // pinned host staging (grow-only)
  size_t pinned_bytes = 0;
  void* readback = nullptr;  // pinned host buffer for a call's closing read-back (grow-only)
  size_t readback_bytes = 0;
  unsigned* d_status = nullptr;  // device status word
  int64_t launches = 0;          // kernels launched by this context (counter)
  // clock-cycle budget of each bounded pipeline wait in the tensor-core
  // MTTKRP (about 1 s by default; tsr_ctx_set_wait_budget lowers it to test
  // the timeout path)
  long long wait_budget = 1ll << 31;
  // kernel timeline tracing (tsr_ctx_set_trace): device start/end arrays,
  // the next free slot and, per slot, the kernel kind and mode
  unsigned long long* trace_start = nullptr;
  unsigned long long* trace_end = nullptr;
  int trace_cap = 0;
  int trace_next = 0;
  std::vector<std::pair<int, int>> trace_meta;
  // SMs the MTTKRP grids leave free so that the side-stream FP64 kernels of
  // the ALS sweep (Gram, inverse, fit) run concurrently instead of queueing
  int reserve_sms = 8;
  // second stream + events for the overlapped ALS sweep
  cudaStream_t aux = nullptr;
  cudaEvent_t ev[24] = {};
  // cached instantiated sweep graph and the arguments it was captured with
  // Instantiated CP-ALS sweep graphs, keyed by the sweep's arguments and the
  // number of sweeps captured; least recently used evicted beyond kMaxGraphs.
  struct SweepGraph {
    std::vector<uint8_t> key;
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;  // kernels per graph launch
    uint64_t last_use = 0;
  };
  static constexpr int kMaxGraphs = 8;
  std::list<SweepGraph> sweep_graphs;  // stable element addresses
  uint64_t graph_clock = 0;
};

namespace tsr {

// Grow-only device buffer for a slot; contents are not preserved on growth.
int slot_get(tsr_ctx* ctx, int slot, size_t bytes, void** out);
int pinned_get(tsr_ctx* ctx, size_t bytes, void** out);
// Pinned host buffer for small device-to-host read-backs (grow-only; growing
// synchronizes the stream first).
int readback_get(tsr_ctx* ctx, size_t bytes, void** out);
int check_ctx(tsr_ctx* ctx);
int read_status(tsr_ctx* ctx, unsigned* out);  // synchronizes the stream
// Evict L2 by reading a buffer of twice its size (clean lines only).
int flush_l2(tsr_ctx* ctx, cudaStream_t s);
int reset_status(tsr_ctx* ctx);
// The next trace slot for a launch of `kind` on `mode` ({nullptr, nullptr}
// when tracing is off or the buffer is full).
TraceSlot trace_slot(tsr_ctx* ctx, int kind, int mode);
// Synchronizes, reads and clears the status word: TSR_E_TIMEOUT when a
// kernel's bounded wait gave up, else TSR_OK.
int check_device_status(tsr_ctx* ctx);

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

// Programmatic dependent launch. A kernel launched with launch_pdl may start
// while the previous kernel of its stream is still running, once every CTA of
// that kernel has called grid_dep_trigger() or exited; it must call
// grid_dep_wait() before it reads anything the previous kernel writes or
// writes anything that kernel reads (the wait returns once the previous grid
// has completed and its memory is visible; without a programmatic
// predecessor it returns at once). Only work on data produced before the
// previous kernel may precede the wait.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Shape bookkeeping for a dense N-way tensor and one of its unfoldings.
constexpr int kMaxModes = 8;
struct Unfolding {
  int ndim;
  int mode;
  int64_t rows;     // I_mode
  int64_t cols;     // prod of the other sizes
  int64_t ld;       // padded row stride (elements), multiple of 8
  int n_other;      // ndim - 1
  int64_t other_size[kMaxModes];  // sizes of the other modes, ascending mode order
  int other_mode[kMaxModes];
};
Unfolding make_unfolding(int ndim, const int64_t* shape, int mode);

// Launch the (fp32) unfold of a row-major dense tensor into X_(mode) with row
// stride u.ld. Pads columns [cols, ld) with zeros.
int launch_unfold_f32(tsr_ctx* ctx, const float* X, const int64_t* shape, const Unfolding& u,
                      float* out);
int launch_unfold_bf16x2(tsr_ctx* ctx, const float* X, const int64_t* shape, const Unfolding& u,
                         __nv_bfloat16* hi, __nv_bfloat16* lo);
// Every unfolding of a 3-way tensor in one pass (bf16 hi/lo for all modes, or
// fp32 for modes 1 and 2), adding ||X||^2 into *norm_sq. Needs J, K multiples
// of 8 (unpadded rows) and I <= 65535.
bool unfold3_supported(int ndim, const int64_t* shape);
int launch_unfold3(tsr_ctx* ctx, const float* X, const int64_t* shape, bool bf16,
                   void* const* hi, void* const* lo, double* norm_sq);

// Raise the dynamic shared-memory limits of every kernel once per process
// (before any stream capture).
void init_kernel_attributes();

// Factor pointer table passed by value to kernels.
struct FactorTable {
  const float* ptr[kMaxModes];
  int64_t rows[kMaxModes];
};

}  // namespace tsr

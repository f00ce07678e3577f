// An allocation-free dense MTTKRP entry point.
//
// Some callers cannot call cudaMalloc. A library embedded in a framework
// whose caching allocator owns the GPU's memory must not allocate behind that
// allocator's back (a raw cudaMalloc fragments its pool, fails once the pool
// has reserved the device, or is forbidden by the host application outright),
// and a service that sizes every device buffer up front cannot tolerate a
// call that may allocate on first use. For them this entry point runs the
// FP32 split-K MTTKRP of mode 0 with its split partials in a fixed,
// file-scope device array instead of a context workspace: it makes no
// cudaMalloc / cudaFree call and needs no tsr_ctx (the caller passes a
// stream, the inputs and the output).
//
// The array below is part of the library image: every GPU that loads the
// library holds its 16 MiB until the process exits. All calls share it and
// it keeps the last call's contents; calls that overlap on the GPU (for
// example on two streams) race on it, so callers must serialise them.
#include <mutex>

#include "kr.cuh"
#include "mttkrp.cuh"

namespace tsr {

namespace {

constexpr size_t kNoAllocScratchFloats = (size_t)4 << 20;  // 16 MiB of fp32 partials
__device__ __align__(256) float g_noalloc_partials[kNoAllocScratchFloats];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
float* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device. The array's
// host-side name is only a stand-in; a kernel must be given this address.
int scratch_for_current_device(float** out) {
  int dev = 0;
  TSR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(TSR_E_UNSUPPORTED, "device ordinal %d", dev);
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p)
      return fail(TSR_E_CUDA, "cudaGetSymbolAddress of the MTTKRP scratch failed: %s",
                  cudaGetErrorString(e));
    g_scratch_ptr[dev] = (float*)p;
  }
  *out = g_scratch_ptr[dev];
  return TSR_OK;
}

}  // namespace

}  // namespace tsr

using namespace tsr;

extern "C" {

int tsr_mttkrp_mode0_noalloc_f32(void* stream, const float* d_tensor, int ndim,
                                 const int64_t* shape, const float* const* d_factors,
                                 int64_t rank, float* d_out) {
  if (!shape || !d_tensor || !d_factors || !d_out) return fail(TSR_E_INVALID_ARG, "null argument");
  if (ndim < 2) return fail(TSR_E_NEED_2_FACTORS, "Need at least 2 factor matrices for MTTKRP");
  if (ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d exceeds the supported %d", ndim, kMaxModes);
  if (rank <= 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  for (int d = 0; d < ndim; ++d)
    if (shape[d] < 0)
      return fail(TSR_E_INVALID_ARG, "mode %d has a negative size (%lld)", d, (long long)shape[d]);
  // the kernels run on the caller's stream, the scratch address and the SM
  // count come from the current device: both must be the same device
  int dev = 0;
  TSR_CUDA(cudaGetDevice(&dev));
  if (stream) {
    int sdev = -1;
    TSR_CUDA(cudaStreamGetDevice((cudaStream_t)stream, &sdev));
    if (sdev != dev)
      return fail(TSR_E_INVALID_ARG,
                  "the stream belongs to device %d but device %d is current", sdev, dev);
  }
  const int64_t nout = shape[0] * rank;
  if (nout == 0) return TSR_OK;
  const Unfolding u = make_unfolding(ndim, shape, 0);
  if (u.cols == 0) {  // an empty sum over the other modes: the output is zero
    TSR_CUDA(cudaMemsetAsync(d_out, 0, sizeof(float) * nout, (cudaStream_t)stream));
    return TSR_OK;
  }
  if (u.cols % 4 != 0 || ((uintptr_t)d_tensor & 15))
    return fail(TSR_E_UNSUPPORTED,
                "allocation-free MTTKRP needs the product of the non-leading mode sizes to be a "
                "multiple of 4 and a 16-byte aligned tensor");
  // the row-major tensor is its own mode-0 unfolding (row stride = cols)
  Unfolding uu = u;
  uu.ld = u.cols;
  tsr_ctx shim;  // launch bookkeeping only: stream and SM count, no allocations
  shim.stream = (cudaStream_t)stream;
  TSR_CUDA(cudaDeviceGetAttribute(&shim.sm_count, cudaDevAttrMultiProcessorCount, dev));
  shim.reserve_sms = 0;
  const SplitPlan plan = plan_simt(&shim, u.rows, u.cols, (int)rank);
  const size_t need = partial_floats(plan, u.rows, (int)rank);
  if (need > kNoAllocScratchFloats)
    return fail(TSR_E_UNSUPPORTED,
                "allocation-free MTTKRP: %zu partial floats exceed the fixed %zu-float scratch "
                "(shape[0] x rank x splits too large)",
                need, kNoAllocScratchFloats);
  init_kernel_attributes();  // host-side launch attributes, once per device
  float* scratch;
  TSR_TRY(scratch_for_current_device(&scratch));
  FactorTable ft{};
  for (int m = 0; m < ndim; ++m) {
    ft.ptr[m] = d_factors[m];
    ft.rows[m] = shape[m];
  }
  const KRSpec kr = make_krspec(uu, ft, (int)rank);
  // every split writes all of its rows: nothing in the scratch needs zeroing
  TSR_TRY(launch_mttkrp_simt(&shim, d_tensor, uu, kr, plan, scratch));
  TSR_TRY(launch_mttkrp_reduce(&shim, scratch, plan.splits, u.rows * rank, d_out));
  return TSR_OK;
}

}  // extern "C"

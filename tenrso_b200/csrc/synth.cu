// Seeded synthetic sparse input on the device: the Zipf COO workload of
// tenrso_b200.synth.zipf_coo, reproduced value for value (SplitMix64 streams,
// the same FP64 Zipf CDF table, the same seeded permutation, the same cut at
// the raw prefix that holds exactly `nnz` distinct coordinates), so that a
// 5e7-entry tensor can be drawn without a host round trip.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <numeric>

#include "common.cuh"

namespace tsr {
namespace {

constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;

__host__ __device__ inline uint64_t mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ inline uint64_t stream_key(uint64_t seed, uint64_t stream) {
  return mix(seed * 0x100000001B3ull + stream * 0x2545F4914F6CDD1Dull + kGolden);
}

__device__ inline double uniform_at(uint64_t key, uint64_t i) {
  return (double)(mix(key + i * kGolden) >> 11) * (1.0 / 9007199254740992.0);
}

struct ZipfMode {
  const double* cdf;       // [size], normalised cumulative Zipf weights
  const int64_t* perm;     // [size], seeded permutation of 0..size-1
  int64_t size;
  uint64_t key;            // stream key of this mode's uniforms
};

struct ZipfArgs {
  int ndim;
  ZipfMode m[kMaxModes];
  uint64_t stride[kMaxModes];  // row-major key strides
};

__global__ void zipf_draw_kernel(ZipfArgs a, int64_t start, int64_t n, int64_t* __restrict__ idx,
                                 uint64_t* __restrict__ keys) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = start + t;
    uint64_t key = 0;
    for (int d = 0; d < a.ndim; ++d) {
      const double u = uniform_at(a.m[d].key, (uint64_t)g);
      // numpy searchsorted(cdf, u, side="right"): first i with cdf[i] > u
      int64_t lo = 0, hi = a.m[d].size;
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a.m[d].cdf[mid] > u)
          hi = mid;
        else
          lo = mid + 1;
      }
      const int64_t z = lo < a.m[d].size - 1 ? lo : a.m[d].size - 1;
      const int64_t v = a.m[d].perm[z];
      idx[g * a.ndim + d] = v;
      key += (uint64_t)v * a.stride[d];
    }
    keys[g] = key;
  }
}

__global__ void iota_kernel(uint32_t* p, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = (uint32_t)i;
}

// first occurrence (smallest position) of each distinct key: run heads of the
// stable sort
__global__ void first_occ_kernel(const uint64_t* __restrict__ skeys,
                                 const uint32_t* __restrict__ spos, int64_t n,
                                 uint32_t* __restrict__ heads_pos, uint32_t* __restrict__ flags) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const bool head = p == 0 || skeys[p] != skeys[p - 1];
    flags[p] = head ? 1u : 0u;
    heads_pos[p] = head ? spos[p] : 0xFFFFFFFFu;
  }
}

__global__ void vals_kernel(uint64_t key, int64_t n, float* __restrict__ vals) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    vals[i] = (float)uniform_at(key, (uint64_t)i);
}

unsigned grid_of(const tsr_ctx* ctx, int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), ctx->sm_count * 16));
}

}  // namespace
}  // namespace tsr

using namespace tsr;

extern "C" {

int tsr_synth_zipf_coo_dev(tsr_ctx* ctx, int ndim, const int64_t* shape, int64_t nnz,
                           uint64_t seed, double s_exp, int64_t capacity, int64_t* d_indices,
                           float* d_values, int64_t* n_raw_out) {
  if (!shape || !d_indices || !d_values || !n_raw_out || nnz <= 0 || ndim <= 0 ||
      ndim > kMaxModes)
    return fail(TSR_E_INVALID_ARG, "invalid argument");
  TSR_TRY(check_ctx(ctx));
  cudaStream_t s = ctx->stream;
  // host tables: Zipf CDF (as numpy: cumsum of rank^-s, then / last) and the
  // permutation argsort(raw_u64(seed, stream + 0x777, size), stable)
  std::vector<void*> allocs;
  auto dalloc = [&](size_t bytes, void** p) -> int {
    cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) return fail(TSR_E_CUDA, "cudaMalloc: %s", cudaGetErrorString(e));
    allocs.push_back(*p);
    return TSR_OK;
  };
  auto release = [&]() {
    cudaStreamSynchronize(s);
    for (void* p : allocs) cudaFree(p);
  };
  ZipfArgs za{};
  za.ndim = ndim;
  uint64_t st = 1;
  for (int d = ndim - 1; d >= 0; --d) {
    za.stride[d] = st;
    st *= (uint64_t)shape[d];
  }
  for (int d = 0; d < ndim; ++d) {
    const int64_t n = shape[d];
    std::vector<double> cdf(n);
    double acc = 0.0;
    for (int64_t r = 0; r < n; ++r) {
      acc += std::pow((double)(r + 1), -s_exp);
      cdf[r] = acc;
    }
    const double last = cdf[n - 1];
    for (auto& c : cdf) c /= last;
    const uint64_t pk = stream_key(seed, 10 + d + 0x777);
    std::vector<uint64_t> raw(n);
    for (int64_t i = 0; i < n; ++i) raw[i] = mix(pk + (uint64_t)i * kGolden);
    std::vector<int64_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int64_t x, int64_t y) { return raw[x] < raw[y]; });
    void *dc, *dp;
    if (dalloc(sizeof(double) * n, &dc) || dalloc(sizeof(int64_t) * n, &dp)) {
      release();
      return TSR_E_CUDA;
    }
    cudaMemcpyAsync(dc, cdf.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dp, perm.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    za.m[d].cdf = (const double*)dc;
    za.m[d].perm = (const int64_t*)dp;
    za.m[d].size = n;
    za.m[d].key = stream_key(seed, 10 + d);
  }
  // draw until the raw prefix holds at least nnz distinct coordinates
  uint64_t* keys;
  uint64_t* skeys;
  uint32_t *pos, *spos, *hpos, *flags, *shpos;
  const int64_t cap = std::min<int64_t>(capacity, INT32_MAX - 1);
  if (dalloc(8 * cap, (void**)&keys) || dalloc(8 * cap, (void**)&skeys) ||
      dalloc(4 * cap, (void**)&pos) || dalloc(4 * cap, (void**)&spos) ||
      dalloc(4 * cap, (void**)&hpos) || dalloc(4 * cap, (void**)&flags) ||
      dalloc(4 * cap, (void**)&shpos)) {
    release();
    return TSR_E_CUDA;
  }
  int bits = 1;
  while (bits < 64 && (long double)(1ull << bits) < (long double)st) ++bits;
  int64_t drawn = 0, batch = std::max<int64_t>(nnz, 1024), distinct = 0;
  int rc = TSR_OK;
  while (true) {
    const int64_t n_new = std::min(batch, cap - drawn);
    if (n_new <= 0) {
      rc = fail(TSR_E_UNSUPPORTED, "Zipf draw needs more than %lld raw entries",
                (long long)cap);
      break;
    }
    zipf_draw_kernel<<<grid_of(ctx, n_new), 256, 0, s>>>(za, drawn, n_new, d_indices, keys);
    ctx->launches++;
    drawn += n_new;
    iota_kernel<<<grid_of(ctx, drawn), 256, 0, s>>>(pos, drawn);
    size_t temp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, temp, keys, skeys, pos, spos, (int)drawn, 0, bits, s);
    void* tmp = nullptr;
    if (dalloc(temp, &tmp)) {
      rc = TSR_E_CUDA;
      break;
    }
    cub::DeviceRadixSort::SortPairs(tmp, temp, keys, skeys, pos, spos, (int)drawn, 0, bits, s);
    first_occ_kernel<<<grid_of(ctx, drawn), 256, 0, s>>>(skeys, spos, drawn, hpos, flags);
    ctx->launches += 2;
    // count distinct keys
    uint32_t* dsum;
    if (dalloc(8, (void**)&dsum)) {
      rc = TSR_E_CUDA;
      break;
    }
    size_t t2 = 0;
    cub::DeviceReduce::Sum(nullptr, t2, flags, dsum, (int)drawn, s);
    void* tmp2 = nullptr;
    if (dalloc(t2, &tmp2)) {
      rc = TSR_E_CUDA;
      break;
    }
    cub::DeviceReduce::Sum(tmp2, t2, flags, dsum, (int)drawn, s);
    uint32_t h = 0;
    cudaMemcpyAsync(&h, dsum, 4, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    distinct = h;
    if (distinct >= nnz) {
      // sort the first-occurrence positions; the nnz-th smallest ends the prefix
      size_t t3 = 0;
      cub::DeviceRadixSort::SortKeys(nullptr, t3, hpos, shpos, (int)drawn, 0, 32, s);
      void* tmp3 = nullptr;
      if (dalloc(t3, &tmp3)) {
        rc = TSR_E_CUDA;
        break;
      }
      cub::DeviceRadixSort::SortKeys(tmp3, t3, hpos, shpos, (int)drawn, 0, 32, s);
      uint32_t cut_pos = 0;
      cudaMemcpyAsync(&cut_pos, shpos + (nnz - 1), 4, cudaMemcpyDeviceToHost, s);
      cudaStreamSynchronize(s);
      const int64_t cut = (int64_t)cut_pos + 1;
      vals_kernel<<<grid_of(ctx, cut), 256, 0, s>>>(stream_key(seed, 50), cut, d_values);
      ctx->launches++;
      *n_raw_out = cut;
      break;
    }
    batch = drawn;  // geometric growth; the prefix does not depend on batching
  }
  cudaError_t e = cudaGetLastError();
  release();
  if (rc != TSR_OK) return rc;
  if (e != cudaSuccess) return fail(TSR_E_CUDA, "%s", cudaGetErrorString(e));
  return TSR_OK;
}

}  // extern "C"

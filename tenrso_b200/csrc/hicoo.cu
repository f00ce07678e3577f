// HiCOO (hierarchical COO) tensors on the device and their MTTKRP.
//
// Construction follows HiCooTensor::from_coo (crates/tenrso-sparse/src/
// hicoo.rs:118-203): every entry splits into its block coordinate i / b and
// its local coordinate i % b per mode; the entries are stably sorted by block
// coordinate (lexicographic, mode 0 most significant), keeping the input
// order inside a block; block_ptrs holds the cumulative entry counts
// (num_blocks + 1 values) and block_coords the distinct blocks in order. No
// entries are merged.
//
// Device layout: block pointers and block coordinates as u32, local
// coordinates as u8 (block sides up to 256), values fp32.
//
// The reference has no HiCOO MTTKRP (the format's documentation names it as
// the use case, hicoo.rs:30-34). Its definition is the sparse MTTKRP
// M[i_n, r] = sum over entries of v * prod_{m != n} U_m[i_m, r]. One warp
// owns one block at a time: lanes hold columns, each entry's factor rows are
// gathered from the block's slices of the factors, and the products collect
// in an fp32 shared-memory tile of the block's b_n output rows; at the end
// of the block the rows it touched are added to the FP64 output with
// atomics and cleared.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "csf.cuh"

struct tsr_hicoo {
  int device = 0;
  int ndim = 0;
  int64_t shape[tsr::kMaxModes] = {};
  int64_t block_shape[tsr::kMaxModes] = {};
  int64_t nnz = 0;
  int64_t n_blocks = 0;
  uint32_t* block_ptr = nullptr;    // [n_blocks + 1]
  uint32_t* block_coord = nullptr;  // [n_blocks][ndim]
  uint8_t* local = nullptr;         // [nnz][ndim]
  float* vals = nullptr;            // [nnz]
  std::vector<void*> allocs;
};

namespace tsr {

namespace {

unsigned hc_grid(const tsr_ctx* ctx, int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), ctx->sm_count * 16));
}

struct BlockSpec {
  int ndim;
  int64_t bs[kMaxModes];      // block side per mode
  uint64_t stride[kMaxModes];  // key stride of each mode's block coordinate
  uint64_t nb[kMaxModes];      // blocks per mode
};

// Block key (row-major over block coordinates) and input position.
__global__ void hicoo_keys_kernel(const int64_t* __restrict__ idx, int64_t nnz, BlockSpec bs,
                                  uint64_t* __restrict__ keys, uint32_t* __restrict__ pos) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
       k += (int64_t)gridDim.x * blockDim.x) {
    uint64_t key = 0;
    for (int m = 0; m < bs.ndim; ++m)
      key += (uint64_t)(idx[k * bs.ndim + m] / bs.bs[m]) * bs.stride[m];
    keys[k] = key;
    pos[k] = (uint32_t)k;
  }
}

// 1 where a new block starts in the sorted order.
__global__ void hicoo_flags_kernel(const uint64_t* __restrict__ keys, int64_t n,
                                   uint32_t* __restrict__ flags) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    flags[k] = (k == 0 || keys[k] != keys[k - 1]) ? 1u : 0u;
}

// Per sorted entry: local coordinates and value; per block start: the block's
// pointer and coordinates.
__global__ void hicoo_fill_kernel(const uint64_t* __restrict__ keys,
                                  const uint32_t* __restrict__ pos,
                                  const uint32_t* __restrict__ flags,
                                  const uint32_t* __restrict__ offs,
                                  const int64_t* __restrict__ idx, const float* __restrict__ vin,
                                  int64_t nnz, BlockSpec bs, uint32_t* __restrict__ bptr,
                                  uint32_t* __restrict__ bcoord, uint8_t* __restrict__ local,
                                  float* __restrict__ vout) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t src = pos[k];
    for (int m = 0; m < bs.ndim; ++m)
      local[k * bs.ndim + m] = (uint8_t)(idx[src * bs.ndim + m] % bs.bs[m]);
    vout[k] = vin[src];
    if (flags[k]) {
      const uint32_t b = offs[k];
      bptr[b] = (uint32_t)k;
      uint64_t key = keys[k];
      for (int m = bs.ndim - 1; m >= 0; --m) {
        bcoord[(int64_t)b * bs.ndim + m] = (uint32_t)(key % bs.nb[m]);
        key /= bs.nb[m];
      }
    }
  }
}

struct HicooArgs {
  int ndim, mode, R;
  int64_t n_blocks;
  int bs[kMaxModes];
  const uint32_t* block_ptr;
  const uint32_t* block_coord;
  const uint8_t* local;
  const float* vals;
  const float* U[kMaxModes];
  double* M;  // FP64 output accumulator (shape[mode] x R), zeroed by the caller
  int tile;   // 1: shared-memory tile of the block's output rows; 0: direct atomics
};

constexpr int HC_WARPS = 4;

__global__ void __launch_bounds__(HC_WARPS * 32) hicoo_mttkrp_kernel(HicooArgs a) {
  extern __shared__ __align__(16) float hc_tile[];  // HC_WARPS x b_n x R
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int R = a.R, ndim = a.ndim, mode = a.mode;
  const int bsn = a.bs[mode];
  float* tile = hc_tile + (size_t)warp * bsn * R;
  if (a.tile)
    for (int e = lane; e < bsn * R; e += 32) tile[e] = 0.f;
  __syncwarp();
  for (int64_t b = (int64_t)blockIdx.x * HC_WARPS + warp; b < a.n_blocks;
       b += (int64_t)gridDim.x * HC_WARPS) {
    const uint32_t* bc = a.block_coord + b * ndim;
    int64_t base[kMaxModes];
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m) base[m] = m < ndim ? (int64_t)bc[m] * a.bs[m] : 0;
    uint32_t touched[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};  // rows 0..255 of the tile
    const uint32_t k1 = a.block_ptr[b + 1];
    for (uint32_t k = a.block_ptr[b]; k < k1; ++k) {
      const uint8_t* lc = a.local + (int64_t)k * ndim;
      const float v = a.vals[k];
      const int rn = lc[mode];
      for (int c = lane; c < R; c += 32) {
        float p = v;
        for (int m = 0; m < ndim; ++m)
          if (m != mode) p *= __ldg(a.U[m] + (base[m] + lc[m]) * R + c);
        if (a.tile)
          tile[rn * R + c] += p;  // the warp's lanes own distinct columns
        else
          atomicAdd(a.M + (base[mode] + rn) * R + c, (double)p);
      }
      touched[rn >> 5] |= 1u << (rn & 31);
    }
    if (a.tile) {
      __syncwarp();
#pragma unroll
      for (int w = 0; w < 8; ++w) {
        uint32_t mask = touched[w];
        while (mask) {
          const int rn = w * 32 + __ffs(mask) - 1;
          mask &= mask - 1u;
          for (int c = lane; c < R; c += 32) {
            atomicAdd(a.M + (base[mode] + rn) * R + c, (double)tile[rn * R + c]);
            tile[rn * R + c] = 0.f;
          }
        }
      }
      __syncwarp();
    }
  }
}

__global__ void hc_f64_to_f32(const double* __restrict__ in, int64_t n, float* __restrict__ out) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    out[e] = (float)in[e];
}

int hicoo_alloc(tsr_hicoo* h, size_t bytes, void** p) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess)
    return fail(TSR_E_CUDA, "cudaMalloc (%zu bytes): %s", bytes, cudaGetErrorString(e));
  h->allocs.push_back(q);
  *p = q;
  return TSR_OK;
}

void hicoo_free(tsr_hicoo* h) {
  for (void* p : h->allocs) cudaFree(p);
  h->allocs.clear();
}

// hicoo.rs:118-133 (same messages).
int check_block_shape(int ndim, const int64_t* block_shape, int n_block) {
  if (n_block != ndim)
    return fail(TSR_E_BLOCK_SHAPE, "Invalid block shape: block_shape length %d != ndim %d",
                n_block, ndim);
  for (int m = 0; m < ndim; ++m)
    if (block_shape[m] == 0)
      return fail(TSR_E_BLOCK_SHAPE, "Invalid block shape: block_shape cannot contain zeros");
  for (int m = 0; m < ndim; ++m)
    if (block_shape[m] < 0 || block_shape[m] > 256)
      return fail(TSR_E_UNSUPPORTED,
                  "block sides above 256 do not fit the u8 local coordinates (got %lld)",
                  (long long)block_shape[m]);
  return TSR_OK;
}

int hicoo_build(tsr_ctx* ctx, const int64_t* d_idx, const float* d_vals, int64_t nnz,
                tsr_hicoo* h) {
  cudaStream_t s = ctx->stream;
  h->nnz = nnz;
  BlockSpec bs;
  bs.ndim = h->ndim;
  long double total = 1.0L;
  for (int m = 0; m < h->ndim; ++m) {
    bs.bs[m] = h->block_shape[m];
    bs.nb[m] = (uint64_t)ceil_div(h->shape[m], h->block_shape[m]);
    total *= (long double)bs.nb[m];
  }
  if (total > 1.8e19L) return fail(TSR_E_UNSUPPORTED, "more than 2^64 blocks");
  uint64_t st = 1;
  for (int m = h->ndim - 1; m >= 0; --m) {
    bs.stride[m] = st;
    st *= bs.nb[m];
  }
  int bits = 1;
  while (bits < 64 && (long double)(1ull << bits) < total) ++bits;
  void *p;
  TSR_TRY(hicoo_alloc(h, sizeof(uint32_t) * (nnz + 1), &p));
  h->block_ptr = (uint32_t*)p;
  if (nnz == 0) {
    // hicoo.rs:135-148: no blocks, block_ptrs = [0]
    TSR_CUDA(cudaMemsetAsync(h->block_ptr, 0, sizeof(uint32_t), s));
    TSR_CUDA(cudaStreamSynchronize(s));
    h->n_blocks = 0;
    return TSR_OK;
  }
  // scratch: keys (2x), positions (2x), flags, offsets, sort temp
  std::vector<void*> scratch;
  auto sget = [&](size_t bytes, void** q) -> int {
    void* r = nullptr;
    cudaError_t e = cudaMalloc(&r, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess)
      return fail(TSR_E_CUDA, "cudaMalloc (%zu bytes): %s", bytes, cudaGetErrorString(e));
    scratch.push_back(r);
    *q = r;
    return TSR_OK;
  };
  auto release = [&]() {
    for (void* q : scratch) cudaFree(q);
  };
  int rc = TSR_OK;
  void *ka, *kb, *pa, *pb, *fl, *of, *tmp;
  do {
    if ((rc = sget(8 * nnz, &ka)) || (rc = sget(8 * nnz, &kb)) || (rc = sget(4 * nnz, &pa)) ||
        (rc = sget(4 * nnz, &pb)) || (rc = sget(4 * nnz, &fl)) || (rc = sget(4 * nnz, &of)))
      break;
    hicoo_keys_kernel<<<hc_grid(ctx, nnz), 256, 0, s>>>(d_idx, nnz, bs, (uint64_t*)ka,
                                                        (uint32_t*)pa);
    ctx->launches++;
    // radix sort is stable: entries of one block keep their input order
    size_t temp = 0, temp2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, temp, (uint64_t*)ka, (uint64_t*)kb,
                                    (uint32_t*)pa, (uint32_t*)pb, (int)nnz, 0, bits, s);
    cub::DeviceScan::ExclusiveSum(nullptr, temp2, (uint32_t*)fl, (uint32_t*)of, (int)nnz, s);
    if ((rc = sget(std::max(temp, temp2), &tmp))) break;
    if (cub::DeviceRadixSort::SortPairs(tmp, temp, (uint64_t*)ka, (uint64_t*)kb, (uint32_t*)pa,
                                        (uint32_t*)pb, (int)nnz, 0, bits, s) != cudaSuccess) {
      rc = fail(TSR_E_CUDA, "block sort failed");
      break;
    }
    hicoo_flags_kernel<<<hc_grid(ctx, nnz), 256, 0, s>>>((uint64_t*)kb, nnz, (uint32_t*)fl);
    ctx->launches++;
    if (cub::DeviceScan::ExclusiveSum(tmp, temp2, (uint32_t*)fl, (uint32_t*)of, (int)nnz, s) !=
        cudaSuccess) {
      rc = fail(TSR_E_CUDA, "block scan failed");
      break;
    }
    uint32_t last[2];
    cudaMemcpyAsync(&last[0], (uint32_t*)of + nnz - 1, 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&last[1], (uint32_t*)fl + nnz - 1, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      rc = fail(TSR_E_CUDA, "block count read failed");
      break;
    }
    h->n_blocks = (int64_t)last[0] + last[1];
    void *bc, *lc, *vv;
    if ((rc = hicoo_alloc(h, sizeof(uint32_t) * h->n_blocks * h->ndim, &bc)) ||
        (rc = hicoo_alloc(h, (size_t)nnz * h->ndim, &lc)) ||
        (rc = hicoo_alloc(h, sizeof(float) * nnz, &vv)))
      break;
    h->block_coord = (uint32_t*)bc;
    h->local = (uint8_t*)lc;
    h->vals = (float*)vv;
    hicoo_fill_kernel<<<hc_grid(ctx, nnz), 256, 0, s>>>(
        (uint64_t*)kb, (uint32_t*)pb, (uint32_t*)fl, (uint32_t*)of, d_idx, d_vals, nnz, bs,
        h->block_ptr, h->block_coord, h->local, h->vals);
    ctx->launches++;
    const uint32_t end = (uint32_t)nnz;
    cudaMemcpyAsync(h->block_ptr + h->n_blocks, &end, 4, cudaMemcpyHostToDevice, s);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
      rc = fail(TSR_E_CUDA, "HiCOO build failed");
  } while (false);
  release();
  return rc;
}

}  // namespace

int launch_mttkrp_hicoo(tsr_ctx* ctx, cudaStream_t s, const tsr_hicoo* h,
                        const float* const* d_factors, int R, int mode, float* d_out,
                        double* d_acc) {
  const int64_t n_out = h->shape[mode] * R;
  TSR_CUDA(cudaMemsetAsync(d_acc, 0, sizeof(double) * n_out, s));
  if (h->n_blocks > 0) {
    HicooArgs a;
    a.ndim = h->ndim;
    a.mode = mode;
    a.R = R;
    a.n_blocks = h->n_blocks;
    for (int m = 0; m < kMaxModes; ++m) {
      a.bs[m] = m < h->ndim ? (int)h->block_shape[m] : 1;
      a.U[m] = m < h->ndim ? d_factors[m] : nullptr;
    }
    a.block_ptr = h->block_ptr;
    a.block_coord = h->block_coord;
    a.local = h->local;
    a.vals = h->vals;
    a.M = d_acc;
    // the b_n x R fp32 tile of each warp must fit in 48 KB
    const size_t tile_bytes = sizeof(float) * (size_t)h->block_shape[mode] * R;
    a.tile = tile_bytes <= 48 * 1024 ? 1 : 0;
    const size_t smem = a.tile ? tile_bytes * HC_WARPS : 0;
    const unsigned grid = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(ceil_div(h->n_blocks, HC_WARPS), 4 * (int64_t)ctx->sm_count));
    hicoo_mttkrp_kernel<<<grid, HC_WARPS * 32, smem, s>>>(a);
    ctx->launches++;
    TSR_CUDA(cudaGetLastError());
  }
  hc_f64_to_f32<<<hc_grid(ctx, n_out), 256, 0, s>>>(d_acc, n_out, d_out);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

void init_hicoo_attributes() {
  cudaFuncSetAttribute(hicoo_mttkrp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       HC_WARPS * 48 * 1024);
}

}  // namespace tsr

using namespace tsr;

extern "C" {

int tsr_hicoo_create_f32(tsr_ctx* ctx, const int64_t* indices, const float* values, int64_t nnz,
                         int ndim, const int64_t* shape, const int64_t* block_shape,
                         int n_block_shape, tsr_hicoo** out) {
  if (!shape || !out || (n_block_shape > 0 && !block_shape) ||
      (nnz > 0 && (!indices || !values)))
    return fail(TSR_E_INVALID_ARG, "null argument");
  *out = nullptr;
  TSR_TRY(coo_check_shape(ndim, shape));
  TSR_TRY(check_block_shape(ndim, block_shape, n_block_shape));
  if (nnz < 0) return fail(TSR_E_INVALID_ARG, "negative entry count");
  TSR_TRY(coo_check_bounds(indices, nnz, ndim, shape));
  if (nnz >= (int64_t)UINT32_MAX) return fail(TSR_E_UNSUPPORTED, "more than 2^32 - 1 entries");
  TSR_TRY(check_ctx(ctx));
  void *a = nullptr, *b = nullptr;
  TSR_TRY(slot_get(ctx, SLOT_SPARSE1, sizeof(int64_t) * std::max<int64_t>(nnz, 1) * ndim, &a));
  TSR_TRY(slot_get(ctx, SLOT_SPARSE1 + 1, sizeof(float) * std::max<int64_t>(nnz, 1), &b));
  if (nnz > 0) {
    TSR_CUDA(cudaMemcpyAsync(a, indices, sizeof(int64_t) * nnz * ndim, cudaMemcpyHostToDevice,
                             ctx->stream));
    TSR_CUDA(
        cudaMemcpyAsync(b, values, sizeof(float) * nnz, cudaMemcpyHostToDevice, ctx->stream));
  }
  tsr_hicoo* h = new tsr_hicoo();
  h->device = ctx->device;
  h->ndim = ndim;
  for (int m = 0; m < ndim; ++m) {
    h->shape[m] = shape[m];
    h->block_shape[m] = block_shape[m];
  }
  int rc = hicoo_build(ctx, (const int64_t*)a, (const float*)b, nnz, h);
  if (rc != TSR_OK) {
    hicoo_free(h);
    delete h;
    return rc;
  }
  *out = h;
  return TSR_OK;
}

int tsr_hicoo_destroy(tsr_hicoo* h) {
  if (!h) return TSR_OK;
  hicoo_free(h);
  delete h;
  return TSR_OK;
}

int tsr_hicoo_info(const tsr_hicoo* h, int64_t* nnz, int64_t* num_blocks) {
  if (!h) return fail(TSR_E_INVALID_ARG, "null argument");
  if (nnz) *nnz = h->nnz;
  if (num_blocks) *num_blocks = h->n_blocks;
  return TSR_OK;
}

int tsr_hicoo_export(tsr_ctx* ctx, const tsr_hicoo* h, int64_t* block_coords,
                     int64_t* block_ptrs, int64_t* local_coords, float* values) {
  if (!h) return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(check_ctx(ctx));
  const int64_t nb = h->n_blocks, nnz = h->nnz, d = h->ndim;
  std::vector<uint32_t> bp(nb + 1), bc(nb * d);
  std::vector<uint8_t> lc(nnz * d);
  TSR_CUDA(cudaMemcpy(bp.data(), h->block_ptr, 4 * (nb + 1), cudaMemcpyDeviceToHost));
  if (nb > 0) TSR_CUDA(cudaMemcpy(bc.data(), h->block_coord, 4 * nb * d, cudaMemcpyDeviceToHost));
  if (nnz > 0) {
    TSR_CUDA(cudaMemcpy(lc.data(), h->local, nnz * d, cudaMemcpyDeviceToHost));
    if (values) TSR_CUDA(cudaMemcpy(values, h->vals, 4 * nnz, cudaMemcpyDeviceToHost));
  }
  if (block_ptrs)
    for (int64_t i = 0; i <= nb; ++i) block_ptrs[i] = bp[i];
  if (block_coords)
    for (int64_t i = 0; i < nb * d; ++i) block_coords[i] = bc[i];
  if (local_coords)
    for (int64_t i = 0; i < nnz * d; ++i) local_coords[i] = lc[i];
  return TSR_OK;
}

int tsr_mttkrp_hicoo_dev_f32(tsr_ctx* ctx, const tsr_hicoo* h, const float* const* d_factors,
                             int64_t rank, int mode, float* d_out) {
  if (!h || !d_factors || !d_out) return fail(TSR_E_INVALID_ARG, "null argument");
  if (mode < 0 || mode >= h->ndim)
    return fail(TSR_E_MODE_OOB, "Mode %d out of bounds for tensor with rank %d", mode, h->ndim);
  if (rank <= 0 || rank > (1 << 20)) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld",
                                                 (long long)rank);
  TSR_TRY(check_ctx(ctx));
  void* acc;
  TSR_TRY(slot_get(ctx, SLOT_MISC2, sizeof(double) * h->shape[mode] * rank, &acc));
  TSR_TRY(launch_mttkrp_hicoo(ctx, ctx->stream, h, d_factors, (int)rank, mode, d_out,
                              (double*)acc));
  return TSR_OK;
}

int tsr_mttkrp_hicoo_f32(tsr_ctx* ctx, const tsr_hicoo* h, const float* const* factors,
                         int64_t rank, int mode, float* out) {
  if (!h || !factors || !out) return fail(TSR_E_INVALID_ARG, "null argument");
  if (mode < 0 || mode >= h->ndim)
    return fail(TSR_E_MODE_OOB, "Mode %d out of bounds for tensor with rank %d", mode, h->ndim);
  if (rank <= 0 || rank > (1 << 20)) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld",
                                                 (long long)rank);
  TSR_TRY(check_ctx(ctx));
  int64_t total = 0;
  for (int m = 0; m < h->ndim; ++m) total += h->shape[m] * rank;
  void* fbuf;
  TSR_TRY(slot_get(ctx, SLOT_FACTORS, sizeof(float) * total, &fbuf));
  const float* dptr[kMaxModes];
  int64_t off = 0;
  for (int m = 0; m < h->ndim; ++m) {
    float* d = (float*)fbuf + off;
    TSR_CUDA(cudaMemcpyAsync(d, factors[m], sizeof(float) * h->shape[m] * rank,
                             cudaMemcpyHostToDevice, ctx->stream));
    dptr[m] = d;
    off += h->shape[m] * rank;
  }
  void* dout;
  TSR_TRY(slot_get(ctx, SLOT_OUT, sizeof(float) * h->shape[mode] * rank, &dout));
  TSR_TRY(tsr_mttkrp_hicoo_dev_f32(ctx, h, dptr, rank, mode, (float*)dout));
  TSR_CUDA(cudaMemcpyAsync(out, dout, sizeof(float) * h->shape[mode] * rank,
                           cudaMemcpyDeviceToHost, ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

}  // extern "C"

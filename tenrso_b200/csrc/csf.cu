// COO deduplication, CSF construction and CSF MTTKRP on the device.
//
// Replaces, in crates/tenrso-sparse/src/:
//   CooTensor::sort / deduplicate   coo.rs:239-257, 320-347
//   CsfTensor::from_coo             csf.rs:137-264
// and adds the sparse MTTKRP that tenrso only mentions (csf.rs:42): the dense
// MTTKRP mathematics (mttkrp.rs:851-875) restricted to the nonzeros.
//
// Construction: each entry gets a mixed-radix key whose digits are its indices
// in mode_order; a stable LSD radix sort of (key, original position) gives the
// order of Rust's stable sort_by (coo.rs:247, csf.rs:178). Level-l fibers start
// where the key prefix of levels 0..l changes; their starts (nnz offsets, as
// the reference stores them) and digits are compacted with a scan. The key sort
// and scans use CUB from the CUDA toolkit (one-time preprocessing); the MTTKRP
// and every ALS kernel are written here.
#include <cub/cub.cuh>

#include <algorithm>
#include <numeric>
#include <string>

#include "csf.cuh"

namespace tsr {

namespace {

struct KeySpec {
  int ndim;
  int mo[kMaxModes];            // mode at each level
  uint64_t stride[kMaxModes];   // key stride of each level
  int64_t shape[kMaxModes];     // by mode
};

__global__ void coo_keys_kernel(const int64_t* __restrict__ idx, int64_t nnz, KeySpec ks,
                                uint64_t* __restrict__ keys, uint32_t* __restrict__ pos,
                                unsigned* status) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
       k += (int64_t)gridDim.x * blockDim.x) {
    uint64_t key = 0;
    bool bad = false;
    for (int l = 0; l < ks.ndim; ++l) {
      const int m = ks.mo[l];
      const int64_t v = idx[k * ks.ndim + m];
      bad |= (v < 0 || v >= ks.shape[m]);
      key += (uint64_t)(v < 0 ? 0 : v) * ks.stride[l];
    }
    keys[k] = key;
    pos[k] = (uint32_t)k;
    if (bad) atomicOr(status, DS_BAD_INDEX);
  }
}

__global__ void flags_kernel(const uint64_t* __restrict__ keys, int64_t n, uint64_t div,
                             uint32_t* __restrict__ flags) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x)
    flags[p] = (p == 0 || keys[p] / div != keys[p - 1] / div) ? 1u : 0u;
}

__global__ void compact_kernel(const uint64_t* __restrict__ keys,
                               const uint32_t* __restrict__ flags,
                               const uint32_t* __restrict__ offs, int64_t n, uint64_t div,
                               uint64_t size, uint32_t* __restrict__ ptr,
                               uint32_t* __restrict__ ids) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    if (flags[p]) {
      const uint32_t o = offs[p];
      ptr[o] = (uint32_t)p;
      if (ids) ids[o] = (uint32_t)((keys[p] / div) % size);
    }
  }
}

__global__ void leaf_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ pos,
                            const float* __restrict__ vin, int64_t n, uint64_t size,
                            uint32_t* __restrict__ ids, float* __restrict__ vout) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    if (ids) ids[p] = (uint32_t)(keys[p] % size);
    vout[p] = vin[pos[p]];
  }
}

// coo.rs:330-346: duplicates (equal keys, consecutive after the stable sort)
// are summed left to right in fp32, in original insertion order.
__global__ void segment_sum_kernel(const uint32_t* __restrict__ heads, int64_t count,
                                   int64_t n, const uint32_t* __restrict__ pos,
                                   const float* __restrict__ vin, float* __restrict__ vout) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < count;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t st = heads[s];
    const int64_t en = s + 1 < count ? (int64_t)heads[s + 1] : n;
    float v = vin[pos[st]];
    for (int64_t p = st + 1; p < en; ++p) v = __fadd_rn(v, vin[pos[p]]);
    vout[s] = v;
  }
}

__global__ void decode_kernel(const uint64_t* __restrict__ keys,
                              const uint32_t* __restrict__ heads, int64_t count, KeySpec ks,
                              int64_t* __restrict__ idx_out) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < count;
       s += (int64_t)gridDim.x * blockDim.x) {
    uint64_t key = keys[heads ? heads[s] : s];
    for (int l = ks.ndim - 1; l >= 0; --l) {
      const int m = ks.mo[l];
      idx_out[s * ks.ndim + m] = (int64_t)(key % (uint64_t)ks.shape[m]);
      key /= (uint64_t)ks.shape[m];
    }
  }
}

// largest f in [0, len) with ptr[f] <= k, for the first entry of every chunk
__global__ void chunk_search_kernel(const uint32_t* __restrict__ ptr, int64_t len,
                                    int64_t chunk_nnz, int64_t n_chunks,
                                    uint32_t* __restrict__ out) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n_chunks;
       c += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = (uint64_t)c * chunk_nnz;
    int64_t lo = 0, hi = len - 1;
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) / 2;
      if ((uint64_t)ptr[mid] <= k)
        lo = mid;
      else
        hi = mid - 1;
    }
    out[c] = (uint32_t)lo;
  }
}

__global__ void sumsq_kernel(const float* __restrict__ v, int64_t n, double* out) {
  double s = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    s += (double)v[k] * v[k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

unsigned grid_for(const tsr_ctx* ctx, int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), ctx->sm_count * 16));
}

// ---------------------------------------------------------------------------
// device allocation helpers for one build (freed by the caller's owner)
struct Arena {
  std::vector<void*> ptrs;
  template <class T>
  int get(T** p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) return fail(TSR_E_CUDA, "cudaMalloc (%zu bytes): %s", n * sizeof(T),
                                      cudaGetErrorString(e));
    ptrs.push_back(q);
    *p = (T*)q;
    return TSR_OK;
  }
  void release() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
  }
};

int make_keyspec(int ndim, const int64_t* shape, const int* mo, KeySpec* ks) {
  ks->ndim = ndim;
  for (int m = 0; m < ndim; ++m) ks->shape[m] = shape[m];
  long double total = 1.0L;
  for (int m = 0; m < ndim; ++m) total *= (long double)shape[m];
  if (total > 1.8e19L)
    return fail(TSR_E_UNSUPPORTED, "tensor has more than 2^64 positions; keys do not fit");
  uint64_t st = 1;
  for (int l = ndim - 1; l >= 0; --l) {
    ks->mo[l] = mo[l];
    ks->stride[l] = st;
    st *= (uint64_t)shape[mo[l]];
  }
  return TSR_OK;
}

int key_bits(int ndim, const int64_t* shape) {
  long double total = 1.0L;
  for (int m = 0; m < ndim; ++m) total *= (long double)shape[m];
  int b = 1;
  while (b < 64 && (long double)(1ull << b) < total) ++b;
  return b;
}

// Sorted keys / positions of the entries in the order of `mo`. Outputs point
// into the arena.
int sort_entries(tsr_ctx* ctx, cudaStream_t s, Arena& ar, const int64_t* d_idx, int64_t nnz,
                 const KeySpec& ks, int bits, uint64_t** keys_out, uint32_t** pos_out) {
  uint64_t *ka, *kb;
  uint32_t *pa, *pb;
  TSR_TRY(ar.get(&ka, nnz));
  TSR_TRY(ar.get(&kb, nnz));
  TSR_TRY(ar.get(&pa, nnz));
  TSR_TRY(ar.get(&pb, nnz));
  TSR_TRY(reset_status(ctx));
  coo_keys_kernel<<<grid_for(ctx, nnz), 256, 0, s>>>(d_idx, nnz, ks, ka, pa, ctx->d_status);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  size_t temp = 0;
  TSR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, ka, kb, pa, pb, (int)nnz, 0, bits, s));
  void* tmp;
  TSR_TRY(ar.get((uint8_t**)&tmp, temp));
  TSR_CUDA(cub::DeviceRadixSort::SortPairs(tmp, temp, ka, kb, pa, pb, (int)nnz, 0, bits, s));
  unsigned st;
  TSR_TRY(read_status(ctx, &st));
  if (st & DS_BAD_INDEX)
    return fail(TSR_E_INDEX_OOB, "Index out of bounds: an index exceeds shape");
  *keys_out = kb;
  *pos_out = pb;
  return TSR_OK;
}

// Fibers of level `l` (key prefix over levels 0..l): nnz-offset starts (+ nnz
// at the end) and the level's index of each fiber. Returns the fiber count.
int level_fibers(tsr_ctx* ctx, cudaStream_t s, Arena& scratch, Arena& keep, const uint64_t* keys,
                 int64_t nnz, uint64_t div, uint64_t size, uint32_t** ptr, uint32_t** ids,
                 int64_t* count) {
  uint32_t *flags, *offs;
  TSR_TRY(scratch.get(&flags, nnz));
  TSR_TRY(scratch.get(&offs, nnz));
  flags_kernel<<<grid_for(ctx, nnz), 256, 0, s>>>(keys, nnz, div, flags);
  ctx->launches++;
  size_t temp = 0;
  TSR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, flags, offs, (int)nnz, s));
  void* tmp;
  TSR_TRY(scratch.get((uint8_t**)&tmp, temp));
  TSR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, temp, flags, offs, (int)nnz, s));
  uint32_t last[2];
  TSR_CUDA(cudaMemcpyAsync(&last[0], offs + nnz - 1, 4, cudaMemcpyDeviceToHost, s));
  TSR_CUDA(cudaMemcpyAsync(&last[1], flags + nnz - 1, 4, cudaMemcpyDeviceToHost, s));
  TSR_CUDA(cudaStreamSynchronize(s));
  const int64_t c = (int64_t)last[0] + last[1];
  TSR_TRY(keep.get(ptr, c + 1));
  if (ids) TSR_TRY(keep.get(ids, c));
  compact_kernel<<<grid_for(ctx, nnz), 256, 0, s>>>(keys, flags, offs, nnz, div, size, *ptr,
                                                    ids ? *ids : nullptr);
  ctx->launches++;
  const uint32_t end = (uint32_t)nnz;
  TSR_CUDA(cudaMemcpyAsync(*ptr + c, &end, 4, cudaMemcpyHostToDevice, s));
  TSR_CUDA(cudaStreamSynchronize(s));
  *count = c;
  return TSR_OK;
}

// Full CSF tree of the given mode order from device COO (AoS int64 indices).
int build_csf(tsr_ctx* ctx, cudaStream_t s, const int64_t* d_idx, const float* d_vals,
              int64_t nnz, int ndim, const int64_t* shape, const int* mo, bool tables,
              CsfDev* out) {
  KeySpec ks;
  TSR_TRY(make_keyspec(ndim, shape, mo, &ks));
  out->ndim = ndim;
  out->nnz = nnz;
  for (int m = 0; m < ndim; ++m) out->shape[m] = shape[m];
  for (int l = 0; l < ndim; ++l) out->mode_order[l] = mo[l];
  if (nnz == 0) return TSR_OK;
  Arena scratch, keep;
  uint64_t* keys;
  uint32_t* pos;
  int rc = sort_entries(ctx, s, scratch, d_idx, nnz, ks, key_bits(ndim, shape), &keys, &pos);
  if (rc != TSR_OK) {
    scratch.release();
    return rc;
  }
  // keep the sorted keys (the generic MTTKRP decodes them)
  uint64_t* kk;
  float* vals;
  TSR_TRY(keep.get(&kk, nnz));
  TSR_TRY(keep.get(&vals, nnz));
  TSR_CUDA(cudaMemcpyAsync(kk, keys, 8 * nnz, cudaMemcpyDeviceToDevice, s));
  out->keys = kk;
  out->vals = vals;
  // levels 0 .. ndim-2 (csf.rs:193-254); ndim == 1 has only its level 0
  const int nlev = ndim == 1 ? 1 : ndim - 1;
  for (int l = 0; l < nlev; ++l) {
    int64_t c;
    rc = level_fibers(ctx, s, scratch, keep, keys, nnz, ks.stride[l],
                      (uint64_t)shape[mo[l]], &out->level_ptr[l], &out->level_ids[l], &c);
    if (rc != TSR_OK) {
      scratch.release();
      keep.release();
      return rc;
    }
    out->level_len[l] = c;
  }
  uint32_t* leaf = nullptr;
  if (ndim > 1) TSR_TRY(keep.get(&leaf, nnz));
  leaf_kernel<<<grid_for(ctx, nnz), 256, 0, s>>>(keys, pos, d_vals, nnz,
                                                 (uint64_t)shape[mo[ndim - 1]], leaf, vals);
  ctx->launches++;
  if (ndim > 1) {
    out->level_ids[ndim - 1] = leaf;
    out->level_len[ndim - 1] = nnz;
    out->level_ptr[ndim - 1] = out->level_ptr[ndim - 2];  // csf.rs: leaf fptr = level ndim-2's
  }
  if (tables && ndim >= 2) {
    out->chunk_nnz = 256;
    out->n_chunks = ceil_div(nnz, out->chunk_nnz);
    TSR_TRY(keep.get(&out->chunk_root, out->n_chunks));
    chunk_search_kernel<<<grid_for(ctx, out->n_chunks), 256, 0, s>>>(
        out->level_ptr[0], out->level_len[0], out->chunk_nnz, out->n_chunks, out->chunk_root);
    ctx->launches++;
    if (ndim >= 3) {
      TSR_TRY(keep.get(&out->chunk_fiber, out->n_chunks));
      chunk_search_kernel<<<grid_for(ctx, out->n_chunks), 256, 0, s>>>(
          out->level_ptr[1], out->level_len[1], out->chunk_nnz, out->n_chunks,
          out->chunk_fiber);
      ctx->launches++;
    }
  }
  TSR_CUDA(cudaGetLastError());
  TSR_CUDA(cudaStreamSynchronize(s));
  scratch.release();
  out->allocs = keep.ptrs;
  return TSR_OK;
}

void free_csf(CsfDev* c) {
  for (void* p : c->allocs) cudaFree(p);
  c->allocs.clear();
}

// csf.rs:141-156 wording
int check_mode_order(int ndim, const int64_t* mo, int n_mo) {
  if (n_mo != ndim)
    return fail(TSR_E_MODE_ORDER, "Invalid mode order: mode_order length %d != ndim %d", n_mo,
                ndim);
  std::vector<int64_t> s(mo, mo + n_mo);
  std::sort(s.begin(), s.end());
  for (int d = 0; d < ndim; ++d) {
    if (s[d] != d) {
      std::string txt = "[";
      for (int i = 0; i < n_mo; ++i) txt += (i ? ", " : "") + std::to_string(mo[i]);
      txt += "]";
      return fail(TSR_E_MODE_ORDER, "Invalid mode order: mode_order %s is not a permutation of 0..%d",
                  txt.c_str(), ndim);
    }
  }
  return TSR_OK;
}

// coo.rs:101-149 shape checks
int check_shape(int ndim, const int64_t* shape) {
  if (ndim <= 0) return fail(TSR_E_SHAPE, "Invalid shape: Shape cannot be empty");
  if (ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d exceeds the supported %d", ndim, kMaxModes);
  for (int d = 0; d < ndim; ++d)
    if (shape[d] <= 0) return fail(TSR_E_SHAPE, "Invalid shape: Shape cannot contain zeros");
  return TSR_OK;
}

int check_host_bounds(const int64_t* idx, int64_t nnz, int ndim, const int64_t* shape) {
  for (int64_t k = 0; k < nnz; ++k)
    for (int d = 0; d < ndim; ++d) {
      const int64_t v = idx[k * ndim + d];
      if (v < 0 || v >= shape[d]) {
        std::string a = "[", b = "[";
        for (int i = 0; i < ndim; ++i) {
          a += (i ? ", " : "") + std::to_string(idx[k * ndim + i]);
          b += (i ? ", " : "") + std::to_string(shape[i]);
        }
        return fail(TSR_E_INDEX_OOB, "Index out of bounds: index %s] exceeds shape %s]",
                    a.c_str(), b.c_str());
      }
    }
  return TSR_OK;
}

// ---------------------------------------------------------------------------
// CSF MTTKRP, 3-way (the CSF rooted at the output mode).
struct Csf3Args {
  const uint32_t* root_ids;
  const uint32_t* root_ptr;
  const uint32_t* fib_ids;
  const uint32_t* fib_ptr;
  const uint32_t* leaf_ids;
  const float* vals;
  const uint32_t* chunk_root;
  const uint32_t* chunk_fiber;
  int64_t chunk_nnz, n_chunks, nnz, n_roots, n_fibers;
  const float* Ua;  // level-1 factor
  const float* Ub;  // leaf factor
  int R;
  double* M;        // FP64 output accumulator (rows of the root mode)
};

// One warp owns a task of 1024 consecutive entries and walks it in batches
// of BS entries (BS <= 32):
//   - lane-parallel loads fetch the batch's leaf row offsets and values and
//     the ends/ids of the next 32 fibers and roots (one batch ahead);
//   - fiber and root ends inside the batch become warp-uniform bit masks
//     (__reduce_or_sync);
//   - lanes form SLOTS = 32 / (R/4) groups of R/4 lanes, each lane holding a
//     float4 of columns, so one step covers SLOTS entries; the batch's leaf
//     rows and fiber (level-1) rows are loaded into registers with 128-bit
//     loads, all in flight together before the first is used (the fiber of
//     an entry is the popcount of the fiber-end mask below it);
//   - every entry adds value * leaf row (*) its fiber's row to the open root
//     sum, with no branch per entry;
//   - at a root end (or the task end) the slots' partial sums are combined by
//     shuffles and added to the output row with float4 atomics, the only
//     atomics in the kernel.
// The per-entry form equals the fiber-factored form of the reference's
// MTTKRP definition (sum over entries of v * prod of factor rows); only the
// fp32 summation order differs.
constexpr int CSF_WARPS = 8;

struct BatchMeta {
  uint32_t off;  // leaf row offset (leaf id * R / 4, float4 units) of entry k + lane
  float val;
  uint32_t fend, fid;  // end offset and level-1 id of fiber f + lane
  uint32_t rend, rid;  // end offset and id of root s + lane
};

__device__ __forceinline__ BatchMeta load_meta(const Csf3Args& a, uint32_t k, int n, uint32_t f,
                                               uint32_t s, int lane) {
  BatchMeta m;
  const bool e = lane < n;
  m.off = e ? __ldg(a.leaf_ids + k + lane) * (uint32_t)(a.R / 4) : 0u;
  m.val = e ? __ldg(a.vals + k + lane) : 0.f;
  const bool fv = f + lane < (uint32_t)a.n_fibers;
  m.fend = fv ? __ldg(a.fib_ptr + f + lane + 1) : 0xffffffffu;
  m.fid = fv ? __ldg(a.fib_ids + f + lane) : 0u;
  const bool rv = s + lane < (uint32_t)a.n_roots;
  m.rend = rv ? __ldg(a.root_ptr + s + lane + 1) : 0xffffffffu;
  m.rid = rv ? __ldg(a.root_ids + s + lane) : 0u;
  return m;
}

template <int R>
struct CsfSlots {
  static constexpr int LPR = R / 4;           // lanes per factor row (float4 each)
  static constexpr int SLOTS = 32 / LPR;      // entries per step
  static constexpr int STEPS = 32 / SLOTS < 8 ? 32 / SLOTS : 8;  // steps per batch
  static constexpr int BS = SLOTS * STEPS;    // entries per batch (<= 32)
};

// Sum the per-slot partial root sums of the lanes that share a column quad
// and add them to output row `rid` (slot-0 lanes issue the atomics).
template <int R>
__device__ __forceinline__ void csf_flush(float4& acc, uint32_t rid, int lane, double* M) {
  constexpr int LPR = CsfSlots<R>::LPR;
#pragma unroll
  for (int o = LPR; o < 32; o <<= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
    acc.z += __shfl_xor_sync(0xffffffffu, acc.z, o);
    acc.w += __shfl_xor_sync(0xffffffffu, acc.w, o);
  }
  if (lane < LPR) {
    // FP64 accumulation: heavy (Zipf-head) rows receive many task sums
    double* o = M + (size_t)rid * R + 4 * lane;
    atomicAdd(o + 0, (double)acc.x);
    atomicAdd(o + 1, (double)acc.y);
    atomicAdd(o + 2, (double)acc.z);
    atomicAdd(o + 3, (double)acc.w);
  }
  acc = make_float4(0.f, 0.f, 0.f, 0.f);
}

__device__ __forceinline__ void fma4(float4& acc, float v, const float4& u, const float4& x) {
  acc.x = fmaf(v * u.x, x.x, acc.x);
  acc.y = fmaf(v * u.y, x.y, acc.y);
  acc.z = fmaf(v * u.z, x.z, acc.z);
  acc.w = fmaf(v * u.w, x.w, acc.w);
}

template <int R>
__global__ void __launch_bounds__(CSF_WARPS * 32, 2)
csf3_slot_kernel(Csf3Args a, int chunks_per_task) {
  using S = CsfSlots<R>;
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int LPR = S::LPR, SLOTS = S::SLOTS, STEPS = S::STEPS, BS = S::BS;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int es = lane / LPR, cq = lane % LPR;  // entry slot, column quad
  const float4* ub_lane = reinterpret_cast<const float4*>(a.Ub) + cq;
  const float4* ua_lane = reinterpret_cast<const float4*>(a.Ua) + cq;
  constexpr uint32_t R4 = R / 4;  // float4 per row
  const uint32_t nnz = (uint32_t)a.nnz;
  const uint32_t n_tasks = (uint32_t)((a.n_chunks + chunks_per_task - 1) / chunks_per_task);
  for (uint32_t task = blockIdx.x * CSF_WARPS + warp; task < n_tasks;
       task += gridDim.x * CSF_WARPS) {
    const uint32_t c = task * (uint32_t)chunks_per_task;
    uint32_t k = c * (uint32_t)a.chunk_nnz;
    const uint32_t kend = min(k + (uint32_t)(chunks_per_task * a.chunk_nnz), nnz);
    uint32_t f = a.chunk_fiber[c];
    uint32_t s = a.chunk_root[c];
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t n = min((uint32_t)BS, kend - k);
    BatchMeta cur = load_meta(a, k, (int)n, f, s, lane);
    while (k < kend) {
      // entry k + j ends a fiber / root  <=>  bit j of fmask / rmask
      const uint32_t fb = (cur.fend > k && cur.fend <= k + n) ? 1u << (cur.fend - k - 1) : 0u;
      const uint32_t rb = (cur.rend > k && cur.rend <= k + n) ? 1u << (cur.rend - k - 1) : 0u;
      const uint32_t fmask = __reduce_or_sync(FULL, fb);
      const uint32_t rmask = __reduce_or_sync(FULL, rb);
      // entry lane j: its fiber is the number of fiber ends before j; its
      // fiber row offset (float4 units) comes from that fiber's lane
      const uint32_t fi_l = __popc(fmask & ((1u << lane) - 1u));
      const uint32_t fo_l = __shfl_sync(FULL, cur.fid, fi_l) * R4;
      // leaf rows and fiber rows of the batch, all loads in flight together
      float4 x[STEPS], u[STEPS];
      float v[STEPS];
      if (n == (uint32_t)BS) {
#pragma unroll
        for (int st = 0; st < STEPS; ++st) {
          const int j = st * SLOTS + es;
          x[st] = __ldg(ub_lane + __shfl_sync(FULL, cur.off, j));
          u[st] = __ldg(ua_lane + __shfl_sync(FULL, fo_l, j));
          v[st] = __shfl_sync(FULL, cur.val, j);
        }
      } else {
#pragma unroll
        for (int st = 0; st < STEPS; ++st) {
          const int j = st * SLOTS + es;
          const uint32_t xo = __shfl_sync(FULL, cur.off, j);
          const uint32_t uo = __shfl_sync(FULL, fo_l, j);
          v[st] = __shfl_sync(FULL, cur.val, j);  // 0 past n
          x[st] = u[st] = make_float4(0.f, 0.f, 0.f, 0.f);
          if ((uint32_t)j < n) {
            x[st] = __ldg(ub_lane + xo);
            u[st] = __ldg(ua_lane + uo);
          }
        }
      }
      // next batch's metadata while the rows are in flight
      const uint32_t kn = k + n;
      const uint32_t fn = f + __popc(fmask);
      const uint32_t sn = s + __popc(rmask);
      const uint32_t nn = min((uint32_t)BS, kend - kn);
      BatchMeta nxt = cur;
      if (kn < kend) nxt = load_meta(a, kn, (int)nn, fn, sn, lane);
      int ri = 0;
      if (rmask == 0u) {
#pragma unroll
        for (int st = 0; st < STEPS; ++st) fma4(acc, v[st], u[st], x[st]);
      } else {
        // root ends inside the batch: add and flush segment by segment
#pragma unroll
        for (int st = 0; st < STEPS; ++st) {
          uint32_t rs = (rmask >> (st * SLOTS)) & ((SLOTS < 32 ? (1u << SLOTS) : 0u) - 1u);
          int lo = 0;
          while (rs) {
            const int e = __ffs(rs) - 1;
            rs &= rs - 1u;
            if (es >= lo && es <= e) fma4(acc, v[st], u[st], x[st]);
            csf_flush<R>(acc, __shfl_sync(FULL, cur.rid, ri), lane, a.M);
            ++ri;
            lo = e + 1;
          }
          if (es >= lo) fma4(acc, v[st], u[st], x[st]);
        }
      }
      // task end: the open root's sum
      if (kn == kend && !((rmask >> (n - 1)) & 1u))
        csf_flush<R>(acc, __shfl_sync(FULL, cur.rid, ri), lane, a.M);
      k = kn;
      f = fn;
      s = sn;
      n = nn;
      cur = nxt;
    }
  }
}

// Any number of modes and any rank: one thread per (entry, column). The
// entry's indices come from its sorted key.
struct CsfGenArgs {
  const uint64_t* keys;
  const float* vals;
  int64_t nnz;
  KeySpec ks;
  int root_mode;
  const float* U[kMaxModes];
  int R;
  double* M;
};

__global__ void csf_generic_mttkrp_kernel(CsfGenArgs a) {
  const int64_t total = a.nnz * a.R;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = t / a.R;
    const int r = (int)(t % a.R);
    uint64_t key = a.keys[k];
    float prod = a.vals[k];
    int64_t root = 0;
    for (int l = a.ks.ndim - 1; l >= 0; --l) {
      const int m = a.ks.mo[l];
      const int64_t i = (int64_t)(key % (uint64_t)a.ks.shape[m]);
      key /= (uint64_t)a.ks.shape[m];
      if (m == a.root_mode)
        root = i;
      else
        prod *= a.U[m][i * a.R + r];
    }
    atomicAdd(a.M + root * a.R + r, (double)prod);
  }
}

__global__ void f64_to_f32_kernel(const double* __restrict__ in, int64_t n, float* __restrict__ out) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    out[e] = (float)in[e];
}

template <int R>
void launch_csf3_slot(tsr_ctx* ctx, cudaStream_t s, const Csf3Args& a) {
  constexpr int kChunksPerTask = 4;  // 1024 entries per warp task
  const int64_t tasks = ceil_div(a.n_chunks, kChunksPerTask);
  const int64_t blocks = ceil_div(tasks, CSF_WARPS);
  const int64_t cap = (int64_t)std::max(1, ctx->sm_count - ctx->reserve_sms) * 2;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min(blocks, cap));
  csf3_slot_kernel<R><<<grid, CSF_WARPS * 32, 0, s>>>(a, kChunksPerTask);
}


}  // namespace

int coo_check_shape(int ndim, const int64_t* shape) { return check_shape(ndim, shape); }
int coo_check_bounds(const int64_t* idx, int64_t nnz, int ndim, const int64_t* shape) {
  return check_host_bounds(idx, nnz, ndim, shape);
}

void init_csf_attributes() {}  // the CSF kernels use no dynamic shared memory

int launch_csf_accumulate(tsr_ctx* ctx, cudaStream_t s, const tsr_sparse* sp,
                          const FactorTable& ft, int R, int mode, double* d_out);

int launch_mttkrp_csf(tsr_ctx* ctx, cudaStream_t s, const tsr_sparse* sp, const FactorTable& ft,
                      int R, int mode, float* d_out, double* d_acc) {
  const CsfDev& c = sp->modes[mode];
  const int64_t n_out = sp->shape[mode] * R;
  if (c.nnz == 0) {
    TSR_CUDA(cudaMemsetAsync(d_out, 0, sizeof(float) * n_out, s));
    return TSR_OK;
  }
  TSR_CUDA(cudaMemsetAsync(d_acc, 0, sizeof(double) * n_out, s));
  TSR_TRY(launch_csf_accumulate(ctx, s, sp, ft, R, mode, d_acc));
  f64_to_f32_kernel<<<grid_for(ctx, n_out), 256, 0, s>>>(d_acc, n_out, d_out);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_csf_accumulate(tsr_ctx* ctx, cudaStream_t s, const tsr_sparse* sp,
                          const FactorTable& ft, int R, int mode, double* d_out) {
  const CsfDev& c = sp->modes[mode];
  bool vec = R % 4 == 0 && R <= 128 && ((uintptr_t)d_out & 15) == 0;
  for (int m = 0; m < c.ndim && vec; ++m) vec = ((uintptr_t)ft.ptr[m] & 15) == 0;
  if (c.ndim == 3 && vec) {
    Csf3Args a;
    a.root_ids = c.level_ids[0];
    a.root_ptr = c.level_ptr[0];
    a.fib_ids = c.level_ids[1];
    a.fib_ptr = c.level_ptr[1];
    a.leaf_ids = c.level_ids[2];
    a.vals = c.vals;
    a.chunk_root = c.chunk_root;
    a.chunk_fiber = c.chunk_fiber;
    a.chunk_nnz = c.chunk_nnz;
    a.n_chunks = c.n_chunks;
    a.nnz = c.nnz;
    a.n_roots = c.level_len[0];
    a.n_fibers = c.level_len[1];
    a.Ua = ft.ptr[c.mode_order[1]];
    a.Ub = ft.ptr[c.mode_order[2]];
    a.R = R;
    a.M = d_out;
    // rows of a factor are addressed with 32-bit element offsets
    bool fast = R == 4 || R == 8 || R == 16 || R == 32 || R == 64 || R == 128;
    for (int l = 1; l < 3 && fast; ++l)
      fast = (uint64_t)sp->shape[c.mode_order[l]] * (uint64_t)R < 0xffffffffull;
    if (fast) {
      switch (R) {
        case 4: launch_csf3_slot<4>(ctx, s, a); break;
        case 8: launch_csf3_slot<8>(ctx, s, a); break;
        case 16: launch_csf3_slot<16>(ctx, s, a); break;
        case 32: launch_csf3_slot<32>(ctx, s, a); break;
        case 64: launch_csf3_slot<64>(ctx, s, a); break;
        default: launch_csf3_slot<128>(ctx, s, a); break;
      }
      ctx->launches++;
      TSR_CUDA(cudaGetLastError());
      return TSR_OK;
    }
  }
  CsfGenArgs g;
  g.keys = c.keys;
  g.vals = c.vals;
  g.nnz = c.nnz;
  TSR_TRY(make_keyspec(c.ndim, c.shape, c.mode_order, &g.ks));
  g.root_mode = mode;
  for (int m = 0; m < c.ndim; ++m) g.U[m] = ft.ptr[m];
  g.R = R;
  g.M = d_out;
  csf_generic_mttkrp_kernel<<<grid_for(ctx, c.nnz * R), 256, 0, s>>>(g);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int sparse_sumsq(tsr_ctx* ctx, cudaStream_t s, const tsr_sparse* sp, double* d_out) {
  const CsfDev& c = sp->modes[0];
  if (c.nnz == 0) return TSR_OK;
  sumsq_kernel<<<grid_for(ctx, c.nnz), 256, 0, s>>>(c.vals, c.nnz, d_out);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

}  // namespace tsr

using namespace tsr;

namespace {

// Upload host COO (AoS int64) to a device scratch buffer.
int upload_coo(tsr_ctx* ctx, const int64_t* idx, const float* vals, int64_t nnz, int ndim,
               int64_t** d_idx, float** d_vals) {
  void *a, *b;
  TSR_TRY(slot_get(ctx, SLOT_SPARSE0, sizeof(int64_t) * std::max<int64_t>(nnz, 1) * ndim, &a));
  TSR_TRY(slot_get(ctx, SLOT_SPARSE0 + 1, sizeof(float) * std::max<int64_t>(nnz, 1), &b));
  if (nnz > 0) {
    TSR_CUDA(cudaMemcpyAsync(a, idx, sizeof(int64_t) * nnz * ndim, cudaMemcpyHostToDevice,
                             ctx->stream));
    TSR_CUDA(cudaMemcpyAsync(b, vals, sizeof(float) * nnz, cudaMemcpyHostToDevice, ctx->stream));
  }
  *d_idx = (int64_t*)a;
  *d_vals = (float*)b;
  return TSR_OK;
}

// coo.rs:239-257 (sort) and :320-347 (deduplicate) on device arrays; the
// result (sorted, optionally merged) overwrites the first *nnz_out entries.
int coo_sort_dedup_dev(tsr_ctx* ctx, int64_t* d_idx, float* d_vals, int64_t nnz, int ndim,
                       const int64_t* shape, bool dedup, int64_t* nnz_out) {
  if (nnz_out) *nnz_out = nnz;
  if (nnz <= 1) return TSR_OK;  // deduplicate returns early (coo.rs:321-323)
  if (nnz >= (int64_t)INT32_MAX) return fail(TSR_E_UNSUPPORTED, "more than 2^31 - 1 entries");
  cudaStream_t s = ctx->stream;
  int mo[kMaxModes];
  for (int d = 0; d < ndim; ++d) mo[d] = d;
  KeySpec ks;
  TSR_TRY(make_keyspec(ndim, shape, mo, &ks));
  Arena ar;
  uint64_t* keys;
  uint32_t* pos;
  int rc = sort_entries(ctx, s, ar, d_idx, nnz, ks, key_bits(ndim, shape), &keys, &pos);
  if (rc == TSR_OK) {
    uint32_t* heads = nullptr;
    int64_t count = nnz;
    if (dedup)
      rc = level_fibers(ctx, s, ar, ar, keys, nnz, 1, UINT64_MAX, &heads, nullptr, &count);
    float* vout = nullptr;
    if (rc == TSR_OK) rc = ar.get(&vout, count);
    if (rc == TSR_OK) {
      if (dedup)
        segment_sum_kernel<<<grid_for(ctx, count), 256, 0, s>>>(heads, count, nnz, pos, d_vals,
                                                                vout);
      else
        leaf_kernel<<<grid_for(ctx, nnz), 256, 0, s>>>(keys, pos, d_vals, nnz, 1, nullptr, vout);
      decode_kernel<<<grid_for(ctx, count), 256, 0, s>>>(keys, heads, count, ks, d_idx);
      ctx->launches += 2;
      cudaError_t e = cudaMemcpyAsync(d_vals, vout, sizeof(float) * count,
                                      cudaMemcpyDeviceToDevice, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) rc = fail(TSR_E_CUDA, "%s", cudaGetErrorString(e));
      if (nnz_out) *nnz_out = count;
    }
  }
  ar.release();
  return rc;
}

int coo_sort_dedup(tsr_ctx* ctx, int64_t* idx, float* vals, int64_t nnz, int ndim,
                   const int64_t* shape, bool dedup, int64_t* nnz_out) {
  TSR_TRY(check_shape(ndim, shape));
  TSR_TRY(check_host_bounds(idx, nnz, ndim, shape));
  if (nnz_out) *nnz_out = nnz;
  if (nnz <= 1) return TSR_OK;
  TSR_TRY(check_ctx(ctx));
  int64_t* d_idx;
  float* d_vals;
  TSR_TRY(upload_coo(ctx, idx, vals, nnz, ndim, &d_idx, &d_vals));
  int64_t count = nnz;
  TSR_TRY(coo_sort_dedup_dev(ctx, d_idx, d_vals, nnz, ndim, shape, dedup, &count));
  TSR_CUDA(cudaMemcpyAsync(idx, d_idx, sizeof(int64_t) * count * ndim, cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaMemcpyAsync(vals, d_vals, sizeof(float) * count, cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  if (nnz_out) *nnz_out = count;
  return TSR_OK;
}

int copy_level_u32_to_i64(const uint32_t* d, int64_t n, int64_t* host) {
  std::vector<uint32_t> tmp(n);
  if (n > 0) TSR_CUDA(cudaMemcpy(tmp.data(), d, 4 * n, cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < n; ++i) host[i] = tmp[i];
  return TSR_OK;
}

}  // namespace

extern "C" {

int tsr_coo_sort_f32(tsr_ctx* ctx, int64_t* indices, float* values, int64_t nnz, int ndim,
                     const int64_t* shape) {
  if (!shape || (nnz > 0 && (!indices || !values))) return fail(TSR_E_INVALID_ARG, "null argument");
  return coo_sort_dedup(ctx, indices, values, nnz, ndim, shape, false, nullptr);
}

int tsr_coo_deduplicate_f32(tsr_ctx* ctx, int64_t* indices, float* values, int64_t nnz,
                            int ndim, const int64_t* shape, int64_t* nnz_out) {
  if (!shape || !nnz_out || (nnz > 0 && (!indices || !values)))
    return fail(TSR_E_INVALID_ARG, "null argument");
  return coo_sort_dedup(ctx, indices, values, nnz, ndim, shape, true, nnz_out);
}

int tsr_csf_from_coo_f32(tsr_ctx* ctx, const int64_t* indices, const float* values, int64_t nnz,
                         int ndim, const int64_t* shape, const int64_t* mode_order,
                         int n_mode_order, int64_t* fptr, int64_t* fids, float* vals_out,
                         int64_t* lens) {
  if (!shape || !mode_order || !fptr || !fids || !lens || (nnz > 0 && (!indices || !values)))
    return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(check_shape(ndim, shape));
  TSR_TRY(check_mode_order(ndim, mode_order, n_mode_order));
  TSR_TRY(check_host_bounds(indices, nnz, ndim, shape));
  const int64_t W = nnz + 1;
  if (nnz == 0) {  // csf.rs:158-168
    for (int l = 0; l < ndim; ++l) {
      fptr[l * W] = 0;
      lens[2 * l] = 1;
      lens[2 * l + 1] = 0;
    }
    return TSR_OK;
  }
  if (nnz >= (int64_t)INT32_MAX) return fail(TSR_E_UNSUPPORTED, "more than 2^31 - 1 entries");
  TSR_TRY(check_ctx(ctx));
  int64_t* d_idx;
  float* d_vals;
  TSR_TRY(upload_coo(ctx, indices, values, nnz, ndim, &d_idx, &d_vals));
  int mo[kMaxModes];
  for (int l = 0; l < ndim; ++l) mo[l] = (int)mode_order[l];
  CsfDev c;
  int rc = build_csf(ctx, ctx->stream, d_idx, d_vals, nnz, ndim, shape, mo, false, &c);
  if (rc != TSR_OK) return rc;
  const int nlev = ndim == 1 ? 1 : ndim - 1;
  for (int l = 0; l < nlev && rc == TSR_OK; ++l) {
    rc = copy_level_u32_to_i64(c.level_ptr[l], c.level_len[l] + 1, fptr + l * W);
    if (rc == TSR_OK) rc = copy_level_u32_to_i64(c.level_ids[l], c.level_len[l], fids + l * nnz);
    lens[2 * l] = c.level_len[l] + 1;
    lens[2 * l + 1] = c.level_len[l];
  }
  if (ndim > 1 && rc == TSR_OK) {
    const int L = ndim - 1;
    std::copy(fptr + (L - 1) * W, fptr + (L - 1) * W + lens[2 * (L - 1)], fptr + L * W);
    lens[2 * L] = lens[2 * (L - 1)];
    rc = copy_level_u32_to_i64(c.level_ids[L], nnz, fids + L * nnz);
    lens[2 * L + 1] = nnz;
    if (rc == TSR_OK && vals_out)
      if (cudaMemcpy(vals_out, c.vals, sizeof(float) * nnz, cudaMemcpyDeviceToHost) !=
          cudaSuccess)
        rc = fail(TSR_E_CUDA, "copy of values failed");
  }
  // ndim == 1: the reference leaves vals empty (its leaf branch never runs)
  free_csf(&c);
  return rc;
}

static int sparse_create(tsr_ctx* ctx, const int64_t* d_idx, const float* d_vals, int64_t nnz,
                         int ndim, const int64_t* shape, tsr_sparse** out) {
  tsr_sparse* sp = new tsr_sparse();
  sp->device = ctx->device;
  sp->ndim = ndim;
  sp->nnz = nnz;
  for (int d = 0; d < ndim; ++d) sp->shape[d] = shape[d];
  for (int n = 0; n < ndim; ++n) {
    // root = n; the other modes follow in ascending size (ties by mode index)
    int mo[kMaxModes];
    mo[0] = n;
    int k = 1;
    for (int m = 0; m < ndim; ++m)
      if (m != n) mo[k++] = m;
    std::stable_sort(mo + 1, mo + ndim, [&](int x, int y) { return shape[x] < shape[y]; });
    int rc = build_csf(ctx, ctx->stream, d_idx, d_vals, nnz, ndim, shape, mo, true, &sp->modes[n]);
    if (rc != TSR_OK) {
      for (int m = 0; m < n; ++m) free_csf(&sp->modes[m]);
      delete sp;
      return rc;
    }
  }
  double* dsum;
  TSR_CUDA(cudaMalloc(&dsum, sizeof(double)));
  TSR_CUDA(cudaMemsetAsync(dsum, 0, sizeof(double), ctx->stream));
  TSR_TRY(sparse_sumsq(ctx, ctx->stream, sp, dsum));
  TSR_CUDA(cudaMemcpyAsync(&sp->norm_sq, dsum, sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  cudaFree(dsum);
  *out = sp;
  return TSR_OK;
}

int tsr_sparse_create_f32(tsr_ctx* ctx, const int64_t* indices, const float* values, int64_t nnz,
                          int ndim, const int64_t* shape, tsr_sparse** out) {
  if (!shape || !out || (nnz > 0 && (!indices || !values)))
    return fail(TSR_E_INVALID_ARG, "null argument");
  *out = nullptr;
  TSR_TRY(check_shape(ndim, shape));
  TSR_TRY(check_host_bounds(indices, nnz, ndim, shape));
  if (nnz >= (int64_t)INT32_MAX) return fail(TSR_E_UNSUPPORTED, "more than 2^31 - 1 entries");
  for (int d = 0; d < ndim; ++d)
    if (shape[d] >= (int64_t)UINT32_MAX) return fail(TSR_E_UNSUPPORTED, "mode size >= 2^32");
  TSR_TRY(check_ctx(ctx));
  int64_t* d_idx;
  float* d_vals;
  TSR_TRY(upload_coo(ctx, indices, values, nnz, ndim, &d_idx, &d_vals));
  return sparse_create(ctx, d_idx, d_vals, nnz, ndim, shape, out);
}

int tsr_sparse_create_dev_f32(tsr_ctx* ctx, const int64_t* d_indices, const float* d_values,
                              int64_t nnz, int ndim, const int64_t* shape, tsr_sparse** out) {
  if (!shape || !out || (nnz > 0 && (!d_indices || !d_values)))
    return fail(TSR_E_INVALID_ARG, "null argument");
  *out = nullptr;
  TSR_TRY(check_shape(ndim, shape));
  if (nnz >= (int64_t)INT32_MAX) return fail(TSR_E_UNSUPPORTED, "more than 2^31 - 1 entries");
  for (int d = 0; d < ndim; ++d)
    if (shape[d] >= (int64_t)UINT32_MAX) return fail(TSR_E_UNSUPPORTED, "mode size >= 2^32");
  TSR_TRY(check_ctx(ctx));
  return sparse_create(ctx, d_indices, d_values, nnz, ndim, shape, out);
}

int tsr_coo_deduplicate_dev_f32(tsr_ctx* ctx, int64_t* d_indices, float* d_values, int64_t nnz,
                                int ndim, const int64_t* shape, int64_t* nnz_out) {
  if (!shape || !nnz_out || (nnz > 0 && (!d_indices || !d_values)))
    return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(check_shape(ndim, shape));
  TSR_TRY(check_ctx(ctx));
  return coo_sort_dedup_dev(ctx, d_indices, d_values, nnz, ndim, shape, true, nnz_out);
}

int tsr_sparse_destroy(tsr_sparse* sp) {
  if (!sp) return TSR_OK;
  cudaSetDevice(sp->device);
  cudaDeviceSynchronize();
  for (int n = 0; n < sp->ndim; ++n) free_csf(&sp->modes[n]);
  delete sp;
  return TSR_OK;
}

int tsr_sparse_info(const tsr_sparse* sp, int mode, int64_t* nnz, int64_t* n_roots,
                    int64_t* n_fibers) {
  if (!sp || mode < 0 || mode >= sp->ndim) return fail(TSR_E_INVALID_ARG, "invalid argument");
  if (nnz) *nnz = sp->nnz;
  if (n_roots) *n_roots = sp->modes[mode].level_len[0];
  if (n_fibers) *n_fibers = sp->ndim >= 3 ? sp->modes[mode].level_len[1] : 0;
  return TSR_OK;
}

int tsr_mttkrp_csf_dev_f32(tsr_ctx* ctx, const tsr_sparse* sp, const float* const* d_factors,
                           int64_t rank, int mode, float* d_out) {
  if (!sp || !d_factors || !d_out) return fail(TSR_E_INVALID_ARG, "null argument");
  if (mode < 0 || mode >= sp->ndim)
    return fail(TSR_E_MODE_OOB, "Mode %d out of bounds for tensor with rank %d", mode, sp->ndim);
  if (sp->ndim < 2) return fail(TSR_E_NEED_2_FACTORS, "Need at least 2 factor matrices for MTTKRP");
  if (rank <= 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  TSR_TRY(check_ctx(ctx));
  FactorTable ft{};
  for (int m = 0; m < sp->ndim; ++m) {
    ft.ptr[m] = d_factors[m];
    ft.rows[m] = sp->shape[m];
  }
  void* acc;
  TSR_TRY(slot_get(ctx, SLOT_MISC1, sizeof(double) * sp->shape[mode] * rank, &acc));
  return launch_mttkrp_csf(ctx, ctx->stream, sp, ft, (int)rank, mode, d_out, (double*)acc);
}

int tsr_mttkrp_csf_f32(tsr_ctx* ctx, const tsr_sparse* sp, const float* const* factors,
                       int64_t rank, int mode, float* out) {
  if (!sp || !factors || !out) return fail(TSR_E_INVALID_ARG, "null argument");
  if (mode < 0 || mode >= sp->ndim)
    return fail(TSR_E_MODE_OOB, "Mode %d out of bounds for tensor with rank %d", mode, sp->ndim);
  TSR_TRY(check_ctx(ctx));
  int64_t total = 0;
  for (int m = 0; m < sp->ndim; ++m) total += sp->shape[m] * rank;
  void *df, *dout;
  TSR_TRY(slot_get(ctx, SLOT_FACTORS, sizeof(float) * total, &df));
  TSR_TRY(slot_get(ctx, SLOT_OUT, sizeof(float) * sp->shape[mode] * rank, &dout));
  const float* ptrs[kMaxModes];
  float* p = (float*)df;
  for (int m = 0; m < sp->ndim; ++m) {
    TSR_CUDA(cudaMemcpyAsync(p, factors[m], sizeof(float) * sp->shape[m] * rank,
                             cudaMemcpyHostToDevice, ctx->stream));
    ptrs[m] = p;
    p += sp->shape[m] * rank;
  }
  TSR_TRY(tsr_mttkrp_csf_dev_f32(ctx, sp, ptrs, rank, mode, (float*)dout));
  TSR_CUDA(cudaMemcpyAsync(out, dout, sizeof(float) * sp->shape[mode] * rank,
                           cudaMemcpyDeviceToHost, ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

int tsr_profile_mttkrp_csf_dev_f32(tsr_ctx* ctx, const tsr_sparse* sp,
                                   const float* const* d_factors, int64_t rank, int mode,
                                   int iters, int flush_l2, double* ms_per_launch) {
  if (!sp || !d_factors || !ms_per_launch || iters <= 0)
    return fail(TSR_E_INVALID_ARG, "invalid argument");
  TSR_TRY(check_ctx(ctx));
  void* dout;
  TSR_TRY(slot_get(ctx, SLOT_OUT, sizeof(float) * sp->shape[mode] * rank, &dout));
  cudaEvent_t a, b;
  TSR_CUDA(cudaEventCreate(&a));
  TSR_CUDA(cudaEventCreate(&b));
  double total = 0.0;
  for (int i = 0; i < iters; ++i) {
    if (flush_l2) TSR_TRY(::tsr::flush_l2(ctx, ctx->stream));
    TSR_CUDA(cudaEventRecord(a, ctx->stream));
    TSR_TRY(tsr_mttkrp_csf_dev_f32(ctx, sp, d_factors, rank, mode, (float*)dout));
    TSR_CUDA(cudaEventRecord(b, ctx->stream));
    TSR_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    TSR_CUDA(cudaEventElapsedTime(&ms, a, b));
    total += ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms_per_launch = total / iters;
  return TSR_OK;
}

}  // extern "C"

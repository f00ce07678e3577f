// Dense 3-way MTTKRP, BF16x3 tensor cores, on one resident copy of the tensor.
//
// X (I x J x K, row-major, K fastest) is split once into bf16 halves
// x = hi + lo (exact to 2^-16) kept in X's own layout. Every mode reads that
// one copy through a mode-specific TMA box, so within a CP-ALS sweep the three
// MTTKRPs stream the same 64 MiB (at 256^3) and it can stay resident in the
// 126 MB L2 from one mode to the next, instead of one unfolding per mode.
//
// Each MTTKRP is a sum over runs P of a small contraction scaled column-wise
// by the run's weight row w_P (the factor of the remaining mode):
//   mode 0: M0 = sum_j (X[:, j, :] . U2) diag(U1[j, :])   rows i, contract k
//   mode 1: M1 = sum_i (X[i, :, :] . U2) diag(U0[i, :])   rows j, contract k
//   mode 2: M2 = sum_i (X[i, :, :]^T . U1) diag(U0[i, :]) rows k, contract j
// In modes 0 and 1 the A tile (128 rows x 64 contracted) is K-major; in mode 2
// its rows are the contiguous k, so it is loaded and consumed MN-major. This
// is the same sum as the unfolded product X_(n) . KR of mttkrp.rs:125-143, with
// the Khatri-Rao rows factored as (weight row) x (contracted factor row).
//
// The contracted factor U (L x R, R <= 64) enters as a prebuilt bf16 hi/lo
// "B image" in global memory: per 64-row k-block, a [2 n_pad][64] K-major tile
// with the 128-byte swizzle, rows 0..n_pad-1 the hi halves of U's columns and
// rows n_pad..2 n_pad-1 the lo halves. The CP-ALS solve that updates U writes
// it, so a CTA fetches it with one bulk copy instead of converting U itself.
// Per 16-wide k-slice two MMAs of N = 2 n_pad accumulate into one TMEM
// accumulator:
//   D += Xhi . [Uhi | Ulo],  D += Xlo . [Uhi | Ulo]
// so D[:, n] + D[:, n_pad + n] = (Xhi + Xlo) . (Uhi + Ulo) column n: every
// product of the split values, the lo.lo term included.
//
// Per CTA: one 128-row M tile and a range of whole runs (split-K).
//   warp 0      TMA producer: the A tiles of every run (hi and lo, 128-byte
//               swizzle, evict-last L2 policy) into a ring of stages; it
//               starts before the programmatic-launch wait (X is written before
//               the sweep).
//   warp 1      TMEM allocation and the MMA-issuing thread; accumulators are
//               double buffered across runs.
//   warps 2..5  after the wait: the B image (bulk copy) and the runs' weights,
//               then per run the epilogue: TMEM -> registers, (hh + cr) . w_P
//               accumulated in fp32; finally the split-K partial rows.
// Every mbarrier wait is bounded; a wait that runs out raises DS_TIMEOUT and
// the CTA drains its copies, waits for its MMAs and frees TMEM before exiting.
#include <algorithm>
#include <mutex>
#include <vector>

#include "mttkrp.cuh"
#include "sm100.cuh"

namespace tsr {

namespace {

constexpr int M3_BM = 128;
constexpr int M3_BK = 64;
constexpr int M3_THREADS = 192;
constexpr int M3_A_TILE = M3_BM * M3_BK * 2;  // 16 KB per half
constexpr int M3_MAX_RUNS = 16;
constexpr int M3_MAX_L = 384;
constexpr long long M3_DRAIN_BUDGET = 1ll << 31;  // ~1 s at B200 clocks
constexpr int kM3MaxSmem = 227 * 1024;

struct M3Params {
  int mode;             // 0, 1, 2 (box and coordinate layout)
  int64_t rows;         // M: I, J or K
  int64_t runs;         // runs in total: J (mode 0) or I
  int L;                // contracted length: K (modes 0, 1) or J (mode 2)
  int runs_per_split;
  int R;
  int n_pad;            // 32 or 64
  int stages;
  const uint8_t* bimg;  // B image of the contracted factor
  uint32_t bimg_bytes;
  const float* wf;      // weight factor, row = run index, row stride R
  float* partials;      // [splits][rows][R]
  unsigned* status;
  long long wait_budget;  // clock cycles for each pipeline wait
  int a_resident;         // X's halves were written before the preceding kernel
  TraceSlot tr;           // timeline tracing (null pointers when off)
};

__device__ __forceinline__ uint64_t evict_last_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ void tma_load_3d_hint(void* dst, const CUtensorMap* map, int32_t x,
                                                 int32_t y, int32_t z, uint64_t* bar,
                                                 uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%2, %3, %4}], [%5], %6;" ::"r"(sm100::smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(sm100::smem_u32(bar)), "l"(policy)
      : "memory");
}

// Shared-memory descriptor of an MN-major operand with the 128-byte swizzle:
// 64 contiguous MN elements (128 B) per row, 8 rows (K) 1024 B apart (SBO),
// the next 64 MN elements `lbo` bytes on (LBO).
__device__ __forceinline__ uint64_t desc_sw128_mnmajor(uint32_t smem_addr, uint32_t lbo) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr & 0x3FFFF) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

__device__ __forceinline__ bool m3_wait(uint64_t* bar, uint32_t parity, volatile int* abort,
                                        long long budget) {
  return sm100::mbar_wait(bar, parity, abort, budget);
}

__global__ void __launch_bounds__(M3_THREADS, 1)
mttkrp3_kernel(const __grid_constant__ CUtensorMap map_hi,
               const __grid_constant__ CUtensorMap map_lo, M3Params p) {
  using namespace sm100;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
  const int S = p.stages;
  const int spr = (p.L + M3_BK - 1) / M3_BK;             // k-blocks per run
  const uint32_t btile = (uint32_t)(2 * p.n_pad) * 128u;  // one k-block of the B image
  uint8_t* a_base = smem;
  uint8_t* b_base = smem + (size_t)S * 2 * M3_A_TILE;
  float* wts = reinterpret_cast<float*>(b_base + (size_t)spr * btile);  // [runs][64]
  uint64_t* bars = reinterpret_cast<uint64_t*>(wts + M3_MAX_RUNS * 64);
  uint64_t* tma_full = bars;
  uint64_t* empty = bars + S;
  uint64_t* acc_full = bars + 2 * S;       // [2]
  uint64_t* acc_empty = bars + 2 * S + 2;  // [2]
  uint64_t* b_full = bars + 2 * S + 4;
  uint64_t* mma_done = bars + 2 * S + 5;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 6);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t m0 = (int64_t)blockIdx.y * M3_BM;
  const int64_t run0 = (int64_t)blockIdx.x * p.runs_per_split;
  const int64_t left = p.runs - run0;
  const int nruns = left <= 0 ? 0 : (int)(left < p.runs_per_split ? left : p.runs_per_split);
  const int nsteps = nruns * spr;
  const int acc_cols = 2 * p.n_pad;  // one accumulator: hh | cr
  const int tmem_cols = 2 * acc_cols;
  trace_begin(p.tr);
  if (threadIdx.x == 0) grid_dep_trigger();

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&tma_full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 4);
    }
    mbar_init(b_full, 1);
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    fence_barrier_init();
    prefetch_tmap(&map_hi);
    prefetch_tmap(&map_lo);
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, (uint32_t)tmem_cols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // a resident X (written before the preceding kernel, as in a CP-ALS
      // sweep) is streamed before the launch wait
      if (!p.a_resident) grid_dep_wait();
      const uint64_t pol = evict_last_policy();
      int issued_upto = 0;
      for (int it = 0; it < nsteps; ++it) {
        const int s = it % S;
        const uint32_t ph = (uint32_t)(it / S) & 1u;
        if (!m3_wait(&empty[s], ph ^ 1u, abort_flag, p.wait_budget)) {
          *abort_flag = 1;
          atomicOr(p.status, DS_TIMEOUT);
          break;
        }
        uint8_t* st = a_base + (size_t)s * 2 * M3_A_TILE;
        mbar_arrive_expect_tx(&tma_full[s], 2u * M3_A_TILE);
        const int32_t kb = (int32_t)((it % spr) * M3_BK);
        const int32_t run = (int32_t)(run0 + it / spr);
        const int32_t m = (int32_t)m0;
        if (p.mode == 0) {  // box (64 k, 1 j, 128 i)
          tma_load_3d_hint(st, &map_hi, kb, run, m, &tma_full[s], pol);
          tma_load_3d_hint(st + M3_A_TILE, &map_lo, kb, run, m, &tma_full[s], pol);
        } else if (p.mode == 1) {  // box (64 k, 128 j, 1 i)
          tma_load_3d_hint(st, &map_hi, kb, m, run, &tma_full[s], pol);
          tma_load_3d_hint(st + M3_A_TILE, &map_lo, kb, m, run, &tma_full[s], pol);
        } else {  // box (64 k, 64 j, 1 i), two per half: rows m .. m+63, m+64 .. m+127
          tma_load_3d_hint(st, &map_hi, m, kb, run, &tma_full[s], pol);
          tma_load_3d_hint(st + M3_A_TILE / 2, &map_hi, m + 64, kb, run, &tma_full[s], pol);
          tma_load_3d_hint(st + M3_A_TILE, &map_lo, m, kb, run, &tma_full[s], pol);
          tma_load_3d_hint(st + 3 * M3_A_TILE / 2, &map_lo, m + 64, kb, run, &tma_full[s], pol);
        }
        issued_upto = it + 1;
      }
      // drain: every issued copy must have landed before the CTA may exit
      for (int it = issued_upto - S > 0 ? issued_upto - S : 0; it < issued_upto; ++it) {
        const int s = it % S;
        const uint32_t ph = (uint32_t)(it / S) & 1u;
        long long t0 = clock64();
        while (!mbar_try_wait(&tma_full[s], ph) && clock64() - t0 < M3_DRAIN_BUDGET) {
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t amaj = p.mode == 2 ? (1u << 15) : 0u;  // transpose A: MN-major
      const uint32_t idesc = idesc_bf16_f32(M3_BM, 2 * p.n_pad) | amaj;
      bool ok = nruns == 0 || m3_wait(b_full, 0, abort_flag, p.wait_budget);
      for (int r = 0; ok && r < nruns; ++r) {
        const int b = r & 1;
        // buffer b was last used by run r - 2: wait until the epilogue read it
        if (r >= 2 && !m3_wait(&acc_empty[b], (uint32_t)((r >> 1) - 1) & 1u, abort_flag,
                               p.wait_budget)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + (uint32_t)(b * acc_cols);
        for (int sp = 0; sp < spr; ++sp) {
          const int it = r * spr + sp;
          const int s = it % S;
          const uint32_t ph = (uint32_t)(it / S) & 1u;
          if (!m3_wait(&tma_full[s], ph, abort_flag, p.wait_budget)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a_hi = smem_u32(a_base + (size_t)s * 2 * M3_A_TILE);
          const uint32_t a_lo = a_hi + M3_A_TILE;
          const uint32_t bt = smem_u32(b_base) + (uint32_t)sp * btile;
#pragma unroll
          for (int kk = 0; kk < M3_BK / 16; ++kk) {
            uint64_t dah, dal;
            if (p.mode == 2) {  // 16 k-rows of 128 B per slice; MN halves 8 KB apart
              dah = desc_sw128_mnmajor(a_hi + kk * 2048u, M3_A_TILE / 2);
              dal = desc_sw128_mnmajor(a_lo + kk * 2048u, M3_A_TILE / 2);
            } else {  // 16 bf16 = 32 bytes along K within each 128-byte row
              dah = desc_sw128_kmajor(a_hi + kk * 32u);
              dal = desc_sw128_kmajor(a_lo + kk * 32u);
            }
            const uint64_t db = desc_sw128_kmajor(bt + kk * 32u);
            const uint32_t first = (sp == 0 && kk == 0) ? 0u : 1u;
            // both products accumulate into the whole accumulator: an MMA into
            // a column range that only overlaps the previous one serialises the
            // tensor pipe, one into the same range pipelines
            mma_bf16(acc, dah, db, idesc, first);  // Xhi . [Uhi | Ulo]
            mma_bf16(acc, dal, db, idesc, 1u);     // + Xlo . [Uhi | Ulo]
          }
          mma_commit(&empty[s]);
        }
        if (!ok) break;
        mma_commit(&acc_full[b]);
      }
      if (!ok) {
        *abort_flag = 1;
        atomicOr(p.status, DS_TIMEOUT);
      }
      // no MMA may still be running when TMEM is freed (bounded wait)
      mma_commit(mma_done);
      long long t0 = clock64();
      while (!mbar_try_wait(mma_done, 0) && clock64() - t0 < M3_DRAIN_BUDGET) {
      }
    }
  } else {
    // warps 2..5
    const int t = threadIdx.x - 64;
    const int R = p.R;
    grid_dep_wait();  // the factors (and the partials' readers) of the previous kernel
    if (t == 0 && nruns > 0) {
      mbar_arrive_expect_tx(b_full, p.bimg_bytes);
      for (uint32_t off = 0; off < p.bimg_bytes; off += 16384u) {
        const uint32_t n = p.bimg_bytes - off < 16384u ? p.bimg_bytes - off : 16384u;
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(smem_u32(b_base + off)),
            "l"(p.bimg + off), "r"(n), "r"(smem_u32(b_full))
            : "memory");
      }
    }
    // weights: run r of this CTA, columns c .. c+3 (zero beyond R)
    const bool wvec = (R & 3) == 0 && ((uintptr_t)p.wf & 15) == 0;
    for (int e = t; e < M3_MAX_RUNS * 16; e += 128) {
      const int r = e >> 4, c = (e & 15) * 4;
      float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
      if (r < nruns) {
        const float* src = p.wf + (size_t)(run0 + r) * R;
        if (wvec && c < R) {
          w = __ldg(reinterpret_cast<const float4*>(src + c));
        } else {
          w.x = c < R ? __ldg(src + c) : 0.f;
          w.y = c + 1 < R ? __ldg(src + c + 1) : 0.f;
          w.z = c + 2 < R ? __ldg(src + c + 2) : 0.f;
          w.w = c + 3 < R ? __ldg(src + c + 3) : 0.f;
        }
      }
      *reinterpret_cast<float4*>(wts + r * 64 + c) = w;
    }
    asm volatile("bar.sync 1, 128;" ::: "memory");  // the four epilogue warps: weights visible
    const int q = warp & 3;  // TMEM lane quadrant this warp may access
    float acc[64];
#pragma unroll
    for (int n = 0; n < 64; ++n) acc[n] = 0.f;
    bool ok = true;
    for (int r = 0; r < nruns; ++r) {
      const int b = r & 1;
      int w_ok = 1;
      if (lane == 0)
        w_ok = m3_wait(&acc_full[b], (uint32_t)(r >> 1) & 1u, abort_flag, p.wait_budget) ? 1 : 0;
      w_ok = __shfl_sync(0xffffffffu, w_ok, 0);
      if (!w_ok) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * acc_cols);
#pragma unroll
      for (int h = 0; h < 2; ++h) {  // columns 32h .. 32h + 31
        if (32 * h < p.n_pad) {
          uint32_t rh[2][16], rc[2][16];
#pragma unroll
          for (int g = 0; g < 2; ++g) {
            tmem_ld16_nowait(base + (uint32_t)(32 * h + 16 * g), rh[g]);
            tmem_ld16_nowait(base + (uint32_t)(p.n_pad + 32 * h + 16 * g), rc[g]);
          }
          tmem_wait_ld();
#pragma unroll
          for (int g = 0; g < 2; ++g)
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int n = 32 * h + 16 * g + i;
              const float v = __uint_as_float(rh[g][i]) + __uint_as_float(rc[g][i]);
              acc[n] = fmaf(v, wts[r * 64 + n], acc[n]);
            }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[b]);
    }
    // The warp's 32 rows are contiguous in the partials (row stride R): staged
    // through the A ring (every copy into it was consumed by an MMA that
    // completed before the last acc_full) and stored as whole rows, coalesced.
    const int64_t row0 = m0 + q * 32;
    float* out0 = p.partials + (int64_t)blockIdx.x * p.rows * R + row0 * R;
    const int64_t rleft = p.rows - row0;
    const int nrows = rleft <= 0 ? 0 : (int)(rleft < 32 ? rleft : 32);
    if (ok) {
      float* stg = reinterpret_cast<float*>(a_base) + q * (32 * 68);
      fence_proxy_async_smem();
      if ((R & 3) == 0) {
#pragma unroll
        for (int n = 0; n < 64; n += 4)
          if (n < R)
            *reinterpret_cast<float4*>(stg + lane * 68 + n) =
                make_float4(acc[n], acc[n + 1], acc[n + 2], acc[n + 3]);
        __syncwarp();
        const int r4 = R >> 2;
        const int total = nrows * r4;
        float4* o4 = reinterpret_cast<float4*>(out0);
#pragma unroll 4
        for (int f = lane; f < total; f += 32) {
          const int i = f / r4, c4 = f - i * r4;
          o4[f] = *reinterpret_cast<const float4*>(stg + i * 68 + 4 * c4);
        }
      } else {
#pragma unroll
        for (int n = 0; n < 64; ++n)
          if (n < R) stg[lane * 68 + n] = acc[n];
        __syncwarp();
        for (int i = 0; i < nrows; ++i)
          for (int c = lane; c < R; c += 32) out0[(int64_t)i * R + c] = stg[i * 68 + c];
      }
    } else {
      if (lane == 0) atomicOr(p.status, DS_TIMEOUT);
      for (int i = 0; i < nrows; ++i)
        for (int c = lane; c < R; c += 32) out0[(int64_t)i * R + c] = 0.f;
    }
    if (t == 0 && nruns > 0) {
      // the B image copy must have landed before the CTA may exit
      long long t0 = clock64();
      while (!mbar_try_wait(b_full, 0) && clock64() - t0 < M3_DRAIN_BUDGET) {
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, (uint32_t)tmem_cols);
  }
  trace_end(p.tr);
}

// X (fp32) -> bf16 hi = rn(x), lo = rn(x - hi), same layout; ||X||^2 in FP64
// added into *norm_sq (one atomic per CTA).
__global__ void __launch_bounds__(256)
split_bf16_kernel(const float4* __restrict__ X, int64_t n4, uint2* __restrict__ hi,
                  uint2* __restrict__ lo, double* norm_sq) {
  double s0 = 0.0, s1 = 0.0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n4;
       e += (int64_t)gridDim.x * blockDim.x) {
    const float4 v = __ldg(X + e);
    const __nv_bfloat16 h0 = __float2bfloat16_rn(v.x), h1 = __float2bfloat16_rn(v.y);
    const __nv_bfloat16 h2 = __float2bfloat16_rn(v.z), h3 = __float2bfloat16_rn(v.w);
    const __nv_bfloat162 hh01 = __halves2bfloat162(h0, h1), hh23 = __halves2bfloat162(h2, h3);
    const __nv_bfloat162 ll01 = __floats2bfloat162_rn(v.x - __bfloat162float(h0),
                                                      v.y - __bfloat162float(h1));
    const __nv_bfloat162 ll23 = __floats2bfloat162_rn(v.z - __bfloat162float(h2),
                                                      v.w - __bfloat162float(h3));
    hi[e] = make_uint2(*reinterpret_cast<const uint32_t*>(&hh01),
                       *reinterpret_cast<const uint32_t*>(&hh23));
    lo[e] = make_uint2(*reinterpret_cast<const uint32_t*>(&ll01),
                       *reinterpret_cast<const uint32_t*>(&ll23));
    s0 += (double)v.x * v.x + (double)v.y * v.y;
    s1 += (double)v.z * v.z + (double)v.w * v.w;
  }
  double s = s0 + s1;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double ws[8];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += ws[w];
    atomicAdd(norm_sq, t);
  }
}

// The full B image of U (L x R): every 16-byte chunk, zero padding included.
// Chunk e sits at byte 16 e = (kb * 2 n_pad + row) * 128 + 16 pos, and holds
// the 8 consecutive k of logical chunk c = pos ^ (row & 7) of k-block kb, for
// column n = row mod n_pad (hi halves for row < n_pad, lo halves after).
__global__ void bimage_kernel(const float* __restrict__ U, int L, int R, int n_pad,
                              uint4* __restrict__ img, int chunks) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= chunks) return;
  const int pos = e & 7;
  const int rows = 2 * n_pad;
  const int row = (e >> 3) % rows;
  const int kb = (e >> 3) / rows;
  const int c = pos ^ (row & 7);
  const int n = row < n_pad ? row : row - n_pad;
  const bool want_lo = row >= n_pad;
  uint32_t w[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float v[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = kb * 64 + c * 8 + 2 * q + h;
      const float x = (n < R && k < L) ? __ldg(U + (size_t)k * R + n) : 0.f;
      const float hx = __bfloat162float(__float2bfloat16_rn(x));
      v[h] = want_lo ? x - hx : hx;
    }
    const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[0], v[1]);
    w[q] = *reinterpret_cast<const uint32_t*>(&b2);
  }
  img[e] = make_uint4(w[0], w[1], w[2], w[3]);
}

// B images of Khatri-Rao products, the layout of bimage_kernel, up to two
// images per launch: row k of a product is the row-major multi-index over its
// factors' rows, each entry the fp32 product of the factors' entries.
__global__ void kr_images_kernel(const __grid_constant__ KRImages a) {
  // programmatic launch: the predecessor's writes first (no-ops for a plain
  // launch); the next kernel may then start its own prologue
  grid_dep_wait();
  if (threadIdx.x == 0) grid_dep_trigger();
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  int w = 0;
  if (e >= a.im[0].chunks) {
    e -= a.im[0].chunks;
    w = 1;
    if (a.n < 2 || e >= a.im[1].chunks) {
      // the threads past both images zero `zero` (float4s)
      const int64_t z = (int64_t)e - (a.n < 2 ? 0 : a.im[1].chunks);
      if (z >= 0 && z < a.zero_n4) reinterpret_cast<float4*>(a.zero)[z] = make_float4(0.f, 0.f, 0.f, 0.f);
      return;
    }
  }
  const KRImage& im = a.im[w];
  const int pos = e & 7;
  const int rows = 2 * a.n_pad;
  const int row = (e >> 3) % rows;
  const int kb = (e >> 3) / rows;
  const int c = pos ^ (row & 7);
  const int n = row < a.n_pad ? row : row - a.n_pad;
  const bool want_lo = row >= a.n_pad;
  uint32_t wv[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float v[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = kb * 64 + c * 8 + 2 * q + h;
      float x = 0.f;
      if (n < a.R && k < im.L) {
        x = 1.f;
        int rem = k;
        for (int f = im.nf - 1; f >= 0; --f) {
          const int sz = im.size[f];
          const int nxt = rem / sz;
          x *= __ldg(im.U[f] + (int64_t)(rem - nxt * sz) * a.R + n);
          rem = nxt;
        }
      }
      const float hx = __bfloat162float(__float2bfloat16_rn(x));
      v[h] = want_lo ? x - hx : hx;
    }
    const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[0], v[1]);
    wv[q] = *reinterpret_cast<const uint32_t*>(&b2);
  }
  reinterpret_cast<uint4*>(im.img)[e] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point.
typedef CUresult (*EncodeTiledFn3)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn3 encode_fn() {
  static EncodeTiledFn3 fn = nullptr;
  if (!fn) {
    void* q = nullptr;
    cudaDriverEntryPointQueryResult r;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &q, cudaEnableDefault, &r) ==
            cudaSuccess &&
        r == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn3)q;
  }
  return fn;
}

// X as (K, J, I) with the box of `mode`: (64, 1, 128), (64, 128, 1) or (64, 64, 1).
int encode_map3(CUtensorMap* map, const __nv_bfloat16* base, const Dense3& d, int mode);

// Encoded maps are cached by (base, sizes, mode): encoding is a driver call of
// a few microseconds, which a timed or repeated launch should not pay again.
int make_map3(CUtensorMap* map, const __nv_bfloat16* base, const Dense3& d, int mode) {
  struct Entry {
    const void* base;
    int64_t I, J, K;
    int mode;
    CUtensorMap map;
  };
  static std::mutex mu;
  static std::vector<Entry> cache;  // small, most recent last
  {
    std::lock_guard<std::mutex> lock(mu);
    for (const Entry& e : cache)
      if (e.base == base && e.I == d.I && e.J == d.J && e.K == d.K && e.mode == mode) {
        *map = e.map;
        return TSR_OK;
      }
  }
  TSR_TRY(encode_map3(map, base, d, mode));
  std::lock_guard<std::mutex> lock(mu);
  if (cache.size() >= 24) cache.erase(cache.begin());
  cache.push_back(Entry{base, d.I, d.J, d.K, mode, *map});
  return TSR_OK;
}

int encode_map3(CUtensorMap* map, const __nv_bfloat16* base, const Dense3& d, int mode) {
  EncodeTiledFn3 enc = encode_fn();
  if (!enc) return fail(TSR_E_CUDA, "cuTensorMapEncodeTiled unavailable");
  if (((uintptr_t)base & 15) || (d.K * 2) % 16)
    return fail(TSR_E_INVALID_ARG, "TMA operand misaligned");
  cuuint64_t dims[3] = {(cuuint64_t)d.K, (cuuint64_t)d.J, (cuuint64_t)d.I};
  cuuint64_t strides[2] = {(cuuint64_t)(d.K * 2), (cuuint64_t)(d.J * d.K * 2)};
  cuuint32_t box[3] = {64, 1, 128};
  if (mode == 1) {
    box[1] = 128;
    box[2] = 1;
  } else if (mode == 2) {
    box[1] = 64;
    box[2] = 1;
  }
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, (void*)base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(TSR_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return TSR_OK;
}

// ---------------------------------------------------------------------------
// Two-sided contraction of X seen as an A x C matrix (row-major bf16 halves,
// C = the trailing modes' product): in one read of X,
//   T = X W    (A x R; W is C x R)      the MTTKRP side of the leading modes
//   P = X^T V  (C x R; V is A x R)      the MTTKRP side of the trailing modes
// W and V enter as B images (hi | lo rows, n_pad = 32). A CTA owns TS_TA
// consecutive 128-row blocks of A and a range of 128-column blocks of C; a
// tile (128 a x 128 c) arrives as four TMA boxes (hi and lo, two 64-column
// boxes each, 128-byte swizzle) plus the W image of its column block and the
// V image of its row block. The same shared-memory tile is
//   the K-major A operand of T's MMA (rows a, K = c), accumulated in TMEM
//     over every column block of the CTA (one accumulator per row block);
//   the MN-major A operand of P's MMA (rows c, K = a), accumulated over the
//     CTA's row blocks, then added into P (fp32 vector atomics) per column
//     block from a double-buffered accumulator.
// BF16x3 as in the MTTKRP above: D += Xhi [Bhi | Blo], D += Xlo [Bhi | Blo],
// the result column n is D[:, n] + D[:, 32 + n].
// Warp 0 TMA producer, warp 1 TMEM and the MMA-issuing thread, warps 2..5
// the epilogue. Every wait is bounded (DS_TIMEOUT, then a drain).
constexpr int TS_BM = 128;
constexpr int TS_BOX = 128 * 64 * 2;                 // one 64-column box, 16 KB
constexpr int TS_NPAD = 32;
constexpr int TS_BTILE = 2 * TS_NPAD * 128;          // one 64-k block of an image, 8 KB
constexpr int TS_STAGE = 4 * TS_BOX + 4 * TS_BTILE;  // X hi, X lo, W and V images
constexpr int TS_STAGES = 2;
constexpr int TS_TA = 4;
constexpr int TS_THREADS = 192;
constexpr uint32_t TS_TMEM_COLS = 512;  // TS_TA T accumulators + 2 P buffers of 64
constexpr size_t TS_SMEM = 1024 + (size_t)TS_STAGES * TS_STAGE + 8 * (2 * TS_STAGES + 6) + 16;

struct TSParams {
  int64_t A, C;
  int R;
  int nab, ncb;        // 128-row blocks of A, 128-column blocks of C
  int cb_per_split;
  const uint8_t* wimg;  // ncb * 2 image blocks
  const uint8_t* vimg;  // nab * 2 image blocks
  float* T;
  float* P;
  unsigned* status;
  long long wait_budget;
};

__device__ __forceinline__ uint64_t evict_first_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ void tma_load_2d_hint(void* dst, const CUtensorMap* map, int32_t x,
                                                 int32_t y, uint64_t* bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%2, %3}], [%4], %5;" ::"r"(sm100::smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(sm100::smem_u32(bar)), "l"(policy)
      : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          sm100::smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(sm100::smem_u32(bar))
      : "memory");
}

// rows row0 .. row0 + 31 (one per lane) of a 64-column accumulator, hh | cr
// halves summed, added into out[row, 0 .. R-1] for row < rows
__device__ __forceinline__ void ts_flush(uint32_t taddr, int64_t row, int64_t rows, int R,
                                         float* out) {
  using namespace sm100;
  uint32_t rh[2][16], rc[2][16];
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    tmem_ld16_nowait(taddr + (uint32_t)(16 * g), rh[g]);
    tmem_ld16_nowait(taddr + (uint32_t)(TS_NPAD + 16 * g), rc[g]);
  }
  tmem_wait_ld();
  if (row >= rows) return;
  float v[32];
#pragma unroll
  for (int g = 0; g < 2; ++g)
#pragma unroll
    for (int i = 0; i < 16; ++i) v[16 * g + i] = __uint_as_float(rh[g][i]) + __uint_as_float(rc[g][i]);
  float* o = out + row * R;
  if ((R & 3) == 0) {
#pragma unroll
    for (int n = 0; n < 32; n += 4)
      if (n < R) atomicAdd(reinterpret_cast<float4*>(o + n), make_float4(v[n], v[n + 1], v[n + 2], v[n + 3]));
  } else {
#pragma unroll
    for (int n = 0; n < 32; ++n)
      if (n < R) atomicAdd(o + n, v[n]);
  }
}

__global__ void __launch_bounds__(TS_THREADS, 1)
twosided_kernel(const __grid_constant__ CUtensorMap map_hi,
                const __grid_constant__ CUtensorMap map_lo, TSParams p) {
  using namespace sm100;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
  constexpr int S = TS_STAGES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)S * TS_STAGE);
  uint64_t* tma_full = bars;
  uint64_t* empty = bars + S;
  uint64_t* p_full = bars + 2 * S;       // [2]
  uint64_t* p_empty = bars + 2 * S + 2;  // [2]
  uint64_t* t_full = bars + 2 * S + 4;
  uint64_t* mma_done = bars + 2 * S + 5;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 6);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ab0 = (int)blockIdx.y * TS_TA;
  const int nta = p.nab - ab0 < TS_TA ? p.nab - ab0 : TS_TA;
  const int cb0 = (int)blockIdx.x * p.cb_per_split;
  const int cleft = p.ncb - cb0;
  const int nc = cleft <= 0 ? 0 : (cleft < p.cb_per_split ? cleft : p.cb_per_split);
  const int nsteps = nta > 0 ? nc * nta : 0;
  if (threadIdx.x == 0) grid_dep_trigger();

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&tma_full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&p_full[b], 1);
      mbar_init(&p_empty[b], 4);
    }
    mbar_init(t_full, 1);
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    fence_barrier_init();
    prefetch_tmap(&map_hi);
    prefetch_tmap(&map_lo);
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, TS_TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  // programmatic launch: the prologue above overlapped the predecessor; its
  // writes (the B images, the zeroed T and P) are complete from here on
  grid_dep_wait();

  if (warp == 0) {
    if (lane == 0) {
      const uint64_t pol = evict_first_policy();  // every tile is read once
      int issued_upto = 0;
      for (int it = 0; it < nsteps; ++it) {
        const int s = it % S;
        const uint32_t ph = (uint32_t)(it / S) & 1u;
        if (!m3_wait(&empty[s], ph ^ 1u, abort_flag, p.wait_budget)) {
          *abort_flag = 1;
          atomicOr(p.status, DS_TIMEOUT);
          break;
        }
        uint8_t* st = smem + (size_t)s * TS_STAGE;
        const int cb = cb0 + it / nta, ab = ab0 + it % nta;
        const int32_t x = cb * 128, y = ab * TS_BM;
        mbar_arrive_expect_tx(&tma_full[s], (uint32_t)TS_STAGE);
        tma_load_2d_hint(st, &map_hi, x, y, &tma_full[s], pol);
        tma_load_2d_hint(st + TS_BOX, &map_hi, x + 64, y, &tma_full[s], pol);
        tma_load_2d_hint(st + 2 * TS_BOX, &map_lo, x, y, &tma_full[s], pol);
        tma_load_2d_hint(st + 3 * TS_BOX, &map_lo, x + 64, y, &tma_full[s], pol);
        bulk_load(st + 4 * TS_BOX, p.wimg + (size_t)cb * 2 * TS_BTILE, 2 * TS_BTILE,
                  &tma_full[s]);
        bulk_load(st + 4 * TS_BOX + 2 * TS_BTILE, p.vimg + (size_t)ab * 2 * TS_BTILE,
                  2 * TS_BTILE, &tma_full[s]);
        issued_upto = it + 1;
      }
      for (int it = issued_upto - S > 0 ? issued_upto - S : 0; it < issued_upto; ++it) {
        const int s = it % S;
        const uint32_t ph = (uint32_t)(it / S) & 1u;
        long long t0 = clock64();
        while (!mbar_try_wait(&tma_full[s], ph) && clock64() - t0 < M3_DRAIN_BUDGET) {
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc_t = idesc_bf16_f32(TS_BM, 2 * TS_NPAD);
      const uint32_t idesc_p = idesc_t | (1u << 15);  // A MN-major (rows c)
      bool ok = true;
      for (int it = 0; it < nsteps; ++it) {
        const int s = it % S;
        const uint32_t ph = (uint32_t)(it / S) & 1u;
        const int ci = it / nta, t = it % nta, pb = ci & 1;
        // P buffer pb was last used by column block ci - 2
        if (t == 0 && ci >= 2 &&
            !m3_wait(&p_empty[pb], (uint32_t)((ci >> 1) - 1) & 1u, abort_flag, p.wait_budget)) {
          ok = false;
          break;
        }
        if (!m3_wait(&tma_full[s], ph, abort_flag, p.wait_budget)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t xh = smem_u32(smem + (size_t)s * TS_STAGE);
        const uint32_t xl = xh + 2 * TS_BOX;
        const uint32_t wi = xh + 4 * TS_BOX;
        const uint32_t vi = wi + 2 * TS_BTILE;
        const uint32_t acc_t = tmem + (uint32_t)(t * 2 * TS_NPAD);
        const uint32_t acc_p = tmem + (uint32_t)(TS_TA * 2 * TS_NPAD + pb * 2 * TS_NPAD);
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {  // T: K = c, 16 columns (32 B) per slice
            const uint64_t db = desc_sw128_kmajor(wi + h * TS_BTILE + kk * 32u);
            const uint32_t first = (ci == 0 && h == 0 && kk == 0) ? 0u : 1u;
            mma_bf16(acc_t, desc_sw128_kmajor(xh + h * TS_BOX + kk * 32u), db, idesc_t, first);
            mma_bf16(acc_t, desc_sw128_kmajor(xl + h * TS_BOX + kk * 32u), db, idesc_t, 1u);
          }
#pragma unroll
        for (int kh = 0; kh < 2; ++kh)
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {  // P: K = a, 16 rows (2 KB) per slice
            const uint32_t off = (uint32_t)(kh * 4 + kk) * 2048u;
            const uint64_t db = desc_sw128_kmajor(vi + kh * TS_BTILE + kk * 32u);
            const uint32_t first = (t == 0 && kh == 0 && kk == 0) ? 0u : 1u;
            mma_bf16(acc_p, desc_sw128_mnmajor(xh + off, TS_BOX), db, idesc_p, first);
            mma_bf16(acc_p, desc_sw128_mnmajor(xl + off, TS_BOX), db, idesc_p, 1u);
          }
        mma_commit(&empty[s]);
        if (t == nta - 1) mma_commit(&p_full[pb]);
      }
      if (ok) mma_commit(t_full);
      if (!ok) {
        *abort_flag = 1;
        atomicOr(p.status, DS_TIMEOUT);
      }
      mma_commit(mma_done);
      long long t0 = clock64();
      while (!mbar_try_wait(mma_done, 0) && clock64() - t0 < M3_DRAIN_BUDGET) {
      }
    }
  } else if (nsteps > 0) {
    const int q = warp & 3;  // TMEM lane quadrant of this warp
    const uint32_t lanes = (uint32_t)(q * 32) << 16;
    bool ok = true;
    for (int ci = 0; ci < nc; ++ci) {
      const int pb = ci & 1;
      int w_ok = 1;
      if (lane == 0)
        w_ok = m3_wait(&p_full[pb], (uint32_t)(ci >> 1) & 1u, abort_flag, p.wait_budget) ? 1 : 0;
      w_ok = __shfl_sync(0xffffffffu, w_ok, 0);
      if (!w_ok) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int64_t c = (int64_t)(cb0 + ci) * 128 + q * 32 + lane;
      ts_flush(tmem + lanes + (uint32_t)(TS_TA * 2 * TS_NPAD + pb * 2 * TS_NPAD), c, p.C, p.R,
               p.P);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&p_empty[pb]);
    }
    if (ok) {
      int w_ok = 1;
      if (lane == 0) w_ok = m3_wait(t_full, 0, abort_flag, p.wait_budget) ? 1 : 0;
      w_ok = __shfl_sync(0xffffffffu, w_ok, 0);
      ok = w_ok != 0;
    }
    if (ok) {
      tc_fence_after();
      for (int t = 0; t < nta; ++t) {
        const int64_t a = (int64_t)(ab0 + t) * TS_BM + q * 32 + lane;
        ts_flush(tmem + lanes + (uint32_t)(t * 2 * TS_NPAD), a, p.A, p.R, p.T);
      }
    } else if (lane == 0) {
      atomicOr(p.status, DS_TIMEOUT);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, TS_TMEM_COLS);
  }
}

int encode_map_2d(CUtensorMap* map, const __nv_bfloat16* base, int64_t rows, int64_t cols) {
  EncodeTiledFn3 enc = encode_fn();
  if (!enc) return fail(TSR_E_CUDA, "cuTensorMapEncodeTiled unavailable");
  if (((uintptr_t)base & 15) || (cols * 2) % 16)
    return fail(TSR_E_INVALID_ARG, "TMA operand misaligned");
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(cols * 2)};
  cuuint32_t box[2] = {64, (cuuint32_t)TS_BM};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(TSR_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return TSR_OK;
}

size_t m3_smem(const Dense3& d, int mode, int stages) {
  const int L = mode == 2 ? (int)d.J : (int)d.K;
  return 1024 + (size_t)stages * 2 * M3_A_TILE + (size_t)ceil_div(L, M3_BK) * 2 * d.n_pad * 128 +
         sizeof(float) * M3_MAX_RUNS * 64 + 8 * (2 * stages + 6) + 16;
}

}  // namespace

void init_mttkrp3_attributes() {
  cudaFuncSetAttribute(mttkrp3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kM3MaxSmem);
  cudaFuncSetAttribute(twosided_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)TS_SMEM);
}

bool dense3_supported(int ndim, const int64_t* shape, int R) {
  if (ndim != 3 || R < 1 || R > 64) return false;
  const int64_t I = shape[0], J = shape[1], K = shape[2];
  if (I < 1 || J < 1 || K < 1 || K % 8 != 0) return false;
  if (round_up(K, M3_BK) > M3_MAX_L || round_up(J, M3_BK) > M3_MAX_L) return false;
  if (I * J * K >= ((int64_t)1 << 40)) return false;
  return I < INT32_MAX && J < INT32_MAX;
}

int dense3_n_pad(int R) { return R <= 32 ? 32 : 64; }

size_t bimage_bytes(int64_t L, int n_pad) {
  return (size_t)ceil_div(L, M3_BK) * 2 * n_pad * 128;
}

int launch_split_bf16(tsr_ctx* ctx, cudaStream_t s, const float* X, int64_t n, __nv_bfloat16* hi,
                      __nv_bfloat16* lo, double* norm_sq) {
  if (n % 4 != 0 || ((uintptr_t)X & 15) || ((uintptr_t)hi & 7) || ((uintptr_t)lo & 7))
    return fail(TSR_E_INVALID_ARG, "bf16 split needs a 16-byte aligned tensor of 4k elements");
  const int64_t n4 = n / 4;
  const unsigned grid = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(ceil_div(n4, 256), 4 * (int64_t)ctx->sm_count));
  split_bf16_kernel<<<grid, 256, 0, s>>>(reinterpret_cast<const float4*>(X), n4,
                                         reinterpret_cast<uint2*>(hi),
                                         reinterpret_cast<uint2*>(lo), norm_sq);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_bimage(tsr_ctx* ctx, cudaStream_t s, const float* U, int64_t L, int R, int n_pad,
                  uint8_t* img, int64_t L_img) {
  const int chunks = (int)(bimage_bytes(std::max(L, L_img), n_pad) / 16);
  bimage_kernel<<<(unsigned)ceil_div(chunks, 256), 256, 0, s>>>(U, (int)L, R, n_pad,
                                                               reinterpret_cast<uint4*>(img),
                                                               chunks);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

SplitPlan plan_mttkrp3(const tsr_ctx* ctx, const Dense3& d, int mode) {
  SplitPlan p;
  const int64_t rows = mode == 0 ? d.I : (mode == 1 ? d.J : d.K);
  const int64_t runs = mode == 0 ? d.J : d.I;
  const int64_t mt = ceil_div(rows, M3_BM);
  const int64_t want = std::max<int64_t>(1, (ctx->sm_count - ctx->reserve_sms) / mt);
  int64_t per = ceil_div(runs, std::min<int64_t>(want, runs));
  per = std::min<int64_t>(per, M3_MAX_RUNS);
  p.splits = (int)ceil_div(runs, per);
  p.k_per_split = per;  // runs per split
  p.run_length = mode == 2 ? (int)d.J : (int)d.K;
  return p;
}

int64_t dense3_rows(const Dense3& d, int mode) { return mode == 0 ? d.I : (mode == 1 ? d.J : d.K); }

int launch_mttkrp3(tsr_ctx* ctx, cudaStream_t s, const Dense3& d, int mode, const FactorTable& ft,
                   const SplitPlan& plan, float* partials, bool a_resident) {
  if (mode < 0 || mode > 2) return fail(TSR_E_MODE_OOB, "mode %d", mode);
  CUtensorMap mh, ml;
  TSR_TRY(make_map3(&mh, d.hi, d, mode));
  TSR_TRY(make_map3(&ml, d.lo, d, mode));
  M3Params q;
  q.mode = mode;
  q.rows = dense3_rows(d, mode);
  q.runs = mode == 0 ? d.J : d.I;
  q.L = mode == 2 ? (int)d.J : (int)d.K;
  q.runs_per_split = (int)plan.k_per_split;
  q.R = d.R;
  q.n_pad = d.n_pad;
  // the contracted factor's image: U2 for modes 0 and 1, U1 for mode 2
  q.bimg = d.bimg[mode == 2 ? 1 : 2];
  q.bimg_bytes = (uint32_t)bimage_bytes(q.L, d.n_pad);
  q.wf = ft.ptr[mode == 0 ? 1 : 0];
  q.partials = partials;
  q.status = ctx->d_status;
  q.wait_budget = ctx->wait_budget;
  q.a_resident = a_resident ? 1 : 0;
  q.tr = trace_slot(ctx, TRACE_MTTKRP, mode);
  if (q.runs_per_split < 1 || q.runs_per_split > M3_MAX_RUNS)
    return fail(TSR_E_INVALID_ARG, "MTTKRP split plan out of range");
  int stages = 4;
  while (stages > 2 && m3_smem(d, mode, stages) > (size_t)kM3MaxSmem) --stages;
  const size_t smem = m3_smem(d, mode, stages);
  if (smem > (size_t)kM3MaxSmem) return fail(TSR_E_UNSUPPORTED, "MTTKRP stage ring too large");
  q.stages = stages;
  dim3 grid((unsigned)plan.splits, (unsigned)ceil_div(q.rows, M3_BM));
  if (grid.y > 65535) return fail(TSR_E_UNSUPPORTED, "MTTKRP grid too large");
  TSR_CUDA(launch_pdl(mttkrp3_kernel, grid, dim3(M3_THREADS), smem, s, mh, ml, q));
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

bool twosided_supported(int64_t A, int64_t C, int R) {
  if (R < 1 || R > TS_NPAD || A < 1 || C < 8 || C % 8 != 0) return false;
  if (A >= INT32_MAX || C >= INT32_MAX) return false;
  return ceil_div(ceil_div(A, TS_BM), TS_TA) <= 65535;
}

int64_t twosided_pad(int64_t L) { return ceil_div(L, 128) * 128; }

int launch_kr_images(tsr_ctx* ctx, cudaStream_t s, const KRImages& a, bool pdl) {
  if (a.n < 1 || a.n > 2) return fail(TSR_E_INVALID_ARG, "one or two images per launch");
  if (a.zero_n4 < 0 || (a.zero_n4 > 0 && ((uintptr_t)a.zero & 15)))
    return fail(TSR_E_INVALID_ARG, "zero-fill buffer misaligned");
  int64_t total = a.zero_n4;
  for (int w = 0; w < a.n; ++w) {
    if (a.im[w].nf < 1 || a.im[w].nf > kMaxModes)
      return fail(TSR_E_INVALID_ARG, "Khatri-Rao image of %d factors", a.im[w].nf);
    // row indices in 32 bits: the padded row count below 2^31
    if ((int64_t)a.im[w].chunks * 16 / (2 * a.n_pad * 2) >= INT32_MAX)
      return fail(TSR_E_UNSUPPORTED, "Khatri-Rao image too large");
    total += a.im[w].chunks;
  }
  if (total <= 0) return TSR_OK;
  if (pdl)
    TSR_CUDA(launch_pdl(kr_images_kernel, dim3((unsigned)ceil_div(total, 256)), dim3(256), 0, s, a));
  else
    kr_images_kernel<<<(unsigned)ceil_div(total, 256), 256, 0, s>>>(a);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_twosided(tsr_ctx* ctx, cudaStream_t s, const TwoSided& a) {
  if (!twosided_supported(a.A, a.C, a.R))
    return fail(TSR_E_UNSUPPORTED, "two-sided contraction: unsupported sizes");
  CUtensorMap mh, ml;
  TSR_TRY(encode_map_2d(&mh, a.hi, a.A, a.C));
  TSR_TRY(encode_map_2d(&ml, a.lo, a.A, a.C));
  TSParams q;
  q.A = a.A;
  q.C = a.C;
  q.R = a.R;
  q.nab = (int)ceil_div(a.A, TS_BM);
  q.ncb = (int)ceil_div(a.C, 128);
  const int nag = (int)ceil_div(q.nab, TS_TA);
  const int want = std::max(1, std::min(q.ncb, ctx->sm_count / nag));
  q.cb_per_split = (int)ceil_div(q.ncb, want);
  const int splits = (int)ceil_div(q.ncb, q.cb_per_split);
  q.wimg = a.wimg;
  q.vimg = a.vimg;
  q.T = a.T;
  q.P = a.P;
  q.status = ctx->d_status;
  q.wait_budget = ctx->wait_budget;
  TSR_CUDA(launch_pdl(twosided_kernel, dim3((unsigned)splits, (unsigned)nag), dim3(TS_THREADS),
                      TS_SMEM, s, mh, ml, q));
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

}  // namespace tsr

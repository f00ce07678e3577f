// Dense MTTKRP, BF16x3 tensor-core path (sm_100a tcgen05).
//
// M = X_(n) . KR computed as  Xhi.KRhi + Xhi.KRlo + Xlo.KRhi  where x = hi + lo
// is an exact-to-2^-16 split of each fp32 value into two bf16 values; the
// three bf16 MMAs accumulate in fp32 in tensor memory (TMEM). The lo.lo term
// (relative size 2^-16 * 2^-16) is dropped.
//
// Per CTA: one 128-row M tile of the unfolding and one K range (split-K).
//   warp 0      TMA producer: X_(n) hi/lo tiles (128 x 64 bf16, 128-byte
//               swizzle) into a ring of shared-memory stages.
//   warp 1      TMEM allocator and the single MMA-issuing thread.
//   warps 2..5  Khatri-Rao producers: form 64 KR rows per stage from the other
//               factors (kr.cuh), split them into bf16 hi/lo and write them as
//               the K-major B operand (N = R padded to 16) in the same
//               swizzled layout; afterwards the epilogue (TMEM -> registers ->
//               split-K partials in HBM).
// KR rows are never written to global memory. Every mbarrier wait is bounded;
// a wait that runs out raises DS_TIMEOUT in the status word and the CTA
// drains and exits (TMA copies waited for, TMEM freed).
//
// Replaces the hot loop of crates/tenrso-kernels/src/mttkrp.rs:135-143 (and
// the KR materialisation of mttkrp.rs:182-240) for the mixed-precision mode.
#include "mttkrp.cuh"
#include "sm100.cuh"

namespace tsr {

namespace {

constexpr int TC_BM = 128;   // M tile (TMEM lanes)
constexpr int TC_BK = 64;    // K per stage: one 128-byte swizzle row of bf16
constexpr int TC_THREADS = 192;
constexpr int A_TILE_BYTES = TC_BM * TC_BK * 2;  // 16 KB
constexpr long long WAIT_BUDGET = 1ll << 31;     // ~1 s at B200 clocks

struct TcParams {
  int64_t rows;
  int64_t K;
  int64_t k_per_split;
  int n_pad;
  int stages;
  int tmem_cols;   // total TMEM columns allocated (n_acc * acc_cols)
  int acc_cols;    // columns per accumulator (power of two >= n_pad, >= 32)
  int n_acc;       // independent fp32 accumulators (even, 2..8)
  KRSpec kr;
  float* partials;
  unsigned* status;
};

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&v);
}

// Convert 8 consecutive-k values of one KR column into bf16 hi/lo and store
// them as one 16-byte chunk of the swizzled K-major B operand (row n, chunk
// kq ^ (n & 7)).
__device__ __forceinline__ void store_kr_chunk(uint8_t* b_hi, uint8_t* b_lo, int n, int kq,
                                               const float (&v)[8]) {
  float h[8], l[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    __nv_bfloat16 hb = __float2bfloat16_rn(v[e]);
    h[e] = __bfloat162float(hb);
    l[e] = v[e] - h[e];
  }
  uint4 hv = make_uint4(pack_bf16x2(h[0], h[1]), pack_bf16x2(h[2], h[3]),
                        pack_bf16x2(h[4], h[5]), pack_bf16x2(h[6], h[7]));
  uint4 lv = make_uint4(pack_bf16x2(l[0], l[1]), pack_bf16x2(l[2], l[3]),
                        pack_bf16x2(l[4], l[5]), pack_bf16x2(l[6], l[7]));
  const uint32_t byte = (uint32_t)n * 128u + ((uint32_t)(kq ^ (n & 7)) << 4);
  *reinterpret_cast<uint4*>(b_hi + byte) = hv;
  *reinterpret_cast<uint4*>(b_lo + byte) = lv;
}

// Row positions of the 8 KR rows j0 .. j0+7 a producer thread covers.
struct KRRows {
  uint32_t idx[8][kMaxModes];
  bool keep[8];
};

__device__ __forceinline__ void kr_rows(const KRSpec& kr, const KRCounter<kMaxModes>& c0,
                                        int64_t j0, int64_t kend, KRRows& r) {
  KRCounter<kMaxModes> c = c0;
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    if (e > 0) c.advance(kr, 1);
    r.keep[e] = j0 + e < kend;
#pragma unroll
    for (int p = 0; p < kMaxModes; ++p) r.idx[e][p] = r.keep[e] ? c.idx[p] : 0u;
  }
}

// Prefetchable part of a stage (fast path: at most two other modes, R % 4 == 0,
// R <= 64): the factor rows for this thread's 8 KR rows and 4 columns, and a
// bit mask of the rows that lie inside this CTA's K range.
struct KRLoads {
  float4 a[8], b[8];
  uint32_t keep;
};

__device__ __forceinline__ void kr_issue(const KRSpec& kr, const KRCounter<2>& c0, int64_t j0,
                                         int64_t kend, int nc, KRLoads& L) {
  KRCounter<2> c = c0;
  L.keep = 0;
  if (kr.n_other > 1 && c.idx[1] + 7 < kr.size[1] && j0 + 7 < kend) {
    // common case: the 8 rows share the slower factor's row and step through
    // consecutive rows of the faster one
    const float4 a0 = __ldg(reinterpret_cast<const float4*>(kr.f[0] + c.idx[0] * kr.R + nc));
    const float* fb = kr.f[1] + c.idx[1] * kr.R + nc;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      L.a[e] = a0;
      L.b[e] = __ldg(reinterpret_cast<const float4*>(fb + e * kr.R));
    }
    L.keep = 0xffu;
    return;
  }
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    if (e > 0) c.advance(kr, 1);
    const bool k = j0 + e < kend;
    L.keep |= (k ? 1u : 0u) << e;
    const uint32_t i0 = k ? c.idx[0] : 0u, i1 = k ? c.idx[1] : 0u;
    L.a[e] = __ldg(reinterpret_cast<const float4*>(kr.f[0] + i0 * kr.R + nc));
    L.b[e] = kr.n_other > 1
                 ? __ldg(reinterpret_cast<const float4*>(kr.f[1] + i1 * kr.R + nc))
                 : make_float4(1.f, 1.f, 1.f, 1.f);
  }
}

__device__ __forceinline__ void kr_finish(const KRLoads& L, int n0, bool col_ok, int kq,
                                          uint8_t* b_hi, uint8_t* b_lo) {
  float v[4][8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const bool ok = ((L.keep >> e) & 1u) && col_ok;
    v[0][e] = ok ? L.a[e].x * L.b[e].x : 0.f;
    v[1][e] = ok ? L.a[e].y * L.b[e].y : 0.f;
    v[2][e] = ok ? L.a[e].z * L.b[e].z : 0.f;
    v[3][e] = ok ? L.a[e].w * L.b[e].w : 0.f;
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) store_kr_chunk(b_hi, b_lo, n0 + c, kq, v[c]);
}

// General stage producer (any R, any number of modes): loads issued per
// 64-column pass, then consumed.
__device__ __forceinline__ void kr_produce_general(const TcParams& p, const KRRows& r,
                                                   uint8_t* b_hi, uint8_t* b_lo, int t) {
  const int kq = t & 7, ng = t >> 3;
  const KRSpec& kr = p.kr;
  const int R = kr.R;
  for (int nb = 0; nb < p.n_pad; nb += 64) {
    const int n0 = nb + ng * 4;
    if (n0 >= p.n_pad) break;
    float v[4][8];
#pragma unroll
    for (int e = 0; e < 8; ++e)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const bool ok = r.keep[e] && n0 + c < R;
        const int col = ok ? n0 + c : 0;
        v[c][e] = ok ? __ldg(kr.f[0] + r.idx[e][0] * R + col) : 0.f;
      }
#pragma unroll
    for (int q = 1; q < kMaxModes; ++q) {
      if (q < kr.n_other) {
#pragma unroll
        for (int e = 0; e < 8; ++e)
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const int col = n0 + c < R ? n0 + c : 0;
            v[c][e] *= __ldg(kr.f[q] + r.idx[e][q] * R + col);
          }
      }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) store_kr_chunk(b_hi, b_lo, n0 + c, kq, v[c]);
  }
}

template <bool VEC4, bool FAST>
__global__ void __launch_bounds__(TC_THREADS, 1)
mttkrp_bf16x3_kernel(const __grid_constant__ CUtensorMap map_hi,
                     const __grid_constant__ CUtensorMap map_lo, TcParams p) {
  using namespace sm100;
  extern __shared__ uint8_t smem_raw[];
  // 1024-byte alignment for the swizzled tiles
  uint8_t* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
  const int S = p.stages;
  const uint32_t b_bytes = (uint32_t)p.n_pad * 128u;
  const uint32_t stage_bytes = 2u * A_TILE_BYTES + 2u * b_bytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)S * stage_bytes);
  uint64_t* tma_full = bars;
  uint64_t* kr_full = bars + S;
  uint64_t* empty = bars + 2 * S;
  uint64_t* done = bars + 3 * S;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 3 * S + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t m0 = (int64_t)blockIdx.y * TC_BM;
  const int64_t kbeg = (int64_t)blockIdx.x * p.k_per_split;
  const int64_t kend = min(p.K, kbeg + p.k_per_split);
  const int nsteps = kend > kbeg ? (int)((kend - kbeg + TC_BK - 1) / TC_BK) : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&tma_full[s], 1);
      mbar_init(&kr_full[s], 4);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    fence_barrier_init();
    prefetch_tmap(&map_hi);
    prefetch_tmap(&map_lo);
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, (uint32_t)p.tmem_cols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  auto stage_ptr = [&](int s) { return smem + (size_t)s * stage_bytes; };

  if (warp == 0) {
    if (lane == 0) {
      int issued_upto = 0;
      for (int it = 0; it < nsteps; ++it) {
        const int s = it % S;
        const uint32_t ph = (uint32_t)(it / S) & 1u;
        if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag, WAIT_BUDGET)) {
          *abort_flag = 1;
          atomicOr(p.status, DS_TIMEOUT);
          break;
        }
        uint8_t* st = stage_ptr(s);
        mbar_arrive_expect_tx(&tma_full[s], 2u * A_TILE_BYTES);
        const int32_t x = (int32_t)(kbeg + (int64_t)it * TC_BK);
        const int32_t y = (int32_t)m0;
        tma_load_2d(st, &map_hi, x, y, &tma_full[s]);
        tma_load_2d(st + A_TILE_BYTES, &map_lo, x, y, &tma_full[s]);
        issued_upto = it + 1;
      }
      // drain: the last issued phase of every stage must have landed before
      // the CTA may exit (bounded; no abort short-cut here)
      for (int it = issued_upto - S > 0 ? issued_upto - S : 0; it < issued_upto; ++it) {
        const int s = it % S;
        const uint32_t ph = (uint32_t)(it / S) & 1u;
        long long t0 = clock64();
        while (!mbar_try_wait(&tma_full[s], ph) && clock64() - t0 < WAIT_BUDGET) {
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(TC_BM, p.n_pad);
      for (int it = 0; it < nsteps; ++it) {
        const int s = it % S;
        const uint32_t ph = (uint32_t)(it / S) & 1u;
        if (!mbar_wait(&tma_full[s], ph, abort_flag, WAIT_BUDGET) ||
            !mbar_wait(&kr_full[s], ph, abort_flag, WAIT_BUDGET)) {
          *abort_flag = 1;
          atomicOr(p.status, DS_TIMEOUT);
          break;
        }
        tc_fence_after();
        uint8_t* st = stage_ptr(s);
        const uint32_t a_hi = smem_u32(st), a_lo = a_hi + A_TILE_BYTES;
        const uint32_t b_hi = a_hi + 2 * A_TILE_BYTES, b_lo = b_hi + b_bytes;
#pragma unroll
        for (int kk = 0; kk < TC_BK / 16; ++kk) {
          const uint32_t koff = kk * 32;  // 16 bf16 = 32 bytes along K
          const uint64_t dah = desc_sw128_kmajor(a_hi + koff);
          const uint64_t dal = desc_sw128_kmajor(a_lo + koff);
          const uint64_t dbh = desc_sw128_kmajor(b_hi + koff);
          const uint64_t dbl = desc_sw128_kmajor(b_lo + koff);
          // The tensor core's fp32 accumulation truncates, so a long chain
          // of accumulations drifts low. k-slices rotate over n_acc/2
          // accumulators for hi.hi and n_acc/2 more for the (2^-8 smaller)
          // correction products; the epilogue adds them in FP64.
          const int half = p.n_acc >> 1;
          const int g = it * (TC_BK / 16) + kk;  // k-slice index in this split
          const uint32_t acc_hh = tmem + (uint32_t)((g % half) * p.acc_cols);
          const uint32_t acc_cr = tmem + (uint32_t)((half + g % half) * p.acc_cols);
          const uint32_t first = g < half ? 0u : 1u;
          mma_bf16(acc_hh, dah, dbh, idesc, first);
          mma_bf16(acc_cr, dah, dbl, idesc, first);
          mma_bf16(acc_cr, dal, dbh, idesc, 1u);
        }
        mma_commit(&empty[s]);
      }
      mma_commit(done);  // tracks every MMA issued above (also on abort)
    }
  } else {
    // Khatri-Rao producers (warps 2..5, 128 threads). Thread t covers KR rows
    // kbase + 8*(t & 7) .. +7 and columns 4*(t >> 3) .. +3 of each 64-column
    // pass. Row positions advance by a mixed-radix counter (no division per
    // row). On the fast path the factor loads of stage it+1 are issued before
    // stage it is converted, so their L2 latency overlaps the work.
    const int t = threadIdx.x - 64;
    const int kq = t & 7;
    const int n0 = (t >> 3) * 4;
    KRCounter<FAST ? 2 : kMaxModes> ctr;
    ctr.init(p.kr, (uint32_t)(kbeg + kq * 8));
    KRLoads loads[2];
    constexpr bool fast = FAST;
    const bool col_ok = n0 < p.kr.R;
    const int nc = col_ok ? n0 : 0;
    const bool active = n0 < p.n_pad;
    auto stage = [&](int it, KRLoads& cur, KRLoads& nxt) -> bool {
      const int s = it % S;
      const uint32_t ph = (uint32_t)(it / S) & 1u;
      if constexpr (FAST) {
        if (active && it + 1 < nsteps) {
          ctr.advance(p.kr, TC_BK);
          kr_issue(p.kr, ctr, kbeg + (int64_t)(it + 1) * TC_BK + kq * 8, kend, nc, nxt);
        }
      }
      int ok = 1;
      if (lane == 0) ok = mbar_wait(&empty[s], ph ^ 1u, abort_flag, WAIT_BUDGET) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) {
          *abort_flag = 1;
          atomicOr(p.status, DS_TIMEOUT);
        }
        return false;
      }
      uint8_t* st = stage_ptr(s);
      uint8_t* bh = st + 2 * A_TILE_BYTES;
      uint8_t* bl = bh + b_bytes;
      if (fast) {
        if (active) kr_finish(cur, n0, col_ok, kq, bh, bl);
      } else {
        if constexpr (!FAST) {
          if (it > 0) ctr.advance(p.kr, TC_BK);
          KRRows rows;
          kr_rows(p.kr, ctr, kbeg + (int64_t)it * TC_BK + kq * 8, kend, rows);
          kr_produce_general(p, rows, bh, bl, t);
        }
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&kr_full[s]);
      return true;
    };
    if constexpr (FAST) {
      if (active && nsteps > 0) kr_issue(p.kr, ctr, kbeg + kq * 8, kend, nc, loads[0]);
    }
    for (int it = 0; it < nsteps; it += 2) {
      if (!stage(it, loads[0], loads[1])) break;
      if (it + 1 < nsteps && !stage(it + 1, loads[1], loads[0])) break;
    }
    // epilogue: TMEM accumulator -> split-K partial rows
    int ok = 1;
    if (lane == 0) ok = mbar_wait(done, 0, abort_flag, WAIT_BUDGET) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    tc_fence_after();
    const int q = warp & 3;  // TMEM lane quadrant this warp may access
    const int64_t row = m0 + q * 32 + lane;
    const int R = p.kr.R;
    float* out = p.partials + (int64_t)blockIdx.x * p.rows * R + row * R;
    if (ok && nsteps > 0) {
      // accumulators that never received a k-slice (short splits) are skipped
      const int used = min(p.n_acc >> 1, nsteps * (TC_BK / 16));
      for (int c0 = 0; c0 < p.n_pad; c0 += 16) {
        double sum[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) sum[i] = 0.0;
        // up to 8 accumulators: all loads in flight, one wait
        uint32_t r[8][16];
        const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0;
#pragma unroll
        for (int a = 0; a < 8; ++a)
          if (a < p.n_acc && (a % (p.n_acc >> 1)) < used)  // warp-uniform
            tmem_ld16_nowait(base + (uint32_t)(a * p.acc_cols), r[a]);
        tmem_wait_ld();
#pragma unroll
        for (int a = 0; a < 8; ++a)
          if (a < p.n_acc && (a % (p.n_acc >> 1)) < used) {
#pragma unroll
            for (int i = 0; i < 16; ++i) sum[i] += (double)__uint_as_float(r[a][i]);
          }
        if (row < p.rows) {
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (c0 + i < R) out[c0 + i] = (float)sum[i];
        }
      }
    } else if (row < p.rows) {
      if (!ok && lane == 0) atomicOr(p.status, DS_TIMEOUT);
      for (int c = 0; c < R; ++c) out[c] = 0.f;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, (uint32_t)p.tmem_cols);
  }
}

// ---------------------------------------------------------------------------
// Prefix-scaled variant. When the fastest other mode has size L (a multiple
// of 64), the KR rows come in runs of L that share every slower mode's row:
// run P is U_last (L x R) with its columns scaled by the weight vector
//   w_P[n] = prod over the slower other modes q of U_q[i_q(P), n],
// so  M = sum_P (X_P . U_last) diag(w_P)  with X_P the L unfolding columns of
// run P. U_last is the same for every run: the producer warps write it once
// per CTA as the swizzled bf16 hi/lo B operand (instead of one KR tile per
// stage). Each run's X_P . U_last accumulates in TMEM (hi.hi and the two
// correction products in separate accumulators, double buffered across
// runs); the epilogue warps scale it by w_P and add it into registers.
// Split-K boundaries fall on run boundaries.
constexpr int TCS_MAX_RUNS = 16;  // runs per CTA (their weights sit in shared memory)
constexpr int TCS_MAX_L = 384;    // U_last tiles must fit beside the stage ring

struct TcsParams {
  int64_t rows;
  int64_t K;
  int64_t k_per_split;  // a whole number of runs
  int runs_per_split;   // k_per_split / L
  int L;                // run length, multiple of 8 (padded to 64-wide k-blocks)
  int n_pad;            // R rounded up to 16 (<= 64)
  int acc_cols;         // TMEM columns per accumulator (power of two >= max(n_pad, 32))
  int stages;
  KRSpec kr;
  float* partials;
  unsigned* status;
  int a_resident;       // the unfolding may be streamed before the launch wait
};

// Launched with programmatic dependent launch: the previous kernel of the
// stream (in a CP-ALS sweep, the solve that updated a factor) may still be
// running at entry. The TMA producer streams the unfolding at once when it
// is resident (written before that kernel); the epilogue warps wait for the
// previous grid before they read any factor and before the partials (which
// that kernel may read) are written.
__global__ void __launch_bounds__(TC_THREADS, 1)
mttkrp_bf16x3_runs_kernel(const __grid_constant__ CUtensorMap map_hi,
                          const __grid_constant__ CUtensorMap map_lo, TcsParams p) {
  using namespace sm100;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
  const int S = p.stages;
  const int spr = (p.L + TC_BK - 1) / TC_BK;            // stages per run (last one padded)
  const uint32_t bblk = (uint32_t)p.n_pad * 128u;       // one k-block of B (hi or lo)
  uint8_t* a_base = smem;
  uint8_t* b_base = smem + (size_t)S * 2 * A_TILE_BYTES;
  float* wts = reinterpret_cast<float*>(b_base + (size_t)spr * 2 * bblk);  // [runs][64]
  uint64_t* bars = reinterpret_cast<uint64_t*>(wts + TCS_MAX_RUNS * 64);
  uint64_t* tma_full = bars;
  uint64_t* empty = bars + S;
  uint64_t* acc_full = bars + 2 * S;   // [2]
  uint64_t* acc_empty = bars + 2 * S + 2;  // [2]
  uint64_t* b_ready = bars + 2 * S + 4;
  uint64_t* mma_done = bars + 2 * S + 5;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 6);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t m0 = (int64_t)blockIdx.y * TC_BM;
  const int64_t kbeg = (int64_t)blockIdx.x * p.k_per_split;
  const int64_t kend = min(p.K, kbeg + p.k_per_split);
  const int nruns = kend > kbeg ? (int)((kend - kbeg) / p.L) : 0;
  const int nsteps = nruns * spr;
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
    mbar_init(b_ready, 4);
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    fence_barrier_init();
    prefetch_tmap(&map_hi);
    prefetch_tmap(&map_lo);
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, (uint32_t)(4 * p.acc_cols));
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      if (!p.a_resident) grid_dep_wait();
      int issued_upto = 0;
      for (int it = 0; it < nsteps; ++it) {
        const int s = it % S;
        const uint32_t ph = (uint32_t)(it / S) & 1u;
        if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag, WAIT_BUDGET)) {
          *abort_flag = 1;
          atomicOr(p.status, DS_TIMEOUT);
          break;
        }
        uint8_t* st = a_base + (size_t)s * 2 * A_TILE_BYTES;
        mbar_arrive_expect_tx(&tma_full[s], 2u * A_TILE_BYTES);
        // [rows][runs][L] view: columns at or beyond L of a run read as zero
        const int32_t x = (int32_t)((it % spr) * TC_BK);
        const int32_t y = (int32_t)((int64_t)blockIdx.x * p.runs_per_split + it / spr);
        const int32_t z = (int32_t)m0;
        tma_load_3d(st, &map_hi, x, y, z, &tma_full[s]);
        tma_load_3d(st + A_TILE_BYTES, &map_lo, x, y, z, &tma_full[s]);
        issued_upto = it + 1;
      }
      // drain: every issued copy must have landed before the CTA may exit
      for (int it = issued_upto - S > 0 ? issued_upto - S : 0; it < issued_upto; ++it) {
        const int s = it % S;
        const uint32_t ph = (uint32_t)(it / S) & 1u;
        long long t0 = clock64();
        while (!mbar_try_wait(&tma_full[s], ph) && clock64() - t0 < WAIT_BUDGET) {
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(TC_BM, p.n_pad);
      bool ok = mbar_wait(b_ready, 0, abort_flag, WAIT_BUDGET);
      for (int r = 0; ok && r < nruns; ++r) {
        const int b = r & 1;
        // buffer b was last used by run r - 2: wait until the epilogue read it
        if (r >= 2 && !mbar_wait(&acc_empty[b], (uint32_t)((r >> 1) - 1) & 1u, abort_flag,
                                 WAIT_BUDGET)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t acc_hh = tmem + (uint32_t)(2 * b * p.acc_cols);
        const uint32_t acc_cr = acc_hh + (uint32_t)p.acc_cols;
        for (int sp = 0; sp < spr; ++sp) {
          const int it = r * spr + sp;
          const int s = it % S;
          const uint32_t ph = (uint32_t)(it / S) & 1u;
          if (!mbar_wait(&tma_full[s], ph, abort_flag, WAIT_BUDGET)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a_hi = smem_u32(a_base + (size_t)s * 2 * A_TILE_BYTES);
          const uint32_t a_lo = a_hi + A_TILE_BYTES;
          const uint32_t b_hi = smem_u32(b_base) + (uint32_t)sp * 2u * bblk;
          const uint32_t b_lo = b_hi + bblk;
#pragma unroll
          for (int kk = 0; kk < TC_BK / 16; ++kk) {
            const uint32_t koff = kk * 32;  // 16 bf16 = 32 bytes along K
            const uint64_t dah = desc_sw128_kmajor(a_hi + koff);
            const uint64_t dal = desc_sw128_kmajor(a_lo + koff);
            const uint64_t dbh = desc_sw128_kmajor(b_hi + koff);
            const uint64_t dbl = desc_sw128_kmajor(b_lo + koff);
            const uint32_t first = (sp == 0 && kk == 0) ? 0u : 1u;
            mma_bf16(acc_hh, dah, dbh, idesc, first);
            mma_bf16(acc_cr, dah, dbl, idesc, first);
            mma_bf16(acc_cr, dal, dbh, idesc, 1u);
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
      while (!mbar_try_wait(mma_done, 0) && clock64() - t0 < WAIT_BUDGET) {
      }
    }
  } else {
    // warps 2..5: write U_last as the B operand and the runs' weights once,
    // then consume every run's accumulators
    const int t = threadIdx.x - 64;
    const KRSpec& kr = p.kr;
    const int R = kr.R;
    const int last = kr.n_other - 1;
    const float* ul = kr.f[last];
    grid_dep_wait();  // the factors (and the partials' readers) of the previous kernel
    {
      // Every global load of the setup waits behind the TMA ring fill of all
      // CTAs, so the loads are grouped into as few round trips as possible:
      // the run weights' factor rows are issued first, together with the
      // first U_last batch, and multiplied after the B operand is written.
      //
      // Weights: thread t covers runs r = (t >> 4) + 8j (j < 2) and columns
      // c0 .. c0+3. Run P = run0 + r of this split decomposes mixed-radix
      // over the slower other modes (q = last - 1 fastest), and
      // w_P = prod_q U_q[i_q(P)] (columns >= R get weight 0).
      const int c0 = (t & 15) * 4;
      bool wvec = (R & 3) == 0;
#pragma unroll
      for (int q = 0; q < kMaxModes - 1; ++q)
        if (q < last) wvec = wvec && ((uintptr_t)kr.f[q] & 15) == 0;
      float4 wf[2][kMaxModes - 1];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int r = (t >> 4) + 8 * j;
        uint32_t idx = (uint32_t)blockIdx.x * (uint32_t)p.runs_per_split + (uint32_t)r;
#pragma unroll
        for (int q = kMaxModes - 2; q >= 0; --q) {
          wf[j][q] = make_float4(1.f, 1.f, 1.f, 1.f);
          if (q < last && r < nruns) {
            const uint32_t sz = kr.size[q];
            const uint32_t qq = idx / sz;
            const uint32_t iq = idx - qq * sz;
            idx = qq;
            const float* src = kr.f[q] + (size_t)iq * R;
            if (wvec && c0 < R) {
              wf[j][q] = __ldg(reinterpret_cast<const float4*>(src + c0));
            } else {
              wf[j][q].x = c0 < R ? __ldg(src + c0) : 1.f;
              wf[j][q].y = c0 + 1 < R ? __ldg(src + c0 + 1) : 1.f;
              wf[j][q].z = c0 + 2 < R ? __ldg(src + c0 + 2) : 1.f;
              wf[j][q].w = c0 + 3 < R ? __ldg(src + c0 + 3) : 1.f;
            }
          }
        }
      }
      // U_last rows kq*8 .. +7 of each 64-row k-block, columns n0 .. n0+3:
      // two k-blocks of loads in flight at a time (128-bit when aligned)
      const int kq = t & 7, n0 = (t >> 3) * 4;
      const bool vec = (R & 3) == 0 && ((uintptr_t)ul & 15) == 0;
      if (n0 < p.n_pad) {
        for (int kb0 = 0; kb0 < spr; kb0 += 2) {
          float v[2][4][8];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int kb = kb0 + h;
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const int64_t k = (int64_t)kb * TC_BK + kq * 8 + e;
              if (k >= p.L) {  // padding rows of the last k-block of a run
#pragma unroll
                for (int c = 0; c < 4; ++c) v[h][c][e] = 0.f;
              } else if (kb < spr && vec && n0 < R) {
                const float4 x = __ldg(reinterpret_cast<const float4*>(ul + k * R + n0));
                v[h][0][e] = x.x;
                v[h][1][e] = x.y;
                v[h][2][e] = x.z;
                v[h][3][e] = x.w;
              } else {
#pragma unroll
                for (int c = 0; c < 4; ++c)
                  v[h][c][e] = (kb < spr && n0 + c < R) ? __ldg(ul + k * R + n0 + c) : 0.f;
              }
            }
          }
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            if (kb0 + h < spr) {
              uint8_t* bh = b_base + (size_t)(kb0 + h) * 2 * bblk;
#pragma unroll
              for (int c = 0; c < 4; ++c) store_kr_chunk(bh, bh + bblk, n0 + c, kq, v[h][c]);
            }
          }
        }
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int r = (t >> 4) + 8 * j;
        if (r < nruns) {
          float4 w = make_float4(c0 < R ? 1.f : 0.f, c0 + 1 < R ? 1.f : 0.f,
                                 c0 + 2 < R ? 1.f : 0.f, c0 + 3 < R ? 1.f : 0.f);
#pragma unroll
          for (int q = 0; q < kMaxModes - 1; ++q) {
            w.x *= wf[j][q].x;
            w.y *= wf[j][q].y;
            w.z *= wf[j][q].z;
            w.w *= wf[j][q].w;
          }
          *reinterpret_cast<float4*>(wts + r * 64 + c0) = w;
        }
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(b_ready);
      asm volatile("bar.sync 1, 128;" ::: "memory");  // the four epilogue warps: weights visible
    }
    const int q = warp & 3;  // TMEM lane quadrant this warp may access
    const int64_t row = m0 + q * 32 + lane;
    float acc[64];
#pragma unroll
    for (int n = 0; n < 64; ++n) acc[n] = 0.f;
    bool ok = true;
    for (int r = 0; r < nruns; ++r) {
      const int b = r & 1;
      int w_ok = 1;
      if (lane == 0)
        w_ok = mbar_wait(&acc_full[b], (uint32_t)(r >> 1) & 1u, abort_flag, WAIT_BUDGET) ? 1 : 0;
      w_ok = __shfl_sync(0xffffffffu, w_ok, 0);
      if (!w_ok) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(2 * b * p.acc_cols);
#pragma unroll
      for (int h = 0; h < 2; ++h) {  // columns 32h .. 32h + 31
        if (32 * h < p.n_pad) {
          uint32_t rh[2][16], rc[2][16];
#pragma unroll
          for (int g = 0; g < 2; ++g)
            if (32 * h + 16 * g < p.n_pad) {  // warp-uniform
              tmem_ld16_nowait(base + (uint32_t)(32 * h + 16 * g), rh[g]);
              tmem_ld16_nowait(base + (uint32_t)(p.acc_cols + 32 * h + 16 * g), rc[g]);
            }
          tmem_wait_ld();
#pragma unroll
          for (int g = 0; g < 2; ++g)
            if (32 * h + 16 * g < p.n_pad) {
#pragma unroll
              for (int i = 0; i < 16; ++i) {
                const int n = 32 * h + 16 * g + i;
                const float v = __uint_as_float(rh[g][i]) + __uint_as_float(rc[g][i]);
                acc[n] = fmaf(v, wts[r * 64 + n], acc[n]);
              }
            }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[b]);
    }
    // The warp's 32 rows are contiguous in the partials (row stride R): stage
    // them through the A ring (every copy into it was consumed by an MMA
    // that completed before the last acc_full) and store whole rows,
    // coalesced. With R % 4 == 0 the rows are staged at a 68-float stride
    // (16-byte aligned; 128-bit shared accesses conflict-free per quarter-warp)
    // and stored as float4, a warp covering 512 contiguous bytes per store;
    // else at a 65-float stride, one float per lane.
    const int64_t row0 = m0 + q * 32;
    if (ok) {
      float* stg = reinterpret_cast<float*>(a_base) + q * (32 * 68);
      fence_proxy_async_smem();
      float* out0 = p.partials + (int64_t)blockIdx.x * p.rows * R + row0 * R;
      const int nrows = (int)(p.rows - row0 < 32 ? p.rows - row0 : 32);
      if ((R & 3) == 0) {
#pragma unroll
        for (int n = 0; n < 64; n += 4)
          if (n < R)
            *reinterpret_cast<float4*>(stg + lane * 68 + n) =
                make_float4(acc[n], acc[n + 1], acc[n + 2], acc[n + 3]);
        __syncwarp();
        const int r4 = R >> 2;  // float4 per row
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
          if (n < R) stg[lane * 65 + n] = acc[n];
        __syncwarp();
        for (int i = 0; i < nrows; ++i)
          for (int c = lane; c < R; c += 32) out0[(int64_t)i * R + c] = stg[i * 65 + c];
      }
    } else {
      if (lane == 0) atomicOr(p.status, DS_TIMEOUT);
      if (row < p.rows) {
        float* out = p.partials + (int64_t)blockIdx.x * p.rows * R + row * R;
        for (int n = 0; n < R; ++n) out[n] = 0.f;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, (uint32_t)(4 * p.acc_cols));
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn get_encode() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

int make_map(CUtensorMap* map, const __nv_bfloat16* base, int64_t rows, int64_t cols,
             int64_t ld) {
  EncodeTiledFn enc = get_encode();
  if (!enc) return fail(TSR_E_CUDA, "cuTensorMapEncodeTiled unavailable");
  if (((uintptr_t)base & 15) || (ld * 2) % 16)
    return fail(TSR_E_INVALID_ARG, "TMA operand misaligned");
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
  cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)TC_BM};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(TSR_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return TSR_OK;
}

// The unfolding as [rows][runs][L] (run stride L, row stride ld), 64 x 1 x 128
// boxes: a box never crosses into the next run, and its columns at or beyond L
// are filled with zeros. Needs L % 8 == 0 (16-byte run stride).
int make_map_runs(CUtensorMap* map, const __nv_bfloat16* base, int64_t rows, int64_t runs,
                  int64_t L, int64_t ld) {
  EncodeTiledFn enc = get_encode();
  if (!enc) return fail(TSR_E_CUDA, "cuTensorMapEncodeTiled unavailable");
  if (((uintptr_t)base & 15) || (ld * 2) % 16 || (L * 2) % 16)
    return fail(TSR_E_INVALID_ARG, "TMA operand misaligned");
  cuuint64_t dims[3] = {(cuuint64_t)L, (cuuint64_t)runs, (cuuint64_t)rows};
  cuuint64_t strides[2] = {(cuuint64_t)(L * 2), (cuuint64_t)(ld * 2)};
  cuuint32_t box[3] = {(cuuint32_t)TC_BK, 1, (cuuint32_t)TC_BM};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, (void*)base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(TSR_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return TSR_OK;
}

int n_pad_of(int R) { return (int)round_up(R, 16); }

int stages_for(int n_pad) {
  int stage = 2 * A_TILE_BYTES + 2 * n_pad * 128;
  int s = (200 * 1024) / stage;
  return s > 4 ? 4 : s;
}

constexpr int kTcMaxSmem = 227 * 1024;

}  // namespace

void init_tc_attributes() {
  cudaFuncSetAttribute(mttkrp_bf16x3_runs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kTcMaxSmem);
  cudaFuncSetAttribute(mttkrp_bf16x3_kernel<true, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, kTcMaxSmem);
  cudaFuncSetAttribute(mttkrp_bf16x3_kernel<false, false>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, kTcMaxSmem);
}

bool tc_supported(const Unfolding& u, int R) {
  return R >= 1 && n_pad_of(R) <= 256 && u.cols < (int64_t)INT32_MAX && u.rows < INT32_MAX;
}

// Run length of the prefix-scaled kernel for this unfolding and rank, or 0
// when it does not apply.
int tc_run_length(const Unfolding& u, int R) {
  if (u.n_other < 1 || n_pad_of(R) > 64) return 0;
  const int64_t L = u.other_size[u.n_other - 1];
  if (L % 8 != 0 || round_up(L, TC_BK) > TCS_MAX_L) return 0;
  return (int)L;
}

SplitPlan plan_tc(const tsr_ctx* ctx, const Unfolding& u, int R) {
  SplitPlan p;
  const int64_t rows = u.rows, K = u.cols;
  int64_t mt = ceil_div(rows, TC_BM);
  int64_t want = std::max<int64_t>(1, (ctx->sm_count - ctx->reserve_sms) / mt);
  const int L = tc_run_length(u, R);
  if (L > 0) {
    const int64_t runs = K / L;
    int64_t per = ceil_div(runs, std::min<int64_t>(want, runs));
    per = std::min<int64_t>(per, TCS_MAX_RUNS);
    p.k_per_split = per * L;
    p.splits = (int)ceil_div(runs, per);
    p.run_length = L;
    return p;
  }
  int64_t steps = ceil_div(K, TC_BK);
  want = std::min<int64_t>(want, steps);
  int64_t steps_per = ceil_div(steps, want);
  p.k_per_split = steps_per * TC_BK;
  p.splits = (int)ceil_div(K, p.k_per_split);
  return p;
}

int launch_mttkrp_tc(tsr_ctx* ctx, const __nv_bfloat16* hi, const __nv_bfloat16* lo,
                     const Unfolding& u, const KRSpec& kr, const SplitPlan& plan,
                     float* partials, bool a_resident) {
  if (!tc_supported(u, kr.R)) return fail(TSR_E_UNSUPPORTED, "BF16X3 MTTKRP: rank too large");
  CUtensorMap mh, ml;
  if (plan.run_length > 0) {
    TSR_TRY(make_map_runs(&mh, hi, u.rows, u.cols / plan.run_length, plan.run_length, u.ld));
    TSR_TRY(make_map_runs(&ml, lo, u.rows, u.cols / plan.run_length, plan.run_length, u.ld));
    if (plan.run_length != tc_run_length(u, kr.R) || plan.k_per_split % plan.run_length != 0 ||
        plan.k_per_split / plan.run_length > TCS_MAX_RUNS)
      return fail(TSR_E_INVALID_ARG, "BF16X3 MTTKRP: split plan does not match the unfolding");
    TcsParams q;
    q.rows = u.rows;
    q.K = u.cols;
    q.k_per_split = plan.k_per_split;
    q.runs_per_split = (int)(plan.k_per_split / plan.run_length);
    q.L = plan.run_length;
    q.n_pad = n_pad_of(kr.R);
    q.acc_cols = q.n_pad <= 32 ? 32 : 64;
    q.kr = kr;
    q.partials = partials;
    q.status = ctx->d_status;
    const size_t fixed = 1024 + (size_t)ceil_div(q.L, TC_BK) * 2 * q.n_pad * 128 +
                         sizeof(float) * TCS_MAX_RUNS * 64 + 8 * 64 + 16;
    q.stages = (int)std::min<size_t>(4, (kTcMaxSmem - fixed) / (2 * A_TILE_BYTES));
    if (q.stages < 2) return fail(TSR_E_UNSUPPORTED, "MTTKRP stage ring too large");
    const size_t smem = fixed + (size_t)q.stages * 2 * A_TILE_BYTES;
    dim3 grid(plan.splits, (unsigned)ceil_div(u.rows, TC_BM));
    if (grid.y > 65535) return fail(TSR_E_UNSUPPORTED, "MTTKRP grid too large");
    q.a_resident = a_resident ? 1 : 0;
    TSR_CUDA(launch_pdl(mttkrp_bf16x3_runs_kernel, grid, dim3(TC_THREADS), smem, ctx->stream, mh,
                        ml, q));
    ctx->launches++;
    TSR_CUDA(cudaGetLastError());
    return TSR_OK;
  }
  TSR_TRY(make_map(&mh, hi, u.rows, u.cols, u.ld));
  TSR_TRY(make_map(&ml, lo, u.rows, u.cols, u.ld));
  TcParams p;
  p.rows = u.rows;
  p.K = u.cols;
  p.k_per_split = plan.k_per_split;
  p.n_pad = n_pad_of(kr.R);
  p.stages = stages_for(p.n_pad);
  p.acc_cols = 32;
  while (p.acc_cols < p.n_pad) p.acc_cols *= 2;
  p.n_acc = 512 / p.acc_cols;
  if (p.n_acc > 8) p.n_acc = 8;
  p.tmem_cols = p.n_acc * p.acc_cols;
  p.kr = kr;
  p.partials = partials;
  p.status = ctx->d_status;
  bool vec4 = (kr.R % 4) == 0;
  for (int q = 0; q < kr.n_other && vec4; ++q) vec4 = ((uintptr_t)kr.f[q] & 15) == 0;
  size_t stage = 2 * A_TILE_BYTES + 2 * (size_t)p.n_pad * 128;
  size_t smem = 1024 + (size_t)p.stages * stage + 8 * (3 * p.stages + 1) + 16;
  dim3 grid(plan.splits, (unsigned)ceil_div(u.rows, TC_BM));
  if (grid.y > 65535) return fail(TSR_E_UNSUPPORTED, "MTTKRP grid too large");
  if (smem > kTcMaxSmem) return fail(TSR_E_UNSUPPORTED, "MTTKRP stage ring too large");
  const bool fast = vec4 && p.n_pad <= 64 && kr.n_other <= 2;
  if (fast)
    mttkrp_bf16x3_kernel<true, true><<<grid, TC_THREADS, smem, ctx->stream>>>(mh, ml, p);
  else
    mttkrp_bf16x3_kernel<false, false><<<grid, TC_THREADS, smem, ctx->stream>>>(mh, ml, p);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

}  // namespace tsr

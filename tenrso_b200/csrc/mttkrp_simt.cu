// Dense MTTKRP, FP32 SIMT path: M = X_(n) . KR with the unfolding X_(n)
// (I_n x K, row stride ld) resident in HBM and the KR rows generated into
// shared memory per K-step. Split-K over the grid: each CTA owns a K range
// and writes a partial I_n x R tile; the partials are summed in a fixed order
// (deterministic) by the consumer (the ALS solve, or mttkrp_reduce_kernel).
//
// Replaces the i/r/j triple loop of crates/tenrso-kernels/src/mttkrp.rs:135-143
// (same sum, different association: per-split partial sums, then a sum over
// splits).
#include <algorithm>

#include "kr.cuh"
#include "mttkrp.cuh"

namespace tsr {

namespace {
constexpr int BK = 32;

template <int BM, int BN>
constexpr int simt_threads() {
  return (BM / 8) * (BN / 4);
}
template <int BM, int BN>
constexpr int simt_min_blocks() {
  return 512 / simt_threads<BM, BN>() > 4 ? 4 : 512 / simt_threads<BM, BN>();
}

// BM x BN output tile per CTA, 8 x 4 per thread; NPF factor rows of each KR
// row are loaded one K-step ahead (the rest, for tensors of more than NPF + 1
// modes, after the FMA loop).
template <int BM, int BN, int NPF>
__global__ void __launch_bounds__(simt_threads<BM, BN>(), simt_min_blocks<BM, BN>())
mttkrp_f32_splitk_kernel(const float* __restrict__ A, int64_t rows, int64_t K, int64_t ld,
                         KRSpec kr, int64_t k_per_split, float* __restrict__ partials) {
  constexpr int NT = simt_threads<BM, BN>();
  constexpr int A_IT = BM * BK / 4 / NT;  // float4 of the A tile per thread
  constexpr int B_TPR = BN / 8;            // threads per KR row (8 columns each)
  constexpr int B_RPP = NT / B_TPR;        // KR rows per pass
  constexpr int B_IT = BK / B_RPP;         // passes per K-step
  static_assert(B_IT >= 1 && BK % B_RPP == 0, "tile");
  extern __shared__ __align__(16) float simt_smem[];
  float(*As)[BK][BM + 4] = reinterpret_cast<float(*)[BK][BM + 4]>(simt_smem);
  float(*Bs)[BK][BN] = reinterpret_cast<float(*)[BK][BN]>(simt_smem + 2 * BK * (BM + 4));
  const int tid = threadIdx.x;
  const int tx = tid % (BN / 4), ty = tid / (BN / 4);
  const int64_t m0 = (int64_t)blockIdx.y * BM;
  const int n0 = blockIdx.z * BN;
  const int R = kr.R;
  const int64_t kbeg = (int64_t)blockIdx.x * k_per_split;
  const int64_t kend = min(K, kbeg + k_per_split);
  const int nsteps = (int)((kend - kbeg + BK - 1) / BK);

  float acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;

  float4 areg[A_IT];
  float breg[B_IT][8];
  // A-tile mapping: 8 threads per row (32 floats = 128 B).
  auto load_a = [&](int64_t k0) {
#pragma unroll
    for (int it = 0; it < A_IT; ++it) {
      int idx = it * NT + tid;
      int m = idx / 8, kq = idx % 8;
      int64_t gm = m0 + m, gk = k0 + kq * 4;
      if (gm < rows && gk < kend)
        areg[it] = __ldg(reinterpret_cast<const float4*>(A + gm * ld + gk));
      else
        areg[it] = make_float4(0.f, 0.f, 0.f, 0.f);
      // columns past kend inside the same float4 belong to the next split
      if (gm < rows && gk < kend && gk + 4 > kend) {
        float* p = reinterpret_cast<float*>(&areg[it]);
        for (int e = (int)(kend - gk); e < 4; ++e) p[e] = 0.f;
      }
    }
  };
  auto store_a = [&](int buf) {
#pragma unroll
    for (int it = 0; it < A_IT; ++it) {
      int idx = it * NT + tid;
      int m = idx / 8, kq = idx % 8;
      As[buf][kq * 4 + 0][m] = areg[it].x;
      As[buf][kq * 4 + 1][m] = areg[it].y;
      As[buf][kq * 4 + 2][m] = areg[it].z;
      As[buf][kq * 4 + 3][m] = areg[it].w;
    }
  };
  // B-tile mapping: thread -> (KR row kk, 8 consecutive columns). The factor
  // values of the next K-step are loaded before the FMA loop of the current
  // one and multiplied after it, so the L2 latency overlaps the math.
  float braw[B_IT][NPF][8];
  uint32_t boff[B_IT][kMaxModes];
  bool bvalid[B_IT];
  auto gen_b_load = [&](int64_t k0) {
#pragma unroll
    for (int bi = 0; bi < B_IT; ++bi) {
      const int kk = bi * B_RPP + tid / B_TPR, c0 = (tid % B_TPR) * 8;
      const int64_t j = k0 + kk;
      bvalid[bi] = j < kend;
      kr_row_offsets(kr, (uint32_t)(bvalid[bi] ? j : kbeg), boff[bi]);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int c = n0 + c0 + e;
        const int cc = c < R ? c : 0;
#pragma unroll
        for (int q = 0; q < NPF; ++q)
          braw[bi][q][e] = q < kr.n_other ? __ldg(kr.f[q] + boff[bi][q] + cc) : 1.f;
      }
    }
  };
  auto gen_b_finish = [&]() {
#pragma unroll
    for (int bi = 0; bi < B_IT; ++bi) {
      const int c0 = (tid % B_TPR) * 8;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int c = n0 + c0 + e;
        float v = braw[bi][0][e];
#pragma unroll
        for (int q = 1; q < NPF; ++q) v *= braw[bi][q][e];
#pragma unroll
        for (int q = NPF; q < kMaxModes; ++q)
          if (q < kr.n_other) v *= __ldg(kr.f[q] + boff[bi][q] + (c < R ? c : 0));
        breg[bi][e] = (bvalid[bi] && c < R) ? v : 0.f;
      }
    }
  };
  auto store_b = [&](int buf) {
#pragma unroll
    for (int bi = 0; bi < B_IT; ++bi) {
      const int kk = bi * B_RPP + tid / B_TPR, c0 = (tid % B_TPR) * 8;
      *reinterpret_cast<float4*>(&Bs[buf][kk][c0]) =
          make_float4(breg[bi][0], breg[bi][1], breg[bi][2], breg[bi][3]);
      *reinterpret_cast<float4*>(&Bs[buf][kk][c0 + 4]) =
          make_float4(breg[bi][4], breg[bi][5], breg[bi][6], breg[bi][7]);
    }
  };

  if (nsteps > 0) {
    load_a(kbeg);
    gen_b_load(kbeg);
    gen_b_finish();
    store_a(0);
    store_b(0);
  }
  __syncthreads();
  for (int s = 0; s < nsteps; ++s) {
    const int buf = s & 1;
    const bool more = s + 1 < nsteps;
    if (more) {
      load_a(kbeg + (int64_t)(s + 1) * BK);
      gen_b_load(kbeg + (int64_t)(s + 1) * BK);
    }
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 8]);
      float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 8 + 4]);
      float4 b = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
      float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    if (more) {
      gen_b_finish();
      store_a(buf ^ 1);
      store_b(buf ^ 1);
    }
    __syncthreads();
  }

  float* P = partials + (int64_t)blockIdx.x * rows * R;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int64_t gm = m0 + ty * 8 + i;
    if (gm >= rows) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int c = n0 + tx * 4 + j;
      if (c < R) P[gm * R + c] = acc[i][j];
    }
  }
}

// Run-scaled FP32 form (the unfolding's columns come in runs of L, the size
// of the fastest other mode): the Khatri-Rao rows of run P are U_last scaled
// column-wise by w_P, the product of the slower modes' factor rows, so
//   M = sum_P (X_P . U_last) diag(w_P)
// with X_P the L columns of run P. U_last (L x BN) stays in shared memory for
// the CTA's whole range of runs; no Khatri-Rao row is formed. The X tiles
// (128 rows x 32 columns) stream in through cp.async, double-buffered. Each
// thread owns rows ty + TY i and 4 columns; a run's products collect in
// `acc`, which is scaled by w_P into `tot` where the run (or the CTA's range)
// ends. The split-K ranges are counted in 32-column steps over all runs, so
// the CTAs get equal work whether or not the runs divide evenly.
constexpr int RUN_BM = 128, RUN_PITCH = 36;  // A tile rows, floats per staged row
constexpr int kRunMaxSmem = 110 * 1024;      // two CTAs per SM

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 16 : 0;  // 0: zero-fill the 16 bytes
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int BN>
__global__ void __launch_bounds__(256, 2)
mttkrp_f32_runs_kernel(const float* __restrict__ A, int64_t rows, int64_t ld, int L, int Lp,
                       int64_t n_runs, int64_t steps_per_split, KRSpec kr,
                       const float* __restrict__ UL, float* __restrict__ partials) {
  constexpr int TX = BN / 4, TY = 256 / TX, RPT = RUN_BM / TY;
  extern __shared__ __align__(16) float run_smem[];
  float* Us = run_smem;                                   // Lp x BN
  float (*As)[RUN_BM][RUN_PITCH] =
      reinterpret_cast<float (*)[RUN_BM][RUN_PITCH]>(run_smem + (size_t)Lp * BN);
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int64_t m0 = (int64_t)blockIdx.y * RUN_BM;
  const int n0 = blockIdx.z * BN;
  const int R = kr.R;
  const int steps_per_run = Lp / 32;
  const int64_t g_begin = (int64_t)blockIdx.x * steps_per_split;
  const int64_t g_end = min(n_runs * steps_per_run, g_begin + steps_per_split);
  // U_last's columns n0..n0+BN-1, zero past L and past R
  for (int e = tid; e < Lp * BN; e += 256) {
    const int k = e / BN, c = e % BN;
    Us[e] = (k < L && n0 + c < R) ? __ldg(UL + (int64_t)k * R + n0 + c) : 0.f;
  }
  // global step g's tile: 128 rows x 32 columns of run g / steps_per_run
  auto issue = [&](int64_t g, int buf) {
    const int64_t P = g / steps_per_run;
    const int k0 = (int)(g % steps_per_run) * 32;
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      const int idx = it * 256 + tid, r = idx / 8, kq = idx % 8;
      const int64_t gm = m0 + r;
      const int k = k0 + kq * 4;
      const bool ok = gm < rows && k < L;
      cp_async16(&As[buf][r][kq * 4], ok ? A + gm * ld + P * L + k : A, ok);
    }
    cp_async_commit();
  };
  float tot[RPT][4], acc[RPT][4];
#pragma unroll
  for (int i = 0; i < RPT; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) tot[i][j] = acc[i][j] = 0.f;
  float w[4] = {0.f, 0.f, 0.f, 0.f};
  if (g_begin < g_end) issue(g_begin, 0);
  for (int64_t g = g_begin; g < g_end; ++g) {
    const int buf = (int)((g - g_begin) & 1);
    const int kstep = (int)(g % steps_per_run);
    if (kstep == 0 || g == g_begin) {
      // this run's weights: the slower modes' factor rows
      const int64_t P = g / steps_per_run;
      uint32_t off[kMaxModes];
      kr_row_offsets(kr, (uint32_t)(P * L), off);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = n0 + tx * 4 + j;
        float v = c < R ? 1.f : 0.f;
#pragma unroll
        for (int q = 0; q < kMaxModes - 1; ++q)
          if (q < kr.n_other - 1 && c < R) v *= __ldg(kr.f[q] + off[q] + c);
        w[j] = v;
      }
    }
    if (g + 1 < g_end) {
      issue(g + 1, buf ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const float* ub = Us + (size_t)kstep * 32 * BN + tx * 4;
#pragma unroll 2
    for (int kq = 0; kq < 8; ++kq) {
      float4 a[RPT];
#pragma unroll
      for (int i = 0; i < RPT; ++i)
        a[i] = *reinterpret_cast<const float4*>(&As[buf][ty + TY * i][kq * 4]);
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const float4 b = *reinterpret_cast<const float4*>(ub + (kq * 4 + t) * BN);
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
          const float av = t == 0 ? a[i].x : (t == 1 ? a[i].y : (t == 2 ? a[i].z : a[i].w));
          acc[i][0] = fmaf(av, b.x, acc[i][0]);
          acc[i][1] = fmaf(av, b.y, acc[i][1]);
          acc[i][2] = fmaf(av, b.z, acc[i][2]);
          acc[i][3] = fmaf(av, b.w, acc[i][3]);
        }
      }
    }
    __syncthreads();  // the buffer is refilled two steps on
    if (kstep == steps_per_run - 1 || g + 1 == g_end) {
#pragma unroll
      for (int i = 0; i < RPT; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          tot[i][j] = fmaf(acc[i][j], w[j], tot[i][j]);
          acc[i][j] = 0.f;
        }
    }
  }
  float* P = partials + (int64_t)blockIdx.x * rows * R;
#pragma unroll
  for (int i = 0; i < RPT; ++i) {
    const int64_t gm = m0 + ty + TY * i;
    if (gm >= rows) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = n0 + tx * 4 + j;
      if (c < R) P[gm * R + c] = tot[i][j];
    }
  }
}

// out[e] = sum over splits of partials[s][e] (FP64), optionally times w[e % R].
// `groups` threads share an element, each summing every groups-th split with
// four loads in flight; the groups combine through shared memory.
__global__ void __launch_bounds__(256)
mttkrp_reduce_kernel(const float* __restrict__ partials, int splits, int64_t n, int groups,
                     int R, const float* __restrict__ w, float* __restrict__ out) {
  __shared__ double red[256];
  const int per = 256 / groups;
  const int g = threadIdx.x / per, l = threadIdx.x % per;
  const int64_t k = (int64_t)blockIdx.x * per + l;
  double s = 0.0;
  if (k < n) {
    const float* p = partials + k;
    int q = g;
    for (; q + 3 * groups < splits; q += 4 * groups) {
      const float v0 = __ldg(p + (int64_t)q * n);
      const float v1 = __ldg(p + (int64_t)(q + groups) * n);
      const float v2 = __ldg(p + (int64_t)(q + 2 * groups) * n);
      const float v3 = __ldg(p + (int64_t)(q + 3 * groups) * n);
      s += ((double)v0 + (double)v1) + ((double)v2 + (double)v3);
    }
    for (; q < splits; q += groups) s += (double)__ldg(p + (int64_t)q * n);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  if (g != 0 || k >= n) return;
  for (int j = 1; j < groups; ++j) s += red[j * per + l];
  if (w) s *= (double)__ldg(w + (int)(k % R));
  out[k] = (float)s;
}

// khatri_rao.rs:56-89: C[a*J + b, k] = A[a, k] * B[b, k].
__global__ void khatri_rao_kernel(const float* __restrict__ A, int64_t I,
                                  const float* __restrict__ B, int64_t J, int64_t K,
                                  float* __restrict__ C) {
  int64_t n = I * J * K;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t k = e % K, row = e / K;
    int64_t a = row / J, b = row % J;
    C[e] = __ldg(A + a * K + k) * __ldg(B + b * K + k);
  }
}
}  // namespace

int launch_khatri_rao(tsr_ctx* ctx, const float* A, int64_t I, const float* B, int64_t J,
                      int64_t K, float* C) {
  int64_t n = I * J * K;
  unsigned grid = (unsigned)std::min<int64_t>(ceil_div(n, 256), (int64_t)ctx->sm_count * 8);
  khatri_rao_kernel<<<grid, 256, 0, ctx->stream>>>(A, I, B, J, K, C);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

template <int BM, int BN>
constexpr size_t simt_smem_bytes() {
  return sizeof(float) * 2 * BK * (BM + 4 + BN);
}

void init_simt_attributes() {
  cudaFuncSetAttribute(mttkrp_f32_runs_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kRunMaxSmem);
  cudaFuncSetAttribute(mttkrp_f32_runs_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kRunMaxSmem);
  cudaFuncSetAttribute(mttkrp_f32_splitk_kernel<128, 64, 2>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)simt_smem_bytes<128, 64>());
  cudaFuncSetAttribute(mttkrp_f32_splitk_kernel<128, 64, 4>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)simt_smem_bytes<128, 64>());
  cudaFuncSetAttribute(mttkrp_f32_splitk_kernel<128, 32, 2>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)simt_smem_bytes<128, 32>());
  cudaFuncSetAttribute(mttkrp_f32_splitk_kernel<128, 32, 4>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)simt_smem_bytes<128, 32>());
}

// Shared memory of the run-scaled kernel: U_last (Lp x BN) and two A tiles.
template <int BN>
constexpr size_t runs_smem_bytes(int Lp) {
  return sizeof(float) * ((size_t)Lp * BN + 2 * RUN_BM * RUN_PITCH);
}

bool simt_runs_ok(int64_t L, int64_t K, int R) {
  if (L < 16 || L % 4 != 0 || K % L != 0 || R < 1 || R > 64) return false;
  const int64_t Lp = round_up(L, 32);
  const size_t smem = R <= 32 ? runs_smem_bytes<32>((int)Lp) : runs_smem_bytes<64>((int)Lp);
  return smem <= (size_t)kRunMaxSmem;
}

SplitPlan plan_simt(const tsr_ctx* ctx, int64_t rows, int64_t K, int R, int64_t L) {
  SplitPlan p;
  p.bn = R <= 32 ? 32 : 64;
  if (L > 0 && simt_runs_ok(L, K, R)) {
    // equal ranges of 32-column steps (k_per_split counts steps here), one
    // full wave at two CTAs per SM
    const int64_t mt = ceil_div(rows, RUN_BM), nt = ceil_div(R, p.bn);
    const int64_t steps = (K / L) * (round_up(L, 32) / 32);
    // rounded up (a grid short of the unreserved slots leaves SMs idle), but
    // within the physical slots so that the grid stays one wave
    const int64_t tiles = mt * nt;
    const int64_t want = std::max<int64_t>(
        1, std::min<int64_t>({steps,
                              ceil_div((int64_t)(ctx->sm_count - ctx->reserve_sms) * 2, tiles),
                              (int64_t)ctx->sm_count * 2 / tiles}));
    const int64_t per = ceil_div(steps, want);
    p.run_length = (int)L;
    p.k_per_split = per;
    p.splits = (int)ceil_div(steps, per);
    return p;
  }
  const int64_t mt = ceil_div(rows, 128), nt = ceil_div(R, p.bn);
  // one full wave at the resident CTAs per SM (2 of 256 threads, 4 of 128)
  const int per_sm = p.bn == 32 ? 4 : 2;
  int64_t want =
      std::max<int64_t>(1, (int64_t)(ctx->sm_count - ctx->reserve_sms) * per_sm / (mt * nt));
  int64_t steps = ceil_div(K, BK);
  want = std::min<int64_t>(want, steps);
  p.k_per_split = round_up(ceil_div(K, want), BK);
  p.splits = (int)ceil_div(K, p.k_per_split);
  return p;
}

template <int BM, int BN, int NPF>
void launch_simt_tile(tsr_ctx* ctx, const float* A, const Unfolding& u, const KRSpec& kr,
                      const SplitPlan& plan, float* partials, dim3 grid) {
  mttkrp_f32_splitk_kernel<BM, BN, NPF>
      <<<grid, simt_threads<BM, BN>(), simt_smem_bytes<BM, BN>(), ctx->stream>>>(
          A, u.rows, u.cols, u.ld, kr, plan.k_per_split, partials);
}

int launch_mttkrp_simt(tsr_ctx* ctx, const float* A, const Unfolding& u, const KRSpec& kr,
                       const SplitPlan& plan, float* partials) {
  if (u.cols >= (int64_t)UINT32_MAX) return fail(TSR_E_UNSUPPORTED, "unfolding too wide");
  if (plan.run_length > 0) {
    // 16-byte cp.async sources need an aligned base and row stride (the plan
    // only selects this kernel for such operands)
    if (((uintptr_t)A & 15) != 0 || (u.ld & 3) != 0)
      return fail(TSR_E_INVALID_ARG, "run-scaled FP32 MTTKRP needs 16-byte aligned rows");
    const int L = plan.run_length, Lp = (int)round_up(L, 32);
    const int64_t runs = u.cols / L;
    const int64_t per = plan.k_per_split;  // 32-column steps per split
    const int bn = plan.bn == 32 ? 32 : 64;
    dim3 grid(plan.splits, (unsigned)ceil_div(u.rows, RUN_BM), (unsigned)ceil_div(kr.R, bn));
    if (grid.y > 65535 || grid.z > 65535) return fail(TSR_E_UNSUPPORTED, "MTTKRP grid too large");
    if (bn == 32)
      mttkrp_f32_runs_kernel<32><<<grid, 256, runs_smem_bytes<32>(Lp), ctx->stream>>>(
          A, u.rows, u.ld, L, Lp, runs, per, kr, kr.f[kr.n_other - 1], partials);
    else
      mttkrp_f32_runs_kernel<64><<<grid, 256, runs_smem_bytes<64>(Lp), ctx->stream>>>(
          A, u.rows, u.ld, L, Lp, runs, per, kr, kr.f[kr.n_other - 1], partials);
    ctx->launches++;
    TSR_CUDA(cudaGetLastError());
    return TSR_OK;
  }
  const int bn = plan.bn == 32 ? 32 : 64;
  dim3 grid(plan.splits, (unsigned)ceil_div(u.rows, 128), (unsigned)ceil_div(kr.R, bn));
  if (grid.y > 65535 || grid.z > 65535) return fail(TSR_E_UNSUPPORTED, "MTTKRP grid too large");
  const bool wide = kr.n_other > 2;
  if (bn == 32) {
    if (wide) launch_simt_tile<128, 32, 4>(ctx, A, u, kr, plan, partials, grid);
    else launch_simt_tile<128, 32, 2>(ctx, A, u, kr, plan, partials, grid);
  } else {
    if (wide) launch_simt_tile<128, 64, 4>(ctx, A, u, kr, plan, partials, grid);
    else launch_simt_tile<128, 64, 2>(ctx, A, u, kr, plan, partials, grid);
  }
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_mttkrp_reduce_scaled(tsr_ctx* ctx, const float* partials, int splits, int64_t rows,
                                int R, const float* w, float* out) {
  const int64_t n = rows * R;
  if (n == 0) return TSR_OK;
  int groups = 1;
  while (groups < 8 && 2 * groups <= splits) groups *= 2;
  const int per = 256 / groups;
  mttkrp_reduce_kernel<<<(unsigned)ceil_div(n, per), 256, 0, ctx->stream>>>(
      partials, splits, n, groups, R > 0 ? R : 1, w, out);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_mttkrp_reduce(tsr_ctx* ctx, const float* partials, int splits, int64_t n, float* out) {
  return launch_mttkrp_reduce_scaled(ctx, partials, splits, n, 1, nullptr, out);
}

}  // namespace tsr

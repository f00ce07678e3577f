// Accelerated CP-ALS: tenrso_decomp::cp_als_accelerated (cp/advanced.rs:51-213)
// with its line search line_search_cp (cp/helpers.rs:130-189) on the GPU.
//
// Per mode n of a sweep the reference solves U_new = M G^-1 as cp_als does,
// then evaluates the fit of five trial factors prev + a (U_new - prev),
// a in {0.25, 0.5, 0.75, 1, 1.25}, prev being U_n before its previous update,
// keeps the first a with the best fit, and from the second iteration on
// extrapolates U_n = U_new + a * alpha * (U_new - prev).
//
// The trial tensors differ from the current model in mode n only, so each
// trial fit needs no MTTKRP of its own: with d = U_new - prev, M the mode-n
// MTTKRP of the current factors and G the Hadamard of the other Grams,
//   <X, Xhat(a)>  = <M, prev> + a <M, d>
//   ||Xhat(a)||^2 = <G, prev^T prev> + 2a <G, prev^T d> + a^2 <G, d^T d>
// (the same identities compute_fit evaluates, helpers.rs:513-579, written
// for a one-factor change). The five scalars are FP64 sums formed in the
// solve pass; every CTA of the apply pass then forms the five fits, picks a,
// writes the final factor, its Gram and, for the last mode, <M, U_n>.
//
// Kernels per mode: MTTKRP (the dense kernels) -> inverse (als.cu) ->
// accel_solve -> accel_apply; after the sweep accel_fit applies the fit,
// the adaptive alpha and the stopping rules of advanced.rs:158-190.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>

#include "als.cuh"
#include "dense.cuh"

namespace tsr {

namespace {

// Device-side state of the accelerated run.
struct AccelState {
  double sums[5];      // <M,prev>, <M,d>, <G,prev'prev>, <G,prev'd>, <G,d'd> of this mode
  double inner;        // <M_last, U_last> of the sweep (after extrapolation)
  double alpha;        // adaptive extrapolation strength
  double prev_fit;
  double fit;
  double final_change;
  int iter;            // iterations completed
  int osc;
  int reason;
  int done;
};

__constant__ double kAlphas[5] = {0.25, 0.5, 0.75, 1.0, 1.25};

// U_new = (sum of partials) G^-1 rounded to fp32 (into unew; M kept in FP64
// in mbuf), and this CTA's share of the five line-search sums into st->sums.
// One row per warp at a time; lane l holds columns l + 32q (q < 4, R <= 112).
__global__ void __launch_bounds__(256)
accel_solve_kernel(const float* __restrict__ partials, int splits, int64_t rows, int R,
                   const double* __restrict__ ginv, const double* __restrict__ G,
                   const float* __restrict__ prev, float* __restrict__ unew,
                   double* __restrict__ mbuf, AccelState* st, const AlsState* als) {
  extern __shared__ __align__(16) double sh[];
  if (als->done || st->done) return;
  double* Gi = sh;            // R x R
  double* Gs = Gi + R * R;    // R x R (the Hadamard G)
  double* red = Gs + R * R;   // [8 warps][5]
  for (int e = threadIdx.x; e < R * R; e += blockDim.x) {
    Gi[e] = ginv[e];
    Gs[e] = G[e];
  }
  __syncthreads();
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const int64_t pstride = rows * R;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t i = (int64_t)blockIdx.x * 8 + warp; i < rows; i += (int64_t)gridDim.x * 8) {
    double m[4], u[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = lane + 32 * q;
      m[q] = u[q] = 0.0;
      if (c < R) {
        double a = 0.0;
        for (int p = 0; p < splits; ++p)
          a += (double)__ldg(partials + (int64_t)p * pstride + i * R + c);
        m[q] = a;
        mbuf[i * R + c] = a;
      }
    }
    // U_new[i, c] = sum_k M[i, k] Gi[k, c], M[i, k] broadcast from its lane
#pragma unroll
    for (int qk = 0; qk < 4; ++qk) {
      if (32 * qk >= R) break;
      for (int t = 0; t < 32 && 32 * qk + t < R; ++t) {
        const int k = 32 * qk + t;
        const double mk = __shfl_sync(0xffffffffu, m[qk], t);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int c = lane + 32 * q;
          if (c < R) u[q] = fma(mk, Gi[k * R + c], u[q]);
        }
      }
    }
    double pv[4], dv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = lane + 32 * q;
      pv[q] = dv[q] = 0.0;
      if (c < R) {
        const float un = (float)u[q];
        const float p = __ldg(prev + i * R + c);
        unew[i * R + c] = un;
        pv[q] = (double)p;
        dv[q] = (double)(un - p);  // the difference in the factors' type (helpers.rs:170)
        s[0] += m[q] * pv[q];
        s[1] += m[q] * dv[q];
      }
    }
    // the row's quadratic forms with G: prev G prev', prev G d', d G d'
#pragma unroll
    for (int qk = 0; qk < 4; ++qk) {
      if (32 * qk >= R) break;
      for (int t = 0; t < 32 && 32 * qk + t < R; ++t) {
        const int k = 32 * qk + t;
        const double pk = __shfl_sync(0xffffffffu, pv[qk], t);
        const double dk = __shfl_sync(0xffffffffu, dv[qk], t);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int c = lane + 32 * q;
          if (c < R) {
            const double g = Gs[k * R + c];
            const double gp = g * pv[q], gd = g * dv[q];
            s[2] = fma(pk, gp, s[2]);
            s[3] = fma(pk, gd, s[3]);
            s[4] = fma(dk, gd, s[4]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 5; ++j)
    for (int o = 16; o > 0; o >>= 1) s[j] += __shfl_down_sync(0xffffffffu, s[j], o);
  if (lane == 0)
    for (int j = 0; j < 5; ++j) red[warp * 5 + j] = s[j];
  __syncthreads();
  if (threadIdx.x < 5) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red[w * 5 + threadIdx.x];
    atomicAdd(&st->sums[threadIdx.x], t);
  }
}

// The step chosen by line_search_cp from the five sums (every CTA computes the
// same value): the fits of helpers.rs:513-530, the first best kept.
__device__ double line_search_step(const AccelState* st, double xn) {
  const double s0 = st->sums[0], s1 = st->sums[1];
  const double q1 = st->sums[2], q2 = st->sums[3], q3 = st->sums[4];
  double best_a = 1.0, best_fit = -INFINITY;
  for (int j = 0; j < 5; ++j) {
    const double a = kAlphas[j];
    const double inner = s0 + a * s1;
    const double xh = q1 + 2.0 * a * q2 + a * a * q3;
    const double err = sqrt(fmax(xn + xh - 2.0 * inner, 0.0));
    double fit = 1.0 - err / sqrt(xn);
    fit = fmin(fmax(fit, 0.0), 1.0);
    if (fit > best_fit) {
      best_fit = fit;
      best_a = a;
    }
  }
  return best_a;
}

// Final factor, prev update, Gram of the final factor (upper triangle, FP64
// atomics into gram, zeroed by the inverse kernel of this mode), <M, U> and,
// when bimg is set, the factor's B image for the single-layout MTTKRP.
template <int RB>
__global__ void __launch_bounds__(256)
accel_apply_kernel(int64_t rows, int R, const float* __restrict__ unew,
                   const double* __restrict__ mbuf, float* __restrict__ U,
                   float* __restrict__ prev, double* __restrict__ gram, AccelState* st,
                   const AlsState* als, double xn, int last, uint8_t* __restrict__ bimg,
                   int img_n_pad) {
  extern __shared__ __align__(16) double sh[];
  if (als->done || st->done) return;
  const double a_ls = line_search_step(st, xn);
  // advanced.rs:137-147: no extrapolation in the first iteration
  const float step = st->iter > 0 ? (float)a_ls * (float)st->alpha : 0.f;
  const int rpc = 16;
  double* Us = sh;  // rpc x R
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[RB][RB];
#pragma unroll
  for (int ai = 0; ai < RB; ++ai)
#pragma unroll
    for (int bj = 0; bj < RB; ++bj) acc[ai][bj] = 0.0;
  double ip = 0.0;
  for (int64_t r0 = (int64_t)blockIdx.x * rpc; r0 < rows; r0 += (int64_t)gridDim.x * rpc) {
    const int nr = (int)(rows - r0 < rpc ? rows - r0 : rpc);
    __syncthreads();
    for (int e = threadIdx.x; e < nr * R; e += blockDim.x) {
      const int64_t g = r0 * R + e;
      const float n = unew[g], p = prev[g];
      const float v = step != 0.f ? n + step * (n - p) : n;
      prev[g] = U[g];  // the factor before this update (advanced.rs:150)
      U[g] = v;
      Us[e] = (double)v;
      if (last) ip += mbuf[g] * (double)v;
      if (bimg) {
        const int64_t k = r0 + e / R;
        const int c = e % R;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
        uint8_t* tile = bimg + (size_t)(k >> 6) * 2 * img_n_pad * 128;
        const int cq = (int)((k & 63) >> 3), el = (int)(k & 7) * 2;
        const int rh = c, rl = img_n_pad + c;
        *reinterpret_cast<__nv_bfloat16*>(tile + rh * 128 + ((cq ^ (rh & 7)) << 4) + el) = h;
        *reinterpret_cast<__nv_bfloat16*>(tile + rl * 128 + ((cq ^ (rl & 7)) << 4) + el) = l;
      }
    }
    __syncthreads();
    for (int i = 0; i < nr; ++i) {
      double x[RB], y[RB];
#pragma unroll
      for (int ai = 0; ai < RB; ++ai) x[ai] = ty + 16 * ai < R ? Us[i * R + ty + 16 * ai] : 0.0;
#pragma unroll
      for (int bj = 0; bj < RB; ++bj) y[bj] = tx + 16 * bj < R ? Us[i * R + tx + 16 * bj] : 0.0;
#pragma unroll
      for (int ai = 0; ai < RB; ++ai)
#pragma unroll
        for (int bj = 0; bj < RB; ++bj) acc[ai][bj] = fma(x[ai], y[bj], acc[ai][bj]);
    }
  }
#pragma unroll
  for (int ai = 0; ai < RB; ++ai)
#pragma unroll
    for (int bj = 0; bj < RB; ++bj) {
      const int a = ty + 16 * ai, c = tx + 16 * bj;
      if (a < R && c < R && c >= a) atomicAdd(gram + a * R + c, acc[ai][bj]);
    }
  if (last) {
    for (int o = 16; o > 0; o >>= 1) ip += __shfl_down_sync(0xffffffffu, ip, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&st->inner, ip);
  }
}

// After the sweep: fit (helpers.rs:513-530 from ||X||^2, the Grams and
// <M_last, U_last>), the adaptive alpha and the stopping rules of
// advanced.rs:158-190. One warp.
__global__ void accel_fit_kernel(const double* __restrict__ grams, int ndim, int R, double xn,
                                 double tol, AccelState* st, const AlsState* als,
                                 double* history) {
  if (als->done || st->done) return;
  double x = 0.0;
  for (int e = threadIdx.x; e < R * R; e += 32) {
    const int i = e / R, j = e % R;
    double h = 1.0;
    for (int m = 0; m < ndim; ++m) h *= grams[(size_t)m * R * R + (i <= j ? i * R + j : j * R + i)];
    x += h;
  }
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  if (threadIdx.x != 0) return;
  const double err = sqrt(fmax(xn + x - 2.0 * st->inner, 0.0));
  double fit = fmin(fmax(1.0 - err / sqrt(xn), 0.0), 1.0);
  const int it = st->iter;
  st->fit = fit;
  history[it] = fit;
  st->iter = it + 1;
  if (it > 0) {
    if (fit > st->prev_fit) {
      st->alpha = fmin(st->alpha * 1.05, 0.9);
    } else {
      st->alpha = fmax(st->alpha * 0.7, 0.1);
      st->osc += 1;
      if (st->osc > 5 && it > 10) {
        st->reason = TSR_REASON_OSCILLATION;
        st->done = 1;
        return;
      }
    }
    const double change = fabs(fit - st->prev_fit);
    st->final_change = change;
    if (change / (fabs(st->prev_fit) + 1e-10) < tol) {
      st->reason = TSR_REASON_FIT_TOLERANCE;
      st->done = 1;
      return;
    }
  }
  st->prev_fit = fit;
}

int launch_accel_solve(tsr_ctx* ctx, const float* partials, int splits, int64_t rows, int R,
                       const double* ginv, const double* G, const float* prev, float* unew,
                       double* mbuf, AccelState* st, const AlsState* als) {
  const unsigned grid = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(ceil_div(rows, 8), 4 * (int64_t)ctx->sm_count));
  const size_t smem = sizeof(double) * (2 * (size_t)R * R + 8 * 5);
  accel_solve_kernel<<<grid, 256, smem, ctx->stream>>>(partials, splits, rows, R, ginv, G,
                                                          prev, unew, mbuf, st, als);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_accel_apply(tsr_ctx* ctx, int64_t rows, int R, const float* unew, const double* mbuf,
                       float* U, float* prev, double* gram, AccelState* st, const AlsState* als,
                       double xn, bool last, uint8_t* bimg, int img_n_pad) {
  const unsigned grid = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(ceil_div(rows, 16), 2 * (int64_t)ctx->sm_count));
  const size_t smem = sizeof(double) * 16 * R;
#define TSR_APPLY(RB)                                                                      \
  accel_apply_kernel<RB><<<grid, 256, smem, ctx->stream>>>(rows, R, unew, mbuf, U, prev, gram, \
                                                           st, als, xn, last ? 1 : 0, bimg, \
                                                           img_n_pad)
  switch ((R + 15) / 16) {
    case 1: TSR_APPLY(1); break;
    case 2: TSR_APPLY(2); break;
    case 3: TSR_APPLY(3); break;
    case 4: TSR_APPLY(4); break;
    case 5: TSR_APPLY(5); break;
    case 6: TSR_APPLY(6); break;
    default: TSR_APPLY(7); break;
  }
#undef TSR_APPLY
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

}  // namespace

// cp_als_accelerated on a device-resident tensor (advanced.rs:51-213).
int cp_als_accelerated_device(tsr_ctx* ctx, const float* dX, int ndim, const int64_t* shape,
                              int64_t rank, int max_iters, double tol, const float* d_init,
                              int precision, double time_limit_s, float* d_out,
                              tsr_cp_info* info) {
  const auto t_start = std::chrono::steady_clock::now();
  // advanced.rs:71-77
  if (rank == 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  if (!(tol > 0.0 && tol < 1.0)) return fail(TSR_E_INVALID_TOL, "Invalid tolerance: %g", tol);
  // no rank <= mode size check: InitStrategy::Random accepts any rank
  // (helpers.rs:214-222) and a rank-deficient Gram takes the ridge retry
  if (ndim < 2 || ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "accelerated CP-ALS needs 2..%d modes", kMaxModes);
  TSR_TRY(check_sizes(ndim, shape, rank));
  TSR_TRY(check_precision(precision));
  if (rank > kMaxRank)
    return fail(TSR_E_UNSUPPORTED, "rank %lld exceeds the supported %d", (long long)rank,
                kMaxRank);
  const int R = (int)rank;
  const int64_t n = numel(ndim, shape);
  int64_t ftotal = 0, rmax = 0;
  FactorTable ft{};
  for (int m = 0; m < ndim; ++m) {
    ft.ptr[m] = d_out + ftotal;
    ft.rows[m] = shape[m];
    ftotal += shape[m] * R;
    rmax = std::max<int64_t>(rmax, shape[m]);
  }
  if (d_init != d_out)
    TSR_CUDA(cudaMemcpyAsync(d_out, d_init, sizeof(float) * ftotal, cudaMemcpyDeviceToDevice,
                             ctx->stream));
  // workspace: prev factors (MISC0), U_new (MISC1), M in FP64 (MISC3), the
  // Grams / Hadamards / inverse and the ALS + accelerated state
  const int hist_n = std::max(max_iters, 1);
  void *pp, *up, *mp, *gp, *stp;
  TSR_TRY(slot_get(ctx, SLOT_MISC0, sizeof(float) * (size_t)ftotal, &pp));
  TSR_TRY(slot_get(ctx, SLOT_MISC1, sizeof(float) * (size_t)rmax * R, &up));
  TSR_TRY(slot_get(ctx, SLOT_MISC3, sizeof(double) * (size_t)rmax * R, &mp));
  TSR_TRY(slot_get(ctx, SLOT_GRAMS, sizeof(double) * (size_t)(2 * ndim + 1) * R * R, &gp));
  TSR_TRY(slot_get(ctx, SLOT_STATE, 512 + sizeof(double) * hist_n, &stp));
  float* prev = (float*)pp;
  float* unew = (float*)up;
  double* mbuf = (double*)mp;
  AlsBuffers b;
  b.grams = (double*)gp;
  b.hadam = b.grams + (size_t)ndim * R * R;
  b.ginv = b.hadam + (size_t)ndim * R * R;
  b.state = (AlsState*)stp;
  AccelState* ast = (AccelState*)((char*)stp + 256);
  b.history = (double*)((char*)stp + 512);
  TSR_CUDA(cudaMemsetAsync(stp, 0, 512 + sizeof(double) * hist_n, ctx->stream));
  TSR_CUDA(cudaMemsetAsync(gp, 0, sizeof(double) * (size_t)(2 * ndim + 1) * R * R, ctx->stream));
  TSR_TRY(reset_status(ctx));
  const double alpha0 = 0.5;
  TSR_CUDA(cudaMemcpyAsync(&ast->alpha, &alpha0, sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
  // prev_factors start as the initial factors (advanced.rs:86)
  TSR_CUDA(cudaMemcpyAsync(prev, d_out, sizeof(float) * ftotal, cudaMemcpyDeviceToDevice,
                           ctx->stream));

  // operands: the single-layout BF16x3 copy of a 3-way tensor, else one
  // unfolding per mode
  const bool d3 = precision == TSR_PREC_BF16X3 && dense3_supported(ndim, shape, R) &&
                  ((uintptr_t)dX & 15) == 0;
  Dense3 d;
  std::memset(&d, 0, sizeof(d));
  std::vector<ModeOperand> ops(ndim);
  size_t pmax = 0;
  void* xn_dev;
  TSR_TRY(slot_get(ctx, SLOT_MISC2, sizeof(double), &xn_dev));
  TSR_CUDA(cudaMemsetAsync(xn_dev, 0, sizeof(double), ctx->stream));
  if (d3) {
    d.I = shape[0];
    d.J = shape[1];
    d.K = shape[2];
    d.R = R;
    d.n_pad = dense3_n_pad(R);
    void *hp, *lp, *ip;
    TSR_TRY(slot_get(ctx, SLOT_D3_HI, sizeof(__nv_bfloat16) * (size_t)n, &hp));
    TSR_TRY(slot_get(ctx, SLOT_D3_LO, sizeof(__nv_bfloat16) * (size_t)n, &lp));
    const size_t img1 = bimage_bytes(d.J, d.n_pad), img2 = bimage_bytes(d.K, d.n_pad);
    TSR_TRY(slot_get(ctx, SLOT_D3_IMG, img1 + img2, &ip));
    d.hi = (const __nv_bfloat16*)hp;
    d.lo = (const __nv_bfloat16*)lp;
    d.bimg[1] = (uint8_t*)ip;
    d.bimg[2] = (uint8_t*)ip + img1;
    for (int m = 0; m < 3; ++m) {
      const SplitPlan p = plan_mttkrp3(ctx, d, m);
      pmax = std::max(pmax, (size_t)p.splits * dense3_rows(d, m) * R);
    }
    TSR_TRY(launch_split_bf16(ctx, ctx->stream, dX, n, (__nv_bfloat16*)hp, (__nv_bfloat16*)lp,
                              (double*)xn_dev));
    TSR_TRY(launch_bimage(ctx, ctx->stream, ft.ptr[1], d.J, R, d.n_pad, d.bimg[1]));
    TSR_TRY(launch_bimage(ctx, ctx->stream, ft.ptr[2], d.K, R, d.n_pad, d.bimg[2]));
  } else {
    for (int m = 0; m < ndim; ++m) {
      TSR_TRY(prepare_mode(ctx, dX, ndim, shape, m, precision, m, &ops[m]));
      const bool tc = precision == TSR_PREC_BF16X3;
      const SplitPlan p = tc ? plan_tc(ctx, ops[m].u, R)
                             : plan_simt(ctx, ops[m].u.rows, ops[m].u.cols, R,
                                         simt_run_len(ops[m]));
      pmax = std::max(pmax, partial_floats(p, ops[m].u.rows, R));
    }
    TSR_TRY(launch_norm_sq(ctx, ctx->stream, dX, n, (double*)xn_dev));
  }
  for (int m = 0; m < ndim; ++m)
    TSR_TRY(launch_gram(ctx, ctx->stream, ft.ptr[m], shape[m], R, b.grams + (size_t)m * R * R,
                        false));
  void* partp;
  TSR_TRY(slot_get(ctx, SLOT_PARTIALS, sizeof(float) * pmax, &partp));
  double xn = 0.0;
  TSR_CUDA(cudaMemcpyAsync(&xn, xn_dev, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  const float ridge = std::numeric_limits<float>::epsilon() * (float)(R * 10);

  bool stopped_by_time = false;
  for (int iter = 0; iter < max_iters; ++iter) {
    if (time_limit_s >= 0.0) {  // advanced.rs:107-113
      const double el =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
      if (el > time_limit_s) {
        stopped_by_time = true;
        break;
      }
    }
    TSR_CUDA(cudaMemsetAsync(&ast->inner, 0, sizeof(double), ctx->stream));
    for (int m = 0; m < ndim; ++m) {
      float* partials = (float*)partp;
      int splits = 1;
      if (d3) {
        const SplitPlan plan = plan_mttkrp3(ctx, d, m);
        TSR_TRY(launch_mttkrp3(ctx, ctx->stream, d, m, ft, plan, partials, true));
        splits = plan.splits;
      } else {
        TSR_TRY(run_mttkrp_partials(ctx, ops[m], ft, R, precision, &partials, &splits));
      }
      TSR_TRY(launch_chol(ctx, ctx->stream, b, ndim, m, R, ridge, false, 0.0));
      TSR_CUDA(cudaMemsetAsync(ast->sums, 0, sizeof(ast->sums), ctx->stream));
      const int64_t off = ft.ptr[m] - ft.ptr[0];
      TSR_TRY(launch_accel_solve(ctx, partials, splits, shape[m], R, b.ginv,
                                 b.hadam + (size_t)m * R * R, prev + off, unew, mbuf, ast,
                                 b.state));
      // modes 1 and 2 of the single-layout path also refresh their B image
      uint8_t* img = (d3 && m > 0) ? d.bimg[m] : nullptr;
      TSR_TRY(launch_accel_apply(ctx, shape[m], R, unew, mbuf, const_cast<float*>(ft.ptr[m]),
                                 prev + off, b.grams + (size_t)m * R * R, ast, b.state, xn,
                                 m == ndim - 1, img, d.n_pad));
    }
    accel_fit_kernel<<<1, 32, 0, ctx->stream>>>(b.grams, ndim, R, xn, tol, ast, b.state,
                                                b.history);
    ctx->launches++;
    TSR_CUDA(cudaGetLastError());
    int done = 0;
    TSR_CUDA(cudaMemcpyAsync(&done, &ast->done, sizeof(int), cudaMemcpyDeviceToHost,
                             ctx->stream));
    AlsState hs;
    TSR_CUDA(cudaMemcpyAsync(&hs, b.state, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
    TSR_TRY(check_device_status(ctx));
    if (hs.status & DS_NOT_SPD)
      return fail(TSR_E_NOT_SPD,
                  "Linear algebra error: Gram matrix is not positive definite (ridge %g also "
                  "failed)",
                  (double)ridge);
    if (done) break;
  }
  AccelState hs;
  AlsState as;
  TSR_CUDA(cudaMemcpyAsync(&hs, ast, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
  TSR_CUDA(cudaMemcpyAsync(&as, b.state, sizeof(as), cudaMemcpyDeviceToHost, ctx->stream));
  TSR_TRY(check_device_status(ctx));
  if (info) {
    info->fit = hs.fit;
    info->iters = hs.iter + (stopped_by_time && hs.iter < max_iters ? 1 : 0);
    info->reason = stopped_by_time ? TSR_REASON_TIME_LIMIT
                   : hs.done       ? hs.reason
                                   : TSR_REASON_MAX_ITERATIONS;
    info->oscillation_count = hs.osc;
    info->oscillated = hs.osc > 0;
    info->final_fit_change = hs.final_change;
    info->ridge_used = as.ridge_used;
    if (info->fit_history && hs.iter > 0)
      TSR_CUDA(cudaMemcpy(info->fit_history, b.history, sizeof(double) * hs.iter,
                          cudaMemcpyDeviceToHost));
  }
  return TSR_OK;
}

void init_accel_attributes() {
  cudaFuncSetAttribute(accel_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(sizeof(double) * (2 * kMaxRank * kMaxRank + 8 * 5)));
}

}  // namespace tsr

using namespace tsr;

extern "C" {

int tsr_cp_als_accelerated_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim,
                                   const int64_t* shape, int64_t rank, int max_iters, double tol,
                                   const float* d_init, int precision, double time_limit_s,
                                   float* d_out_factors, tsr_cp_info* info) {
  if (!shape || !d_tensor || !d_init || !d_out_factors)
    return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(check_ctx(ctx));
  return cp_als_accelerated_device(ctx, d_tensor, ndim, shape, rank, max_iters, tol, d_init,
                                   precision, time_limit_s, d_out_factors, info);
}

int tsr_cp_als_accelerated_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                               int64_t rank, int max_iters, double tol,
                               const float* init_factors, uint64_t seed, int precision,
                               double time_limit_s, float* out_factors, tsr_cp_info* info) {
  if (!shape || !tensor || !out_factors) return fail(TSR_E_INVALID_ARG, "null argument");
  if (rank == 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  if (!(tol > 0.0 && tol < 1.0)) return fail(TSR_E_INVALID_TOL, "Invalid tolerance: %g", tol);
  if (ndim < 2 || ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "accelerated CP-ALS needs 2..%d modes", kMaxModes);
  TSR_TRY(check_sizes(ndim, shape, rank));
  TSR_TRY(check_precision(precision));
  TSR_TRY(check_ctx(ctx));
  int64_t ftotal = 0;
  for (int m = 0; m < ndim; ++m) ftotal += shape[m] * rank;
  std::vector<float> init_buf;
  const float* init = init_factors;
  if (!init) {  // InitStrategy::Random from the library's seeded stream
    init_buf.resize(ftotal);
    int64_t off = 0;
    for (int m = 0; m < ndim; ++m) {
      seeded_uniform(seed, 200 + m, shape[m] * rank, init_buf.data() + off);
      off += shape[m] * rank;
    }
    init = init_buf.data();
  }
  float* dX;
  TSR_TRY(upload_tensor(ctx, tensor, ndim, shape, nullptr, &dX));
  void* df;
  TSR_TRY(slot_get(ctx, SLOT_OUT, sizeof(float) * ftotal, &df));
  TSR_CUDA(cudaMemcpyAsync(df, init, sizeof(float) * ftotal, cudaMemcpyHostToDevice, ctx->stream));
  TSR_TRY(cp_als_accelerated_device(ctx, dX, ndim, shape, rank, max_iters, tol, (const float*)df,
                                    precision, time_limit_s, (float*)df, info));
  TSR_CUDA(cudaMemcpyAsync(out_factors, df, sizeof(float) * ftotal, cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

}  // extern "C"

// The f64 instantiation of the drop-in: tenrso_kernels::mttkrp<f64>
// (crates/tenrso-kernels/src/mttkrp.rs:74-146) and tenrso_decomp::cp_als<f64>
// (crates/tenrso-decomp/src/cp/core.rs:59-182) with every value in FP64.
//
// MTTKRP: M (I_n x R) = X_(n) KR with X viewed as A x I_n x B (A = prod of
// the modes before n, B = prod after): the unfolding's column j = a B + b is
// also the forward Khatri-Rao row (mttkrp.rs:182-240), so no unfolding is
// stored. A CTA owns 32 rows x 64 columns of M and a range of j (split-K);
// each 32-wide j slice stages its X tile and its Khatri-Rao rows (formed from
// the factors, one base offset per other mode and j) in shared memory; split
// partial sums meet in M with FP64 atomics.
//
// CP-ALS: the same device state, inverse and fit kernels as the fp32 sweep
// (als.cu), with an FP64 solve (U = M G^-1, the new Gram and, for the last
// mode, <M, U> and ||Xhat||^2) and FP64 factors; the ridge of
// solve_least_squares is f64's eps * rank * 10 (helpers.rs:477-490).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "als.cuh"
#include "dense.cuh"

namespace tsr {

namespace {

struct M64Args {
  const double* X;
  int64_t A, I, B;   // X as A x I x B (the mode's size is I)
  int R;
  int n_other;       // modes other than the MTTKRP mode, ascending
  int64_t osize[kMaxModes];
  const double* U[kMaxModes];  // their factors (rows x R)
  int64_t j_per_split;
  double* M;         // I x R, zeroed by the caller
};

constexpr int F64_BI = 32, F64_BC = 64, F64_BJ = 32;

__global__ void __launch_bounds__(256) mttkrp_f64_kernel(M64Args g) {
  __shared__ double xs[F64_BI][F64_BJ + 1];
  __shared__ double ks[F64_BJ][F64_BC + 1];
  __shared__ int64_t koff[F64_BJ][kMaxModes];  // row offsets (x R) of each other factor
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  const int64_t i0 = (int64_t)blockIdx.x * F64_BI;
  const int c0 = blockIdx.y * F64_BC;
  const int64_t J = g.A * g.B;
  const int64_t jb = (int64_t)blockIdx.z * g.j_per_split;
  const int64_t je = min(jb + g.j_per_split, J);
  double acc[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
  for (int64_t j0 = jb; j0 < je; j0 += F64_BJ) {
    // per j of the slice: the other modes' indices (row-major over the other
    // modes in ascending order, i.e. the forward Khatri-Rao row)
    if (t < F64_BJ) {
      int64_t j = j0 + t, r = j < je ? j : jb;
      for (int p = g.n_other - 1; p >= 0; --p) {
        koff[t][p] = (r % g.osize[p]) * g.R;
        r /= g.osize[p];
      }
    }
    for (int e = t; e < F64_BI * F64_BJ; e += 256) {
      const int ii = e / F64_BJ, jj = e % F64_BJ;
      const int64_t i = i0 + ii, j = j0 + jj;
      double v = 0.0;
      if (i < g.I && j < je) {
        const int64_t a = j / g.B, b = j % g.B;
        v = __ldg(g.X + (a * g.I + i) * g.B + b);
      }
      xs[ii][jj] = v;
    }
    __syncthreads();
    for (int e = t; e < F64_BJ * F64_BC; e += 256) {
      const int jj = e / F64_BC, cc = e % F64_BC;
      const int c = c0 + cc;
      double v = 0.0;
      if (j0 + jj < je && c < g.R) {
        v = 1.0;
        for (int p = 0; p < g.n_other; ++p) v *= __ldg(g.U[p] + koff[jj][p] + c);
      }
      ks[jj][cc] = v;
    }
    __syncthreads();
#pragma unroll 8
    for (int jj = 0; jj < F64_BJ; ++jj) {
      const double x0 = xs[ty][jj], x1 = xs[ty + 16][jj];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double k = ks[jj][tx + 16 * q];
        acc[0][q] = fma(x0, k, acc[0][q]);
        acc[1][q] = fma(x1, k, acc[1][q]);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    const int64_t i = i0 + ty + 16 * p;
    if (i >= g.I) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = c0 + tx + 16 * q;
      if (c < g.R) atomicAdd(g.M + i * g.R + c, acc[p][q]);
    }
  }
}

// Upper triangle of the Gram of rows r0.. of a (rows x R) FP64 block held in
// shared memory (Us, nr rows), accumulated into registers.
template <int RB>
__device__ __forceinline__ void gram_rows(const double* Us, int nr, int R,
                                          double (&acc)[RB][RB]) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  for (int i = 0; i < nr; ++i) {
    double x[RB], y[RB];
#pragma unroll
    for (int a = 0; a < RB; ++a) x[a] = ty + 16 * a < R ? Us[i * R + ty + 16 * a] : 0.0;
#pragma unroll
    for (int b = 0; b < RB; ++b) y[b] = tx + 16 * b < R ? Us[i * R + tx + 16 * b] : 0.0;
#pragma unroll
    for (int a = 0; a < RB; ++a)
#pragma unroll
      for (int b = 0; b < RB; ++b) acc[a][b] = fma(x[a], y[b], acc[a][b]);
  }
}

// U (rows x R, FP64) = M G^-1 with G^-1 from the inverse kernel (b.ginv);
// gram += U^T U (upper, FP64 atomics); for the last mode <M, U> and
// ||Xhat||^2 = sum(H o U^T U) into the state, and the fit marked pending.
// With M null the kernel only accumulates the Gram of U (initial Grams).
template <int RB>
__global__ void __launch_bounds__(256)
solve_f64_kernel(AlsBuffers b, int ndim, int R, int64_t rows, const double* __restrict__ M,
                 double* __restrict__ U, double* __restrict__ gram, int last) {
  extern __shared__ __align__(16) double sm[];
  __shared__ double red[16];
  AlsState* st = b.state;
  if (M && st->done) return;
  constexpr int rpc = 16;
  double* Gi = sm;                    // R x R (solve only)
  double* Us = sm + (M ? R * R : 0);  // rpc x R
  if (M)
    for (int e = threadIdx.x; e < R * R; e += blockDim.x) Gi[e] = b.ginv[e];
  double acc[RB][RB];
#pragma unroll
  for (int a = 0; a < RB; ++a)
#pragma unroll
    for (int c = 0; c < RB; ++c) acc[a][c] = 0.0;
  double ip = 0.0;
  for (int64_t r0 = (int64_t)blockIdx.x * rpc; r0 < rows; r0 += (int64_t)gridDim.x * rpc) {
    const int nr = (int)(rows - r0 < rpc ? rows - r0 : rpc);
    __syncthreads();
    for (int e = threadIdx.x; e < nr * R; e += blockDim.x) {
      const int64_t g = r0 * R + e;
      double u;
      if (M) {
        const int i = e / R, c = e % R;
        const double* m = M + (r0 + i) * R;
        u = 0.0;
        for (int k = 0; k < R; ++k) u = fma(m[k], Gi[k * R + c], u);
        U[g] = u;
        if (last) ip += M[g] * u;
      } else {
        u = U[g];
      }
      Us[e] = u;
    }
    __syncthreads();
    gram_rows<RB>(Us, nr, R, acc);
  }
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double xs = 0.0;
  const double* H = b.hadam + (int64_t)(ndim - 1) * R * R;
#pragma unroll
  for (int a = 0; a < RB; ++a)
#pragma unroll
    for (int c = 0; c < RB; ++c) {
      const int i = ty + 16 * a, j = tx + 16 * c;
      if (i < R && j < R && j >= i) {
        atomicAdd(gram + i * R + j, acc[a][c]);
        if (last) xs += (i == j ? 1.0 : 2.0) * H[i * R + j] * acc[a][c];
      }
    }
  if (!last || !M) return;
  for (int o = 16; o > 0; o >>= 1) {
    ip += __shfl_down_sync(0xffffffffu, ip, o);
    xs += __shfl_down_sync(0xffffffffu, xs, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = ip;
    red[8 + (threadIdx.x >> 5)] = xs;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0, x = 0.0;
    for (int w = 0; w < 8; ++w) {
      s += red[w];
      x += red[8 + w];
    }
    atomicAdd(&st->inner, s);
    atomicAdd(&st->xhat_sq, x);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->fit_pending = 1;
}

__global__ void norm_sq_f64_kernel(const double* __restrict__ X, int64_t n, double* out) {
  double s = 0.0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const double v = X[e];
    s = fma(v, v, s);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

unsigned f64_grid(const tsr_ctx* ctx, int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), ctx->sm_count * 8));
}

int launch_mttkrp_f64(tsr_ctx* ctx, const double* X, int ndim, const int64_t* shape,
                      const double* const* U, int R, int mode, double* M) {
  cudaStream_t s = ctx->stream;
  M64Args g;
  std::memset(&g, 0, sizeof(g));
  g.X = X;
  g.A = 1;
  g.B = 1;
  for (int m = 0; m < mode; ++m) g.A *= shape[m];
  for (int m = mode + 1; m < ndim; ++m) g.B *= shape[m];
  g.I = shape[mode];
  g.R = R;
  g.M = M;
  for (int m = 0; m < ndim; ++m)
    if (m != mode) {
      g.osize[g.n_other] = shape[m];
      g.U[g.n_other] = U[m];
      ++g.n_other;
    }
  TSR_CUDA(cudaMemsetAsync(M, 0, sizeof(double) * g.I * R, s));
  const int64_t J = g.A * g.B;
  if (g.I == 0 || R == 0 || J == 0) return TSR_OK;
  const int64_t tiles = ceil_div(g.I, F64_BI) * ceil_div(R, F64_BC);
  const int64_t want = std::max<int64_t>(1, (4 * (int64_t)ctx->sm_count + tiles - 1) / tiles);
  const int64_t splits = std::max<int64_t>(1, std::min<int64_t>(want, ceil_div(J, 4 * F64_BJ)));
  g.j_per_split = round_up(ceil_div(J, splits), F64_BJ);
  const int64_t nsplit = std::min<int64_t>(ceil_div(J, g.j_per_split), 65535);
  g.j_per_split = std::max<int64_t>(g.j_per_split, ceil_div(J, nsplit));
  dim3 grid((unsigned)ceil_div(g.I, F64_BI), (unsigned)ceil_div(R, F64_BC),
            (unsigned)ceil_div(J, g.j_per_split));
  if (grid.x > 2147483647u || grid.y > 65535u)
    return fail(TSR_E_UNSUPPORTED, "f64 MTTKRP grid too large");
  mttkrp_f64_kernel<<<grid, 256, 0, s>>>(g);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_solve_f64(tsr_ctx* ctx, const AlsBuffers& b, int ndim, int R, int64_t rows,
                     const double* M, double* U, double* gram, bool last) {
  const unsigned grid = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(ceil_div(rows, 16), 2 * (int64_t)ctx->sm_count));
  const size_t smem = sizeof(double) * ((M ? (size_t)R * R : 0) + 16 * (size_t)R);
  const int lst = last ? 1 : 0;
#define TSR_S64(RB) \
  solve_f64_kernel<RB><<<grid, 256, smem, ctx->stream>>>(b, ndim, R, rows, M, U, gram, lst)
  switch ((R + 15) / 16) {
    case 1: TSR_S64(1); break;
    case 2: TSR_S64(2); break;
    case 3: TSR_S64(3); break;
    case 4: TSR_S64(4); break;
    case 5: TSR_S64(5); break;
    case 6: TSR_S64(6); break;
    default: TSR_S64(7); break;
  }
#undef TSR_S64
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

// Host seeded U(0,1) doubles of the library's stream (InitStrategy::Random).
void seeded_uniform_f64(uint64_t seed, uint64_t stream, int64_t n, double* out) {
  auto mix = [](uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  const uint64_t golden = 0x9E3779B97F4A7C15ull;
  const uint64_t key = mix(seed * 0x100000001B3ull + stream * 0x2545F4914F6CDD1Dull + golden);
  for (int64_t i = 0; i < n; ++i)
    out[i] = (double)(mix(key + (uint64_t)i * golden) >> 11) * (1.0 / 9007199254740992.0);
}

struct DevMem {
  std::vector<void*> p;
  template <class T>
  int get(T** q, size_t n) {
    void* r = nullptr;
    cudaError_t e = cudaMalloc(&r, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess)
      return fail(TSR_E_CUDA, "cudaMalloc (%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    p.push_back(r);
    *q = (T*)r;
    return TSR_OK;
  }
  ~DevMem() {
    for (void* r : p) cudaFree(r);
  }
};

}  // namespace

void init_f64_attributes() {
  const int big = (int)(sizeof(double) * (kMaxRank * kMaxRank + 16 * kMaxRank));
  cudaFuncSetAttribute(solve_f64_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(solve_f64_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(solve_f64_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(solve_f64_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(solve_f64_kernel<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(solve_f64_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(solve_f64_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
}

// cp_als<f64> on device data (dX row-major FP64; factors FP64 in d_out).
int cp_als_f64_device(tsr_ctx* ctx, const double* dX, int ndim, const int64_t* shape,
                      int64_t rank, int max_iters, double tol, double time_limit_s,
                      double* d_out, tsr_cp_info* info) {
  const auto t_start = std::chrono::steady_clock::now();
  const int R = (int)rank;
  cudaStream_t s = ctx->stream;
  int64_t rmax = 0, n = numel(ndim, shape);
  const double* U[kMaxModes];
  int64_t off = 0;
  for (int m = 0; m < ndim; ++m) {
    U[m] = d_out + off;
    off += shape[m] * R;
    rmax = std::max<int64_t>(rmax, shape[m]);
  }
  const int hist_n = std::max(max_iters, 1);
  DevMem mem;
  double *grams, *Mbuf;
  void* stp;
  TSR_TRY(mem.get(&grams, (size_t)(2 * ndim + 1) * R * R));
  TSR_TRY(mem.get(&Mbuf, (size_t)rmax * R));
  TSR_TRY(mem.get((uint8_t**)&stp, 256 + sizeof(double) * hist_n));
  AlsBuffers b;
  b.grams = grams;
  b.hadam = grams + (size_t)ndim * R * R;
  b.ginv = b.hadam + (size_t)ndim * R * R;
  b.state = (AlsState*)stp;
  b.history = (double*)((char*)stp + 256);
  TSR_CUDA(cudaMemsetAsync(stp, 0, 256 + sizeof(double) * hist_n, s));
  TSR_CUDA(cudaMemsetAsync(grams, 0, sizeof(double) * (2 * ndim + 1) * R * R, s));
  norm_sq_f64_kernel<<<f64_grid(ctx, n), 256, 0, s>>>(dX, n, &b.state->xnorm_sq);
  ctx->launches++;
  for (int m = 0; m < ndim; ++m)
    TSR_TRY(launch_solve_f64(ctx, b, ndim, R, shape[m], nullptr, const_cast<double*>(U[m]),
                             grams + (size_t)m * R * R, false));
  const float ridge = (float)(std::numeric_limits<double>::epsilon() * (double)(R * 10));
  bool by_time = false;
  for (int iter = 0; iter < max_iters; ++iter) {
    if (time_limit_s >= 0.0) {  // core.rs:104-110
      const double el =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
      if (el > time_limit_s) {
        by_time = true;
        break;
      }
    }
    for (int m = 0; m < ndim; ++m) {
      const bool last = m == ndim - 1;
      TSR_TRY(launch_chol(ctx, s, b, ndim, m, R, ridge, last, tol));
      TSR_TRY(launch_mttkrp_f64(ctx, dX, ndim, shape, U, R, m, Mbuf));
      TSR_TRY(launch_solve_f64(ctx, b, ndim, R, shape[m], Mbuf, const_cast<double*>(U[m]),
                               grams + (size_t)m * R * R, last));
    }
    // the fit of this sweep, then the stop decision on the host
    TSR_TRY(launch_fit(ctx, s, b, ndim, R, tol));
    AlsState hs;
    TSR_CUDA(cudaMemcpyAsync(&hs, b.state, sizeof(hs), cudaMemcpyDeviceToHost, s));
    TSR_CUDA(cudaStreamSynchronize(s));
    if (hs.status & DS_NOT_SPD)
      return fail(TSR_E_NOT_SPD,
                  "Linear algebra error: Gram matrix is not positive definite (ridge %g also "
                  "failed)",
                  (double)ridge);
    if (hs.done) break;
  }
  AlsState hs;
  TSR_CUDA(cudaMemcpyAsync(&hs, b.state, sizeof(hs), cudaMemcpyDeviceToHost, s));
  TSR_CUDA(cudaStreamSynchronize(s));
  if (info) {
    info->fit = hs.fit;
    // core.rs:116-124: the time check comes before the sweep is counted
    info->iters = hs.iter;
    info->reason = by_time    ? TSR_REASON_TIME_LIMIT
                   : hs.done ? hs.reason
                             : TSR_REASON_MAX_ITERATIONS;
    info->oscillation_count = hs.osc;
    info->oscillated = hs.osc > 0;
    info->final_fit_change = hs.final_change;
    info->ridge_used = hs.ridge_used;
    if (info->fit_history && hs.iter > 0)
      TSR_CUDA(cudaMemcpy(info->fit_history, b.history, sizeof(double) * hs.iter,
                          cudaMemcpyDeviceToHost));
  }
  return TSR_OK;
}

}  // namespace tsr

using namespace tsr;

extern "C" {

int tsr_mttkrp_f64(tsr_ctx* ctx, const double* tensor, int ndim, const int64_t* shape,
                   const double* const* factors, int n_factors, const int64_t* factor_rows,
                   const int64_t* factor_cols, int mode, double* out) {
  if (!tensor || !shape || !factors || !factor_rows || !factor_cols || !out)
    return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(validate_mttkrp(ndim, shape, n_factors, factor_rows, factor_cols, mode));
  TSR_TRY(check_sizes(ndim, shape, factor_cols[0]));
  TSR_TRY(check_ctx(ctx));
  const int R = (int)factor_cols[0];
  const int64_t n = numel(ndim, shape);
  DevMem mem;
  double *dX, *dF, *dM;
  int64_t ftotal = 0;
  for (int m = 0; m < ndim; ++m) ftotal += shape[m] * R;
  TSR_TRY(mem.get(&dX, (size_t)n));
  TSR_TRY(mem.get(&dF, (size_t)ftotal));
  TSR_TRY(mem.get(&dM, (size_t)shape[mode] * R));
  TSR_CUDA(cudaMemcpyAsync(dX, tensor, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  const double* U[kMaxModes];
  int64_t off = 0;
  for (int m = 0; m < ndim; ++m) {
    TSR_CUDA(cudaMemcpyAsync(dF + off, factors[m], sizeof(double) * shape[m] * R,
                             cudaMemcpyHostToDevice, ctx->stream));
    U[m] = dF + off;
    off += shape[m] * R;
  }
  TSR_TRY(launch_mttkrp_f64(ctx, dX, ndim, shape, U, R, mode, dM));
  TSR_CUDA(cudaMemcpyAsync(out, dM, sizeof(double) * shape[mode] * R, cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

int tsr_cp_als_f64(tsr_ctx* ctx, const double* tensor, int ndim, const int64_t* shape,
                   int64_t rank, int max_iters, double tol, const double* init_factors,
                   uint64_t seed, double time_limit_s, double* out_factors, tsr_cp_info* info) {
  if (!shape || !tensor || !out_factors) return fail(TSR_E_INVALID_ARG, "null argument");
  // core.rs:82-94 (as the f32 entry point)
  if (rank == 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  for (int d = 0; d < ndim; ++d)
    if (rank > shape[d]) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  if (!(tol >= 0.0 && tol < 1.0)) return fail(TSR_E_INVALID_TOL, "Invalid tolerance: %g", tol);
  TSR_TRY(check_sizes(ndim, shape, rank));
  if (ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d exceeds the supported %d", ndim, kMaxModes);
  if (rank > kMaxRank)
    return fail(TSR_E_UNSUPPORTED, "rank %lld exceeds the supported %d", (long long)rank,
                kMaxRank);
  if (ndim < 2 && max_iters > 0)
    return fail(TSR_E_SHAPE, "Shape mismatch: Need at least 2 factor matrices for MTTKRP");
  TSR_TRY(check_ctx(ctx));
  const int64_t n = numel(ndim, shape);
  int64_t ftotal = 0;
  for (int m = 0; m < ndim; ++m) ftotal += shape[m] * rank;
  std::vector<double> init_buf;
  const double* init = init_factors;
  if (!init) {  // InitStrategy::Random from the library's seeded stream, in FP64
    init_buf.resize(ftotal);
    int64_t off = 0;
    for (int m = 0; m < ndim; ++m) {
      seeded_uniform_f64(seed, 200 + m, shape[m] * rank, init_buf.data() + off);
      off += shape[m] * rank;
    }
    init = init_buf.data();
  }
  DevMem mem;
  double *dX, *dF;
  TSR_TRY(mem.get(&dX, (size_t)n));
  TSR_TRY(mem.get(&dF, (size_t)ftotal));
  TSR_CUDA(cudaMemcpyAsync(dX, tensor, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  TSR_CUDA(cudaMemcpyAsync(dF, init, sizeof(double) * ftotal, cudaMemcpyHostToDevice,
                           ctx->stream));
  TSR_TRY(cp_als_f64_device(ctx, dX, ndim, shape, rank, max_iters, tol, time_limit_s, dF, info));
  TSR_CUDA(cudaMemcpyAsync(out_factors, dF, sizeof(double) * ftotal, cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

}  // extern "C"

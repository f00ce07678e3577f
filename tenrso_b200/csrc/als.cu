// FP64 kernels of the ALS sweep. Replace, from crates/tenrso-decomp/src/cp/:
//   compute_gram_hadamard / compute_gram_matrix   helpers.rs:409-452
//   solve_least_squares (per-row lstsq + ridge)   helpers.rs:455-495
//   compute_norm_squared / compute_fit            helpers.rs:498-579
//   convergence + oscillation bookkeeping          core.rs:173-198
// The per-row least-squares solves become one Cholesky factorisation of the
// symmetric Gram G (FP64), its inverse, and a row-parallel product M . G^-1.
// ||Xhat||^2 and <X, Xhat> come from the Grams and the last mode's MTTKRP
// (mathematically identical to the extra mode-0 MTTKRP of helpers.rs:558-579).
#include "als.cuh"

namespace tsr {

namespace {

__global__ void gram_kernel(const float* __restrict__ U, int64_t rows, int R, int rows_per_cta,
                            double* __restrict__ gram) {
  extern __shared__ double sh[];
  double* Us = sh;  // [rows_per_cta][R]
  int64_t r0 = (int64_t)blockIdx.x * rows_per_cta;
  int nr = (int)(rows - r0 < rows_per_cta ? rows - r0 : rows_per_cta);
  for (int k = threadIdx.x; k < nr * R; k += blockDim.x) Us[k] = (double)U[r0 * R + k];
  __syncthreads();
  for (int e = threadIdx.x; e < R * R; e += blockDim.x) {
    int a = e / R, c = e % R;
    if (c < a) continue;  // symmetric: compute upper, mirror
    double s = 0.0;
    for (int i = 0; i < nr; ++i) s += Us[i * R + a] * Us[i * R + c];
    atomicAdd(gram + a * R + c, s);
    if (c != a) atomicAdd(gram + c * R + a, s);
  }
}

__global__ void norm_sq_kernel(const float* __restrict__ X, int64_t n, AlsState* st) {
  double s = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    double v = X[k];
    s += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) atomicAdd(&st->xnorm_sq, s);
  }
}

// Outer-product Cholesky on A (R x R, row-major, shared). One barrier per
// column: step j subtracts a_ij a_kj / a_jj from the trailing lower triangle.
// Afterwards L_ij = a_ij / sqrt(a_jj). Returns false (to all threads) if a
// pivot is not positive or not finite.
__device__ bool chol_inplace(double* A, int R, int* bad) {
  if (threadIdx.x == 0) *bad = 0;
  __syncthreads();
  for (int j = 0; j < R; ++j) {
    double d = A[j * R + j];
    if (!(d > 0.0) || !isfinite(d)) {
      if (threadIdx.x == 0) *bad = 1;
      break;  // every thread sees the same d and breaks together
    }
    int n = R - 1 - j;
    int tri = n * (n + 1) / 2;
    double inv = 1.0 / d;
    for (int e = threadIdx.x; e < tri; e += blockDim.x) {
      // e -> (i, k) with j < k <= i, row-major over the lower triangle
      int i = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
      while ((i + 1) * (i + 2) / 2 <= e) ++i;
      while (i * (i + 1) / 2 > e) --i;
      int k = e - i * (i + 1) / 2;
      int gi = j + 1 + i, gk = j + 1 + k;
      A[gi * R + gk] -= A[gi * R + j] * A[gk * R + j] * inv;
    }
    __syncthreads();
  }
  __syncthreads();
  bool ok = *bad == 0;
  __syncthreads();
  if (!ok) return false;
  // scale columns: L_ij = a_ij / sqrt(a_jj), i >= j; zero the upper part
  for (int e = threadIdx.x; e < R * R; e += blockDim.x) {
    int i = e / R, j = e % R;
    if (i < j) A[e] = 0.0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < R * R; e += blockDim.x) {
    int i = e / R, j = e % R;
    if (i > j) A[e] = A[e] / sqrt(A[j * R + j]);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < R; j += blockDim.x) A[j * R + j] = sqrt(A[j * R + j]);
  __syncthreads();
  return true;
}

__global__ void chol_kernel(AlsBuffers b, int ndim, int mode, int R, float ridge_eps, int last) {
  extern __shared__ double sh[];
  double* G = sh;            // R x R Hadamard; reused for L^{-1} once factored
  double* L = sh + R * R;    // R x R Cholesky factor
  double* W = G;
  __shared__ int bad;
  AlsState* st = b.state;
  if (st->done) return;
  const int RR = R * R;
  for (int e = threadIdx.x; e < RR; e += blockDim.x) {
    double g = 1.0;  // compute_gram_hadamard starts from ones (helpers.rs:414)
    for (int m = 0; m < ndim; ++m)
      if (m != mode) g *= b.grams[(int64_t)m * RR + e];
    G[e] = g;
    b.hadam[(int64_t)mode * RR + e] = g;
  }
  __syncthreads();
  // solve_least_squares solves gram^T x = b (helpers.rs:462,471); G is
  // symmetric by construction so G^T = G.
  for (int e = threadIdx.x; e < RR; e += blockDim.x) L[e] = G[e];
  __syncthreads();
  bool ok = chol_inplace(L, R, &bad);
  if (!ok) {
    // helpers.rs:477-490: retry with eps * rank * 10 on the diagonal
    for (int e = threadIdx.x; e < RR; e += blockDim.x)
      L[e] = G[e] + ((e / R == e % R) ? (double)ridge_eps : 0.0);
    __syncthreads();
    ok = chol_inplace(L, R, &bad);
    if (threadIdx.x == 0) st->ridge_used = 1;
    if (!ok) {
      if (threadIdx.x == 0) {
        st->status |= DS_NOT_SPD;
        st->done = 1;
      }
      return;
    }
  }
  __syncthreads();  // G is dead from here on: W (= L^{-1}) takes its place
  // W = L^{-1}: column c by forward substitution (thread per column).
  for (int c = threadIdx.x; c < R; c += blockDim.x) {
    for (int i = 0; i < R; ++i) {
      if (i < c) {
        W[i * R + c] = 0.0;
        continue;
      }
      double s = (i == c) ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) s -= L[i * R + k] * W[k * R + c];
      W[i * R + c] = s / L[i * R + i];
    }
  }
  __syncthreads();
  // G^{-1} = W^T W
  for (int e = threadIdx.x; e < RR; e += blockDim.x) {
    int a = e / R, c = e % R;
    int k0 = a > c ? a : c;
    double s = 0.0;
    for (int k = k0; k < R; ++k) s += W[k * R + a] * W[k * R + c];
    b.ginv[e] = s;
  }
  // the Gram of U_mode is recomputed by the solve that follows
  for (int e = threadIdx.x; e < RR; e += blockDim.x) b.grams[(int64_t)mode * RR + e] = 0.0;
  if (last && threadIdx.x == 0) st->inner = 0.0;
}

// rows_per_cta rows of U_mode. Shared: Ginv (R x R), M (rows x R), U (rows x R).
__global__ void solve_kernel(AlsBuffers b, const float* __restrict__ partials, int splits,
                             int64_t rows, int R, int rows_per_cta, float* __restrict__ U,
                             int mode, int last) {
  extern __shared__ double sh[];
  AlsState* st = b.state;
  if (st->done) return;
  const int RR = R * R;
  double* Gi = sh;
  double* Ms = sh + RR;
  double* Us = Ms + rows_per_cta * R;
  int64_t r0 = (int64_t)blockIdx.x * rows_per_cta;
  int nr = (int)(rows - r0 < rows_per_cta ? rows - r0 : rows_per_cta);
  for (int e = threadIdx.x; e < RR; e += blockDim.x) Gi[e] = b.ginv[e];
  const int64_t pstride = rows * R;
  for (int e = threadIdx.x; e < nr * R; e += blockDim.x) {
    const float* p = partials + r0 * R + e;
    double s = 0.0;
    for (int q = 0; q < splits; ++q) s += (double)__ldg(p + (int64_t)q * pstride);
    Ms[e] = s;
  }
  __syncthreads();
  double ip = 0.0;
  for (int e = threadIdx.x; e < nr * R; e += blockDim.x) {
    int i = e / R, c = e % R;
    double s = 0.0;
    for (int k = 0; k < R; ++k) s += Ms[i * R + k] * Gi[k * R + c];
    float v = (float)s;
    U[(r0 + i) * R + c] = v;
    Us[e] = (double)v;
    ip += Ms[e] * (double)v;
  }
  __syncthreads();
  double* gram = b.grams + (int64_t)mode * RR;
  for (int e = threadIdx.x; e < RR; e += blockDim.x) {
    int a = e / R, c = e % R;
    if (c < a) continue;
    double s = 0.0;
    for (int i = 0; i < nr; ++i) s += Us[i * R + a] * Us[i * R + c];
    atomicAdd(gram + a * R + c, s);
    if (c != a) atomicAdd(gram + c * R + a, s);
  }
  if (last) {
    for (int o = 16; o > 0; o >>= 1) ip += __shfl_down_sync(0xffffffffu, ip, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&st->inner, ip);
  }
}

__global__ void fit_kernel(AlsBuffers b, int ndim, int R, double tol) {
  AlsState* st = b.state;
  if (st->done) return;
  const int RR = R * R;
  const int last = ndim - 1;
  double s = 0.0;
  for (int e = threadIdx.x; e < RR; e += blockDim.x)
    s += b.hadam[(int64_t)last * RR + e] * b.grams[(int64_t)last * RR + e];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x != 0) return;
  double rn = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) rn += ws[w];
  // helpers.rs:513-530
  double xn = st->xnorm_sq;
  double err_sq = xn + rn - 2.0 * st->inner;
  double err = sqrt(fmax(err_sq, 0.0));
  double fit = 1.0 - err / sqrt(xn);
  fit = fmin(fmax(fit, 0.0), 1.0);
  // core.rs:173-198
  int iter = st->iter;
  st->fit = fit;
  b.history[iter] = fit;
  if (iter > 0 && fit < st->prev_fit) st->osc += 1;
  double change = fabs(fit - st->prev_fit);
  st->final_change = change;
  st->iter = iter + 1;
  if (iter > 0 && change < tol) {
    st->reason = TSR_REASON_FIT_TOLERANCE;
    st->done = 1;
    return;
  }
  if (st->osc > 5 && iter > 10) {
    st->reason = TSR_REASON_OSCILLATION;
    st->done = 1;
    return;
  }
  st->prev_fit = fit;
}

}  // namespace

int launch_gram(tsr_ctx* ctx, const float* U, int64_t rows, int R, double* gram) {
  TSR_CUDA(cudaMemsetAsync(gram, 0, sizeof(double) * R * R, ctx->stream));
  int rpc = 32;
  while (rpc > 1 && (size_t)rpc * R * 8 > 48 * 1024) rpc /= 2;
  unsigned grid = (unsigned)ceil_div(rows, rpc);
  gram_kernel<<<grid, 256, (size_t)rpc * R * 8, ctx->stream>>>(U, rows, R, rpc, gram);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_norm_sq(tsr_ctx* ctx, const float* X, int64_t n, AlsState* st) {
  int grid = ctx->sm_count * 4;
  norm_sq_kernel<<<grid, 256, 0, ctx->stream>>>(X, n, st);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_chol(tsr_ctx* ctx, const AlsBuffers& b, int ndim, int mode, int R, float ridge_eps,
                bool last) {
  size_t smem = (size_t)2 * R * R * sizeof(double);
  static bool attr_set = false;
  if (!attr_set) {
    TSR_CUDA(cudaFuncSetAttribute(chol_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  2 * kMaxRank * kMaxRank * 8));
    attr_set = true;
  }
  if (smem > 227 * 1024) return fail(TSR_E_UNSUPPORTED, "rank %d too large for the FP64 solve", R);
  chol_kernel<<<1, 256, smem, ctx->stream>>>(b, ndim, mode, R, ridge_eps, last ? 1 : 0);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_solve(tsr_ctx* ctx, const AlsBuffers& b, const float* partials, int splits,
                 int64_t rows, int R, float* U, int mode, bool last) {
  // Rows per CTA: enough CTAs to spread the partial-sum reads over the SMs.
  int rpc = (int)std::max<int64_t>(1, std::min<int64_t>(16, ceil_div(rows, ctx->sm_count)));
  size_t smem = (size_t)(R * R + 2 * rpc * R) * sizeof(double);
  static bool attr_set = false;
  if (!attr_set) {
    TSR_CUDA(cudaFuncSetAttribute(solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  200 * 1024));
    attr_set = true;
  }
  if (smem > 200 * 1024) return fail(TSR_E_UNSUPPORTED, "rank %d too large for the FP64 solve", R);
  unsigned grid = (unsigned)ceil_div(rows, rpc);
  solve_kernel<<<grid, 256, smem, ctx->stream>>>(b, partials, splits, rows, R, rpc, U, mode,
                                                 last ? 1 : 0);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_fit(tsr_ctx* ctx, const AlsBuffers& b, int ndim, int R, double tol) {
  fit_kernel<<<1, 256, 0, ctx->stream>>>(b, ndim, R, tol);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

}  // namespace tsr

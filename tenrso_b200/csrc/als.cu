// FP64 kernels of the ALS sweep. Replace, from crates/tenrso-decomp/src/cp/:
//   compute_gram_matrix / compute_gram_hadamard   helpers.rs:409-452
//   solve_least_squares (per-row lstsq + ridge)   helpers.rs:455-495
//   compute_norm_squared / compute_fit            helpers.rs:498-579
//   convergence + oscillation bookkeeping          core.rs:142-166
// The per-row least-squares solves become one in-place Gauss-Jordan inverse of
// the symmetric Gram G (FP64, no pivoting: every pivot of an SPD matrix is
// positive, so a non-positive pivot is the "not SPD" signal that triggers the
// reference's ridge retry) and a row-parallel product M . G^-1.
// ||Xhat||^2 and <X, Xhat> come from the Grams and the last mode's MTTKRP
// (mathematically identical to the extra mode-0 MTTKRP of helpers.rs:558-579).
// Grams are stored as their upper triangle (row a, column c >= a).
#include "als.cuh"
#include "sm100.cuh"

namespace tsr {

namespace {

// Upper triangle of U^T U accumulated into `gram` (pre-zeroed); the body is
// gram_rows_accumulate (als.cuh), rows_per_cta rows per CTA.
template <int RB>
__global__ void __launch_bounds__(256)
gram_kernel(const float* __restrict__ U, int64_t rows, int R, int64_t rows_per_cta,
            double* __restrict__ gram) {
  __shared__ double Us[kGramChunk * 16 * RB];
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_cta;
  const int64_t r1 = rows < r0 + rows_per_cta ? rows : r0 + rows_per_cta;
  gram_rows_accumulate<RB>(U, r0, r1, R, gram, Us);
}

__global__ void norm_sq_kernel(const float* __restrict__ X, int64_t n, double* out) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  const int64_t n4 = ((uintptr_t)X & 15) ? 0 : n / 4;
  const float4* X4 = reinterpret_cast<const float4*>(X);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n4; k += stride) {
    float4 v = __ldg(X4 + k);
    s0 += (double)v.x * v.x;
    s1 += (double)v.y * v.y;
    s2 += (double)v.z * v.z;
    s3 += (double)v.w * v.w;
  }
  for (int64_t k = n4 * 4 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride)
    s0 += (double)X[k] * X[k];
  double s = (s0 + s1) + (s2 + s3);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) atomicAdd(out, s);
  }
}

// Gauss-Jordan inverse of the (padded) Hadamard G in N/2 steps of 2 x 2
// pivot blocks, no pivoting.
//
// G is first scaled to unit diagonal, G' = D G D with D = diag(1/sqrt(G_ii)),
// so that G^-1 = D G'^-1 D. Step s eliminates the pivot pair K = {k, k+1},
// k = 2s, with the 2 x 2 block P = A[K][K] (symmetric and, for an SPD G,
// positive definite: its determinant is the product of two LDL^T pivots).
// One step is exactly the uniform rank-2 update
//   A <- A - U W^T,  U[i] = A[i][K]          (i not in K),  U[K] = P - I,
//                    W[j] = P^-1 A[K][j]     (j not in K),  W[K] = I + P^-1,
// which yields the pivot rows P^-1 A[K][j], the pivot columns -A[i][K] P^-1
// and the corner P^-1 without special cases (block form of the scalar
// identities u_k = p - 1, w_k = (p + 1) / p). P^-1 = adj(P) / det(P) costs one
// reciprocal per step. After steps 0..s-1 the matrix is symmetric within the
// processed and within the unprocessed indices and antisymmetric across them,
// so U follows from the pivot rows with the sign of the processed entries
// flipped: a step needs the two pivot rows only.
//
// Roles (kGjThreads = 512 threads = 16 warps; warp w runs on scheduler w % 4):
//   pivot warp 0      the serial chain, alone on its scheduler so that its
//                     dependent FP64 operations do not queue behind bulk FMAs.
//                     Lane l holds both rows of the next pivot pair at columns
//                     l + 32c. At step s it reads the 2 x 2 block of step s+1
//                     (its three entries follow from seven broadcast shared
//                     loads and two FMAs each, without waiting for the rows),
//                     applies step s to rows 2s+2, 2s+3 as staged during step
//                     s-1, and writes U and W of step s+1 for its columns.
//   bulk warps        the 12 warps on schedulers 1-3 (w % 4 != 0), a 16 x 24
//                     grid: thread (ty, tx) owns rows ty + 16a (a < RB) and
//                     columns tx + 24b (b < CB) in registers and only applies
//                     the published updates. During step s the owners of rows
//                     2s+4 and 2s+5 also copy them, updated through step s,
//                     into a staging buffer.
//   warps 4, 8, 12    idle (they keep scheduler 0 to the pivot warp).
// One barrier per step. A pivot that is not positive, not finite or below
// 1e-290 (a non-positive diagonal included) sets the "not SPD" flag, read once
// after the last step.
constexpr int kGjThreads = 512;
constexpr int kGjCW = 24;  // bulk grid width (columns per sweep of a thread)

template <int RB>
struct GjLayout {
  static constexpr int N = 16 * RB;                   // padded matrix size
  static constexpr int CB = (N + kGjCW - 1) / kGjCW;  // column blocks per bulk thread
  static constexpr int CP = (N + 31) / 32;            // pivot-warp columns per lane
};

__device__ __forceinline__ bool gj_bulk() { return ((threadIdx.x >> 5) & 3) != 0; }
// bulk thread index 0..383 (warps 1, 2, 3, 5, 6, 7, ... in order)
__device__ __forceinline__ int gj_bulk_index() {
  const int w = threadIdx.x >> 5;
  return gj_bulk() ? (w - (w >> 2) - 1) * 32 + (threadIdx.x & 31) : 0;
}

template <int RB>
struct GjShared {
  static constexpr int N = 16 * RB;
  double2 u[2][N];        // [buffer][row]: (U[i][0], U[i][1]) of the step
  double2 w[2][N];        // [buffer][column]: (W[j][0], W[j][1]) of the step
  double stage[2][2][N];  // [slot][pivot row of the pair][column]
  double dsc[N];          // the diagonal scaling 1 / sqrt(G_ii)
  double scale;
  int bad;
};

// 1/p by two Newton-Raphson steps x <- x (2 - p x) from the hardware
// approximation (rcp.approx.ftz.f64, about 20 correct bits -> 40 -> 80,
// i.e. FP64 rounding). Called for p in [1e-290, 1].
__device__ __forceinline__ double recip_nr(double p) {
  double x;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(p));
  x = x * fma(-p, x, 2.0);
  x = x * fma(-p, x, 2.0);
  return x;
}

// The pivot warp: r0/r1 hold rows k and k+1 (k even, their values after every
// earlier step) at columns lane + 32c, and (a, b, d) = (A[k][k], A[k][k+1],
// A[k+1][k+1]). Publishes U and W of the step into buffer `buf`.
template <int RB>
__device__ __forceinline__ void gj2_publish(const double (&r0)[GjLayout<RB>::CP],
                                            const double (&r1)[GjLayout<RB>::CP], double a,
                                            double b, double d, int k, int buf,
                                            GjShared<RB>& sh) {
  constexpr int N = GjLayout<RB>::N, CP = GjLayout<RB>::CP;
  const int lane = threadIdx.x & 31;
  const double det = fma(a, d, -(b * b));
  // LDL^T pivots a and det / a
  const bool good = a >= 1e-290 && det >= 1e-290 * a && isfinite(a) && isfinite(det);
  if (!good && lane == 0) sh.bad = 1;
  const double id = recip_nr(good ? det : 1.0);
  const double p00 = d * id, p01 = -b * id, p11 = a * id;  // P^-1 (symmetric)
#pragma unroll
  for (int c = 0; c < CP; ++c) {
    const int j = lane + 32 * c;
    if (j < N) {
      double w0 = fma(p00, r0[c], p01 * r1[c]), w1 = fma(p01, r0[c], p11 * r1[c]);
      double u0 = j < k ? -r0[c] : r0[c], u1 = j < k ? -r1[c] : r1[c];
      if (j == k) {
        w0 = 1.0 + p00;
        w1 = p01;
        u0 = a - 1.0;
        u1 = b;
      } else if (j == k + 1) {
        w0 = p01;
        w1 = 1.0 + p11;
        u0 = b;
        u1 = d - 1.0;
      }
      sh.w[buf][j] = make_double2(w0, w1);
      sh.u[buf][j] = make_double2(u0, u1);
    }
  }
}

// Whole CTA (kGjThreads). `a` is meaningful in the bulk threads only.
template <int RB>
__device__ bool gj_inverse(double (&a)[RB][GjLayout<RB>::CB], GjShared<RB>& sh) {
  constexpr int N = GjLayout<RB>::N, CB = GjLayout<RB>::CB, CP = GjLayout<RB>::CP;
  constexpr int STEPS = N / 2;
  const bool bulk = gj_bulk(), pivot = threadIdx.x < 32;
  const int t = gj_bulk_index(), ty = t / kGjCW, tx = t % kGjCW;
  const int lane = threadIdx.x & 31;
  // diagonal scaling (a non-positive diagonal scales its row to zero, whose
  // pivot then reports "not SPD")
  if (threadIdx.x == 0) sh.bad = 0;
  if (bulk) {
#pragma unroll
    for (int ai = 0; ai < RB; ++ai)
#pragma unroll
      for (int bj = 0; bj < CB; ++bj)
        if (ty + 16 * ai == tx + kGjCW * bj) {
          const double g = a[ai][bj];
          sh.dsc[ty + 16 * ai] = (g > 0.0 && isfinite(g)) ? rsqrt(g) : 0.0;
        }
  }
  __syncthreads();
  double di[RB], dj[CB];
#pragma unroll
  for (int ai = 0; ai < RB; ++ai) di[ai] = sh.dsc[ty + 16 * ai];
#pragma unroll
  for (int bj = 0; bj < CB; ++bj) dj[bj] = tx + kGjCW * bj < N ? sh.dsc[tx + kGjCW * bj] : 0.0;
  if (bulk) {
#pragma unroll
    for (int ai = 0; ai < RB; ++ai)
#pragma unroll
      for (int bj = 0; bj < CB; ++bj) a[ai][bj] *= di[ai] * dj[bj];
    // rows 0, 1 (step 0's pivots) into slot 0 and rows 2, 3 into slot 1
    if (ty < 4) {
#pragma unroll
      for (int bj = 0; bj < CB; ++bj)
        if (tx + kGjCW * bj < N) sh.stage[ty >> 1][ty & 1][tx + kGjCW * bj] = a[0][bj];
    }
  }
  __syncthreads();
  double r0[CP], r1[CP];  // pivot warp: the pair's two rows at columns lane + 32c
  if (pivot) {
#pragma unroll
    for (int c = 0; c < CP; ++c) {
      const int j = lane + 32 * c;
      r0[c] = j < N ? sh.stage[0][0][j] : 0.0;
      r1[c] = j < N ? sh.stage[0][1][j] : 0.0;
    }
    gj2_publish<RB>(r0, r1, sh.stage[0][0][0], sh.stage[0][0][1], sh.stage[0][1][1], 0, 0, sh);
  }
  __syncthreads();
#pragma unroll 1
  for (int s = 0; s < STEPS; ++s) {
    const int buf = s & 1, k = 2 * s;
    if (bulk) {
      double2 u[RB], w[CB];
#pragma unroll
      for (int ai = 0; ai < RB; ++ai) u[ai] = sh.u[buf][ty + 16 * ai];
#pragma unroll
      for (int bj = 0; bj < CB; ++bj)
        w[bj] = tx + kGjCW * bj < N ? sh.w[buf][tx + kGjCW * bj] : make_double2(0.0, 0.0);
#pragma unroll
      for (int ai = 0; ai < RB; ++ai)
#pragma unroll
        for (int bj = 0; bj < CB; ++bj)
          a[ai][bj] = fma(-u[ai].x, w[bj].x, fma(-u[ai].y, w[bj].y, a[ai][bj]));
      // rows k+4, k+5 (step s+2's pivots), updated through step s, to the
      // pivot warp: staged in slot s & 1
      const int k4 = k + 4;
      if (k4 < N && (ty >> 1) == ((k4 & 15) >> 1)) {
        const int ab = k4 >> 4;
#pragma unroll
        for (int bj = 0; bj < CB; ++bj) {
          double v = a[0][bj];
#pragma unroll
          for (int ai = 1; ai < RB; ++ai)
            if (ai == ab) v = a[ai][bj];
          if (tx + kGjCW * bj < N) sh.stage[buf][ty & 1][tx + kGjCW * bj] = v;
        }
      }
    } else if (pivot && s + 1 < STEPS) {
      // step s+1's pivot block first (seven broadcast loads, two FMAs each),
      // then rows k+2, k+3 as staged during step s-1 (slot (s+1) & 1) with
      // step s applied
      const int k2 = k + 2;
      const double2 ua = sh.u[buf][k2], ub = sh.u[buf][k2 + 1];
      const double2 wa = sh.w[buf][k2], wb = sh.w[buf][k2 + 1];
      const double* st0 = sh.stage[buf ^ 1][0];
      const double* st1 = sh.stage[buf ^ 1][1];
      const double pa = fma(-ua.x, wa.x, fma(-ua.y, wa.y, st0[k2]));
      const double pb = fma(-ua.x, wb.x, fma(-ua.y, wb.y, st0[k2 + 1]));
      const double pd = fma(-ub.x, wb.x, fma(-ub.y, wb.y, st1[k2 + 1]));
#pragma unroll
      for (int c = 0; c < CP; ++c) {
        const int j = lane + 32 * c;
        if (j < N) {
          const double2 wv = sh.w[buf][j];
          r0[c] = fma(-ua.x, wv.x, fma(-ua.y, wv.y, st0[j]));
          r1[c] = fma(-ub.x, wv.x, fma(-ub.y, wv.y, st1[j]));
        }
      }
      gj2_publish<RB>(r0, r1, pa, pb, pd, k2, buf ^ 1, sh);
    }
    __syncthreads();
  }
  if (sh.bad) return false;
  // G^-1 = D G'^-1 D
  if (bulk) {
#pragma unroll
    for (int ai = 0; ai < RB; ++ai)
#pragma unroll
      for (int bj = 0; bj < CB; ++bj) a[ai][bj] *= di[ai] * dj[bj];
  }
  return true;
}

// G(i, j) = prod_{m != mode} Gram_m(i, j) for this bulk thread's entries
// (rows ty + 16a, columns tx + 24b). All loads are issued before any store
// (grams and hadam are distinct buffers).
template <int RB>
__device__ void load_hadamard(const double* __restrict__ grams, double* __restrict__ hadam,
                              int ndim, int mode, int R, double ridge,
                              double (&a)[RB][GjLayout<RB>::CB], bool write_h) {
  constexpr int N = GjLayout<RB>::N, CB = GjLayout<RB>::CB;
  const int t = gj_bulk_index(), ty = t / kGjCW, tx = t % kGjCW;
  const int RR = R * R;
#pragma unroll
  for (int ai = 0; ai < RB; ++ai)
#pragma unroll
    for (int bj = 0; bj < CB; ++bj) a[ai][bj] = 1.0;  // helpers.rs:414 starts from ones
  for (int m = 0; m < ndim; ++m) {
    if (m == mode) continue;
    const double* g = grams + (int64_t)m * RR;
    double v[RB][CB];
#pragma unroll
    for (int ai = 0; ai < RB; ++ai)
#pragma unroll
      for (int bj = 0; bj < CB; ++bj) {
        const int i = ty + 16 * ai, j = tx + kGjCW * bj;
        v[ai][bj] = (i < R && j < R) ? __ldg(g + (i <= j ? i * R + j : j * R + i)) : 1.0;
      }
#pragma unroll
    for (int ai = 0; ai < RB; ++ai)
#pragma unroll
      for (int bj = 0; bj < CB; ++bj) a[ai][bj] *= v[ai][bj];
  }
#pragma unroll
  for (int ai = 0; ai < RB; ++ai)
#pragma unroll
    for (int bj = 0; bj < CB; ++bj) {
      const int i = ty + 16 * ai, j = tx + kGjCW * bj;
      if (i < R && j < R) {
        if (write_h) hadam[(int64_t)mode * RR + i * R + j] = a[ai][bj];
        if (i == j) a[ai][bj] += ridge;
      } else {
        // padding: identity block, inverted harmlessly (columns >= N unused)
        a[ai][bj] = (i == j && j < N) ? 1.0 : 0.0;
      }
    }
}

// a += l2 * I on this bulk thread's entries (the ridge of cp_als_constrained)
template <int RB>
__device__ __forceinline__ void add_diagonal(double (&a)[RB][GjLayout<RB>::CB], int R, double l2) {
  constexpr int CB = GjLayout<RB>::CB;
  const int t = gj_bulk_index(), ty = t / kGjCW, tx = t % kGjCW;
#pragma unroll
  for (int ai = 0; ai < RB; ++ai)
#pragma unroll
    for (int bj = 0; bj < CB; ++bj)
      if (ty + 16 * ai == tx + kGjCW * bj && ty + 16 * ai < R) a[ai][bj] += l2;
}

// Coefficient (i, j) of the finite-difference penalty that
// apply_tikhonov_to_gram (helpers.rs:630-700) adds, times lambda, to an
// n x n Gram: order 1 D1^T D1 (n >= 2; nothing for n < 2), order >= 2 the
// reference's banded second-order form (n >= 3; lambda I for n < 3).
__device__ __forceinline__ double tikhonov_coef(int i, int j, int n, int order) {
  if (order == 1) {
    if (n < 2) return 0.0;
    if (i == j) return (i == 0 || i == n - 1) ? 1.0 : 2.0;
    return (i - j == 1 || j - i == 1) ? -1.0 : 0.0;
  }
  if (n < 3) return i == j ? 1.0 : 0.0;
  if (i == j) return (i == 0 || i == n - 1) ? 1.0 : ((i == 1 || i == n - 2) ? 5.0 : 6.0);
  const int lo = i < j ? i : j, d = i < j ? j - i : i - j;
  if (d == 1) return (lo == 0 || lo == n - 2) ? -2.0 : -4.0;
  if (d == 2) return 1.0;
  return 0.0;
}

// a += lambda * P (the Tikhonov penalty of order > 0) on this bulk thread's
// entries.
template <int RB>
__device__ __forceinline__ void add_tikhonov(double (&a)[RB][GjLayout<RB>::CB], int R,
                                             double lambda, int order) {
  constexpr int CB = GjLayout<RB>::CB;
  const int t = gj_bulk_index(), ty = t / kGjCW, tx = t % kGjCW;
#pragma unroll
  for (int ai = 0; ai < RB; ++ai)
#pragma unroll
    for (int bj = 0; bj < CB; ++bj) {
      const int i = ty + 16 * ai, j = tx + kGjCW * bj;
      if (i < R && j < R) a[ai][bj] += lambda * tikhonov_coef(i, j, R, order);
    }
}

// fit, fit_history, oscillation and convergence rules (helpers.rs:513-530,
// core.rs:142-166) of the sweep whose last solve has finished, from the
// scalars that solve accumulated: ||X||^2 + ||Xhat||^2 - 2 <X, Xhat>. Called
// by a whole CTA; it ends with a barrier, after which every thread may read
// st->done.
__device__ void fit_update(const AlsBuffers& b, double tol) {
  AlsState* st = b.state;
  if (threadIdx.x == 0) {
    const double xn = __ldcg(&st->xnorm_sq);
    const double rn = __ldcg(&st->xhat_sq);
    const double inner = __ldcg(&st->inner);
    const double prev_fit = __ldcg(&st->prev_fit);
    const int iter = __ldcg(&st->iter);
    int osc = __ldcg(&st->osc);
    const double err_sq = xn + rn - 2.0 * inner;
    const double err = sqrt(fmax(err_sq, 0.0));
    double fit = 1.0 - err / sqrt(xn);
    fit = fmin(fmax(fit, 0.0), 1.0);
    st->fit = fit;
    b.history[iter] = fit;
    if (iter > 0 && fit < prev_fit) st->osc = ++osc;
    const double change = fabs(fit - prev_fit);
    st->final_change = change;
    st->iter = iter + 1;
    st->fit_pending = 0;
    if (iter > 0 && change < tol) {
      st->reason = TSR_REASON_FIT_TOLERANCE;
      st->done = 1;
    } else if (osc > 5 && iter > 10) {
      st->reason = TSR_REASON_OSCILLATION;
      st->done = 1;
    } else {
      st->prev_fit = fit;
    }
    __threadfence_block();
  }
  __syncthreads();
}

__global__ void clamp_nonneg_kernel(float* __restrict__ U, int64_t n) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    U[e] = fmaxf(U[e], 0.f);
}

__global__ void any_negative_kernel(const float* __restrict__ X, int64_t n, int* flag) {
  bool neg = false;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    neg |= __ldg(X + e) < 0.f;
  if (__any_sync(0xffffffffu, neg) && (threadIdx.x & 31) == 0) *flag = 1;
}

__global__ void fit_kernel(AlsBuffers b, double tol) {
  AlsState* st = b.state;
  if (st->done || !st->fit_pending) return;
  fit_update(b, tol);
}

// One CTA: G = Hadamard of the other Grams and G^-1 (ridge retry, as
// solve_least_squares does, helpers.rs:477-490); zeroes this mode's Gram
// accumulator (and <X,Xhat> for the last mode) for the solve that follows.
template <int RB>
__global__ void __launch_bounds__(kGjThreads, 1) chol_kernel(AlsBuffers b, int ndim, int mode, int R,
                                                   float ridge_eps, int last, double tol,
                                                   double l2, int tik_order, double tik_lambda,
                                                   TraceSlot tr) {
  __shared__ GjShared<RB> gsh;
  trace_begin(tr);
  AlsState* st = b.state;
  if (st->done) return;
  if (mode == 0 && st->fit_pending) {
    // the previous sweep's fit and stopping rules come first: a sweep that
    // stops the run leaves the factors as they are (core.rs:142-166)
    fit_update(b, tol);
    if (*(volatile int*)&st->done) return;
  }
  const int RR = R * R;
  // the bulk warps hold the matrix (16 x 24 grid); warp 0 is the inverse's
  // pivot warp
  const bool bulk = gj_bulk();
  double a[RB][GjLayout<RB>::CB];
  if (bulk) {
    load_hadamard<RB>(b.grams, b.hadam, ndim, mode, R, 0.0, a, true);
    if (l2 != 0.0) add_diagonal<RB>(a, R, l2);
    if (tik_order > 0) add_tikhonov<RB>(a, R, tik_lambda, tik_order);
  }
  // solve_least_squares solves gram^T x = b (helpers.rs:462,471); G is
  // symmetric by construction so G^T = G.
  bool ok = gj_inverse<RB>(a, gsh);
  if (!ok) {
    __syncthreads();
    if (bulk) {
      load_hadamard<RB>(b.grams, b.hadam, ndim, mode, R, (double)ridge_eps, a, false);
      if (l2 != 0.0) add_diagonal<RB>(a, R, l2);
      if (tik_order > 0) add_tikhonov<RB>(a, R, tik_lambda, tik_order);
    }
    ok = gj_inverse<RB>(a, gsh);
    if (threadIdx.x == 0) st->ridge_used = 1;
  }
  if (!ok) {
    // lstsq (the reference's solver) returns a least-squares solution for a
    // numerically singular Gram; the Cholesky-type stand-in needs a ridge on
    // the scale of G for that: eps * rank * 10 times the mean diagonal.
    __syncthreads();
    if (threadIdx.x == 0) gsh.scale = 0.0;
    __syncthreads();
    const double* H = b.hadam + (int64_t)mode * RR;
    if (threadIdx.x < 32) {
      double d = 0.0;
      for (int i = threadIdx.x; i < R; i += 32) d += fabs(H[i * R + i]);
      for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
      if (threadIdx.x == 0) gsh.scale = d / R;
    }
    __syncthreads();
    if (bulk) {
      load_hadamard<RB>(b.grams, b.hadam, ndim, mode, R,
                        (double)ridge_eps * fmax(gsh.scale, 1.0), a, false);
      if (l2 != 0.0) add_diagonal<RB>(a, R, l2);
      if (tik_order > 0) add_tikhonov<RB>(a, R, tik_lambda, tik_order);
    }
    ok = gj_inverse<RB>(a, gsh);
    if (threadIdx.x == 0) st->ridge_used = 2;
  }
  if (!ok) {
    if (threadIdx.x == 0) {
      st->status |= DS_NOT_SPD;
      st->done = 1;
    }
    return;
  }
  if (bulk) {
    const int t = gj_bulk_index(), ty = t / kGjCW, tx = t % kGjCW;
#pragma unroll
    for (int ai = 0; ai < RB; ++ai)
#pragma unroll
      for (int bj = 0; bj < GjLayout<RB>::CB; ++bj) {
        const int i = ty + 16 * ai, j = tx + kGjCW * bj;
        if (i < R && j < R) b.ginv[i * R + j] = a[ai][bj];
      }
  }
  double* gm = b.grams + (int64_t)mode * RR;
  for (int e = threadIdx.x; e < RR; e += blockDim.x) gm[e] = 0.0;
  if (last && threadIdx.x == 0) {
    st->inner = 0.0;
    st->xhat_sq = 0.0;
  }
  trace_end(tr);
}

// Thread groups per element in the split sums of a chunk of `full` outputs:
// 256 threads cover full / 4 float4 columns (R a multiple of 4) or `full`
// scalars, the rest of the threads take interleaved subsets of the splits.
__host__ __device__ inline int solve_groups(int full, int R) {
  const int cols = (R & 3) == 0 ? full / 4 : full;
  return cols >= 256 ? 1 : 256 / cols;
}


// U_mode = (sum over splits of the partial MTTKRP) . G^-1, then the Gram of
// the new factor, U^T U (upper triangle, FP64, into `gram`, which the inverse
// kernel of this mode zeroed), and for the last mode <M, U> = <X, Xhat> and,
// in the CTA that finishes last, the fit and the stopping rules.
//
// Launched with programmatic dependent launch after the MTTKRP: G^-1 (from
// the inverse kernel, a full dependency) is staged before the wait for the
// MTTKRP grid.
//
// Each CTA walks chunks of rpc rows (grid-strided): the split partials of a
// chunk are summed in FP64 into shared memory (float4 loads, 16 in flight per
// thread, the threads beyond one per column group taking interleaved subsets
// of the splits), multiplied by G^-1 (shared), rounded to fp32 for U, and the
// rounded rows are added into the thread's RB x RB block of the Gram (thread
// (ty, tx) owns entries (ty + 16a, tx + 16b), as in gram_kernel); one FP64
// atomic per owned upper entry at the end. Products of fp32 values are exact
// in FP64, so the Gram equals gram_kernel's up to the order of the sums.
template <int RB>
__global__ void __launch_bounds__(256)
solve_kernel(AlsBuffers b, const float* __restrict__ partials, int splits, int64_t rows, int R,
             int rpc, float* __restrict__ U, double* __restrict__ gram, int last, int ndim,
             double tol, float l1, int nonneg, uint8_t* __restrict__ bimg, int img_n_pad,
             TraceSlot tr) {
  extern __shared__ __align__(16) double sh[];
  __shared__ __align__(8) uint64_t gi_bar;
  __shared__ int gi_state;  // 0 copy in flight, 1 landed, 2 gave up
  trace_begin(tr);
  if (threadIdx.x == 0) grid_dep_trigger();
  AlsState* st = b.state;
  if (st->done) return;
  const int RR = R * R;
  double* Gi = sh;               // R x R
  double* Ms = Gi + RR;          // rpc x R  (FP64 MTTKRP rows)
  double* Us = Ms + rpc * R;     // rpc x R  (the fp32 factor rows, widened)
  double* red = Us + rpc * R;    // [groups][rpc x R]
  // G^-1 (a full dependency, complete at launch) comes in by bulk async
  // copies that overlap the split sums when its size is a multiple of 16 B
  // (R even); else by plain loads
  const uint32_t gi_bytes = (uint32_t)RR * 8u;
  const bool gi_bulk = (gi_bytes & 15u) == 0;
  if (gi_bulk) {
    if (threadIdx.x == 0) {
      gi_state = 0;
      sm100::mbar_init(&gi_bar, 1);
      sm100::fence_barrier_init();
      sm100::mbar_arrive_expect_tx(&gi_bar, gi_bytes);
      for (uint32_t off = 0; off < gi_bytes; off += 16384u) {
        const uint32_t n = gi_bytes - off < 16384u ? gi_bytes - off : 16384u;
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(sm100::smem_u32((const char*)Gi + off)),
            "l"((const char*)b.ginv + off), "r"(n), "r"(sm100::smem_u32(&gi_bar))
            : "memory");
      }
    }
  } else {
#pragma unroll 8
    for (int e = threadIdx.x; e < RR; e += blockDim.x) Gi[e] = __ldg(b.ginv + e);
  }
  // the partials come from the MTTKRP that precedes this kernel in its stream
  grid_dep_wait();
  const int64_t pstride = rows * R;
  const int full = rpc * R;
  const int groups = solve_groups(full, R);
  // float4 loads of the partials when rows of R floats keep 16-byte alignment
  const bool vec = (R & 3) == 0 && ((uintptr_t)partials & 15) == 0;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[RB][RB];
#pragma unroll
  for (int ai = 0; ai < RB; ++ai)
#pragma unroll
    for (int bj = 0; bj < RB; ++bj) acc[ai][bj] = 0.0;
  double ip = 0.0;
  for (int64_t r0 = (int64_t)blockIdx.x * rpc; r0 < rows; r0 += (int64_t)gridDim.x * rpc) {
    const int nr = (int)(rows - r0 < rpc ? rows - r0 : rpc);
    const int ne = nr * R;
    __syncthreads();  // G^-1 staged; the previous chunk's Ms / Us are consumed
    if (vec) {
      const int ne4 = ne >> 2;
      const int64_t pstride4 = pstride >> 2;
      for (int t = threadIdx.x; t < ne4 * groups; t += blockDim.x) {
        const int e4 = t % ne4, g = t / ne4;
        const float4* p = reinterpret_cast<const float4*>(partials + r0 * R) + e4;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int q = g;
        for (; q + 15 * groups < splits; q += 16 * groups) {
          float4 v[16];
#pragma unroll
          for (int u = 0; u < 16; ++u) v[u] = __ldg(p + (int64_t)(q + u * groups) * pstride4);
#pragma unroll
          for (int u = 0; u < 16; ++u) {
            s0 += (double)v[u].x;
            s1 += (double)v[u].y;
            s2 += (double)v[u].z;
            s3 += (double)v[u].w;
          }
        }
        for (; q < splits; q += groups) {
          const float4 v = __ldg(p + (int64_t)q * pstride4);
          s0 += (double)v.x;
          s1 += (double)v.y;
          s2 += (double)v.z;
          s3 += (double)v.w;
        }
        double* r = red + g * ne + 4 * e4;
        r[0] = s0;
        r[1] = s1;
        r[2] = s2;
        r[3] = s3;
      }
    } else {
      for (int t = threadIdx.x; t < ne * groups; t += blockDim.x) {
        const int e = t % ne, g = t / ne;
        const float* p = partials + r0 * R + e;
        double s = 0.0;
        int q = g;
        for (; q + 15 * groups < splits; q += 16 * groups) {
          float v[16];
#pragma unroll
          for (int u = 0; u < 16; ++u) v[u] = __ldg(p + (int64_t)(q + u * groups) * pstride);
#pragma unroll
          for (int u = 0; u < 16; ++u) s += (double)v[u];
        }
        for (; q < splits; q += groups) s += (double)__ldg(p + (int64_t)q * pstride);
        red[g * ne + e] = s;
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ne; e += blockDim.x) {
      double s = 0.0;
      for (int g = 0; g < groups; ++g) s += red[g * ne + e];
      Ms[e] = s;
    }
    if (gi_bulk && threadIdx.x == 0 && gi_state == 0) {
      // bounded wait (~1 s); on timeout report, and let the copy land (again
      // bounded) before the CTA may exit
      long long t0 = clock64();
      bool ok;
      while (!(ok = sm100::mbar_try_wait(&gi_bar, 0)) && clock64() - t0 < (1ll << 31)) {
      }
      if (!ok) {
        atomicOr(&st->status, DS_TIMEOUT);
        st->done = 1;
        t0 = clock64();
        while (!sm100::mbar_try_wait(&gi_bar, 0) && clock64() - t0 < (1ll << 31)) {
        }
      }
      gi_state = ok ? 1 : 2;
    }
    __syncthreads();
    if (gi_bulk && gi_state == 2) return;
    for (int e = threadIdx.x; e < ne; e += blockDim.x) {
      const int i = e / R, c = e % R;
      double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;  // four chains for ILP
      int k = 0;
      for (; k + 4 <= R; k += 4) {
        s0 += Ms[i * R + k] * Gi[k * R + c];
        s1 += Ms[i * R + k + 1] * Gi[(k + 1) * R + c];
        s2 += Ms[i * R + k + 2] * Gi[(k + 2) * R + c];
        s3 += Ms[i * R + k + 3] * Gi[(k + 3) * R + c];
      }
      for (; k < R; ++k) s0 += Ms[i * R + k] * Gi[k * R + c];
      float v = (float)((s0 + s1) + (s2 + s3));
      // cp_als_constrained: soft threshold (helpers.rs:610-623), then the
      // projection onto v >= 0 (core.rs:356-359)
      if (l1 > 0.f) v = v > l1 ? v - l1 : (v < -l1 ? v + l1 : 0.f);
      if (nonneg) v = fmaxf(v, 0.f);
      U[(r0 + i) * R + c] = v;
      if (bimg) {
        // the new entry's bf16 hi/lo halves into the next MTTKRP's B image:
        // k-block k >> 6, rows c (hi) and img_n_pad + c (lo), 16-byte chunk
        // (k & 63) >> 3 at its 128-byte-swizzled position, element k & 7
        const int64_t k = r0 + i;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
        uint8_t* tile = bimg + (size_t)(k >> 6) * 2 * img_n_pad * 128;
        const int cq = (int)((k & 63) >> 3), el = (int)(k & 7) * 2;
        const int rh = c, rl = img_n_pad + c;
        *reinterpret_cast<__nv_bfloat16*>(tile + rh * 128 + ((cq ^ (rh & 7)) << 4) + el) = h;
        *reinterpret_cast<__nv_bfloat16*>(tile + rl * 128 + ((cq ^ (rl & 7)) << 4) + el) = l;
      }
      Us[e] = (double)v;
      ip += Ms[e] * (double)v;
    }
    __syncthreads();
    for (int i = 0; i < nr; ++i) {
      double x[RB], y[RB];
#pragma unroll
      for (int ai = 0; ai < RB; ++ai) {
        const int a = ty + 16 * ai;
        x[ai] = a < R ? Us[i * R + a] : 0.0;
      }
#pragma unroll
      for (int bj = 0; bj < RB; ++bj) {
        const int c = tx + 16 * bj;
        y[bj] = c < R ? Us[i * R + c] : 0.0;
      }
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
  if (!last) {
    trace_end(tr);
    return;
  }
  // ||Xhat||^2 = sum_ac H_ac (U^T U)_ac with H the Hadamard of the other
  // Grams (this mode's inverse kernel wrote it): this CTA's share from its
  // Gram blocks, off-diagonal entries counted twice
  const double* H = b.hadam + (int64_t)(ndim - 1) * RR;
  double xs = 0.0;
#pragma unroll
  for (int ai = 0; ai < RB; ++ai)
#pragma unroll
    for (int bj = 0; bj < RB; ++bj) {
      const int a = ty + 16 * ai, c = tx + 16 * bj;
      if (a < R && c < R && c >= a) xs += (c == a ? 1.0 : 2.0) * __ldg(H + a * R + c) * acc[ai][bj];
    }
  // one atomic per CTA for each sum (same-address atomics serialise at L2)
  for (int o = 16; o > 0; o >>= 1) {
    ip += __shfl_down_sync(0xffffffffu, ip, o);
    xs += __shfl_down_sync(0xffffffffu, xs, o);
  }
  __syncthreads();  // the chunk loop's shared buffers are no longer read
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = ip;
    red[8 + (threadIdx.x >> 5)] = xs;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0, x = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      s += red[w];
      x += red[8 + w];
    }
    atomicAdd(&st->inner, s);
    atomicAdd(&st->xhat_sq, x);
  }
  // the fit of this sweep is formed by the next inverse kernel (or by
  // fit_kernel after the last sweep), once this grid's atomics are complete
  if (blockIdx.x == 0 && threadIdx.x == 0) st->fit_pending = 1;
  trace_end(tr);
}

// orthonormalize_factor, step 1 (one CTA): the Cholesky factor R of the
// factor's Gram (upper triangle in gram, from the solve), R^-1 into b.ginv;
// gram (and, for the last mode, <X, Xhat> and ||Xhat||^2) zeroed for step 2.
__global__ void __launch_bounds__(256) orth_chol_kernel(AlsBuffers b, int R, double* gram,
                                                        int last) {
  extern __shared__ __align__(16) double oa[];  // R x R working copy
  __shared__ int bad;
  AlsState* st = b.state;
  if (st->done) return;
  if (threadIdx.x == 0) bad = 0;
  for (int e = threadIdx.x; e < R * R; e += blockDim.x) {
    const int i = e / R, j = e % R;
    oa[e] = i <= j ? gram[i * R + j] : 0.0;
  }
  __syncthreads();
  // right-looking Cholesky on the upper triangle: row k of R, then the
  // trailing update
  for (int k = 0; k < R; ++k) {
    if (threadIdx.x == 0) {
      const double d = oa[k * R + k];
      if (!(d > 0.0) || !isfinite(d)) bad = 1;
      oa[k * R + k] = sqrt(fmax(d, 0.0));
    }
    __syncthreads();
    if (bad) break;
    const double dk = oa[k * R + k];
    for (int j = k + 1 + threadIdx.x; j < R; j += blockDim.x) oa[k * R + j] /= dk;
    __syncthreads();
    const int m = R - k - 1;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int i = k + 1 + e / m, j = k + 1 + e % m;
      if (i <= j) oa[i * R + j] -= oa[k * R + i] * oa[k * R + j];
    }
    __syncthreads();
  }
  if (bad) {
    if (threadIdx.x == 0) {
      st->status |= DS_NOT_SPD;
      st->done = 1;
    }
    return;
  }
  // R^-1 (upper triangular), one column per thread by back substitution
  for (int j = threadIdx.x; j < R; j += blockDim.x) {
    double* x = b.ginv + j;  // column j, stride R
    for (int i = j + 1; i < R; ++i) x[i * R] = 0.0;
    x[j * R] = 1.0 / oa[j * R + j];
    for (int i = j - 1; i >= 0; --i) {
      double t = 0.0;
      for (int l = i + 1; l <= j; ++l) t += oa[i * R + l] * x[l * R];
      x[i * R] = -t / oa[i * R + i];
    }
  }
  for (int e = threadIdx.x; e < R * R; e += blockDim.x) gram[e] = 0.0;
  if (last && threadIdx.x == 0) {
    st->inner = 0.0;
    st->xhat_sq = 0.0;
  }
}

// orthonormalize_factor, step 2: Q = U R^-1 row by row (FP64, stored fp32),
// Q^T Q into gram (upper triangle, FP64 atomics) and, for the last mode,
// <M, Q> (M = the sum of the split partials) and ||Xhat||^2 = sum(H o Q^T Q).
template <int RB>
__global__ void __launch_bounds__(256)
orth_apply_kernel(AlsBuffers b, int ndim, int R, int64_t rows, float* __restrict__ U,
                  double* __restrict__ gram, int last, const float* __restrict__ partials,
                  int splits) {
  extern __shared__ __align__(16) double os[];
  __shared__ double red[16];
  AlsState* st = b.state;
  if (st->done) return;
  constexpr int rpc = 16;
  double* Ri = os;            // R x R
  double* Qs = os + R * R;    // rpc x R
  for (int e = threadIdx.x; e < R * R; e += blockDim.x) Ri[e] = b.ginv[e];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[RB][RB];
#pragma unroll
  for (int ai = 0; ai < RB; ++ai)
#pragma unroll
    for (int bj = 0; bj < RB; ++bj) acc[ai][bj] = 0.0;
  double ip = 0.0;
  const int64_t pstride = rows * R;
  for (int64_t r0 = (int64_t)blockIdx.x * rpc; r0 < rows; r0 += (int64_t)gridDim.x * rpc) {
    const int nr = (int)(rows - r0 < rpc ? rows - r0 : rpc);
    __syncthreads();
    for (int e = threadIdx.x; e < nr * R; e += blockDim.x) {
      const int i = e / R, c = e % R;
      const float* u = U + (r0 + i) * R;
      double q = 0.0;
      for (int k = 0; k <= c; ++k) q = fma((double)u[k], Ri[k * R + c], q);
      Qs[e] = q;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nr * R; e += blockDim.x) {
      const float qf = (float)Qs[e];
      const int64_t g = r0 * R + e;
      U[g] = qf;
      Qs[e] = (double)qf;  // the stored value enters the Gram and the fit
      if (last) {
        double m = 0.0;
        for (int p = 0; p < splits; ++p) m += (double)partials[(int64_t)p * pstride + g];
        ip += m * (double)qf;
      }
    }
    __syncthreads();
    for (int i = 0; i < nr; ++i) {
      double x[RB], y[RB];
#pragma unroll
      for (int ai = 0; ai < RB; ++ai) x[ai] = ty + 16 * ai < R ? Qs[i * R + ty + 16 * ai] : 0.0;
#pragma unroll
      for (int bj = 0; bj < RB; ++bj) y[bj] = tx + 16 * bj < R ? Qs[i * R + tx + 16 * bj] : 0.0;
#pragma unroll
      for (int ai = 0; ai < RB; ++ai)
#pragma unroll
        for (int bj = 0; bj < RB; ++bj) acc[ai][bj] = fma(x[ai], y[bj], acc[ai][bj]);
    }
  }
  double xs = 0.0;
  const double* H = b.hadam + (int64_t)(ndim - 1) * R * R;
#pragma unroll
  for (int ai = 0; ai < RB; ++ai)
#pragma unroll
    for (int bj = 0; bj < RB; ++bj) {
      const int a = ty + 16 * ai, c = tx + 16 * bj;
      if (a < R && c < R && c >= a) {
        atomicAdd(gram + a * R + c, acc[ai][bj]);
        if (last) xs += (c == a ? 1.0 : 2.0) * __ldg(H + a * R + c) * acc[ai][bj];
      }
    }
  if (!last) return;
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
    double a = 0.0, x = 0.0;
    for (int w = 0; w < 8; ++w) {
      a += red[w];
      x += red[8 + w];
    }
    atomicAdd(&st->inner, a);
    atomicAdd(&st->xhat_sq, x);
  }
}

}  // namespace

int launch_orthonormalize(tsr_ctx* ctx, cudaStream_t s, const AlsBuffers& b, int ndim, int mode,
                          int R, int64_t rows, float* U, double* gram, bool last,
                          const float* partials, int splits) {
  (void)mode;
  if (R > kMaxRank) return fail(TSR_E_UNSUPPORTED, "rank %d too large for the FP64 solve", R);
  orth_chol_kernel<<<1, 256, sizeof(double) * R * R, s>>>(b, R, gram, last ? 1 : 0);
  const unsigned grid = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(ceil_div(rows, 16), 2 * (int64_t)ctx->sm_count));
  const size_t smem = sizeof(double) * ((size_t)R * R + 16 * (size_t)R);
#define TSR_ORTH(RB)                                                                  \
  orth_apply_kernel<RB><<<grid, 256, smem, s>>>(b, ndim, R, rows, U, gram, last ? 1 : 0, \
                                                partials, splits)
  switch ((R + 15) / 16) {
    case 1: TSR_ORTH(1); break;
    case 2: TSR_ORTH(2); break;
    case 3: TSR_ORTH(3); break;
    case 4: TSR_ORTH(4); break;
    case 5: TSR_ORTH(5); break;
    case 6: TSR_ORTH(6); break;
    default: TSR_ORTH(7); break;
  }
#undef TSR_ORTH
  ctx->launches += 2;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

void init_als_attributes() {
  cudaFuncSetAttribute(orth_chol_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(sizeof(double) * kMaxRank * kMaxRank));
  cudaFuncSetAttribute(orth_apply_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(orth_apply_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(orth_apply_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(orth_apply_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(orth_apply_kernel<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(orth_apply_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(orth_apply_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(solve_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(solve_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(solve_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(solve_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(solve_kernel<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(solve_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(solve_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

int launch_gram(tsr_ctx* ctx, cudaStream_t s, const float* U, int64_t rows, int R,
                double* gram, bool zero_first) {
  if (R > kMaxRank) return fail(TSR_E_UNSUPPORTED, "rank %d too large", R);
  if (zero_first) TSR_CUDA(cudaMemsetAsync(gram, 0, sizeof(double) * R * R, s));
  int64_t ctas = std::min<int64_t>(ceil_div(rows, 16), 2 * ctx->sm_count);
  int64_t rpc = ceil_div(rows, ctas);
  ctas = ceil_div(rows, rpc);
  const unsigned g = (unsigned)ctas;
  switch ((R + 15) / 16) {
    case 1: gram_kernel<1><<<g, 256, 0, s>>>(U, rows, R, rpc, gram); break;
    case 2: gram_kernel<2><<<g, 256, 0, s>>>(U, rows, R, rpc, gram); break;
    case 3: gram_kernel<3><<<g, 256, 0, s>>>(U, rows, R, rpc, gram); break;
    case 4: gram_kernel<4><<<g, 256, 0, s>>>(U, rows, R, rpc, gram); break;
    case 5: gram_kernel<5><<<g, 256, 0, s>>>(U, rows, R, rpc, gram); break;
    case 6: gram_kernel<6><<<g, 256, 0, s>>>(U, rows, R, rpc, gram); break;
    default: gram_kernel<7><<<g, 256, 0, s>>>(U, rows, R, rpc, gram); break;
  }
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_norm_sq(tsr_ctx* ctx, cudaStream_t s, const float* X, int64_t n, double* out) {
  const int grid = ctx->sm_count * 8;
  norm_sq_kernel<<<grid, 256, 0, s>>>(X, n, out);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_chol(tsr_ctx* ctx, cudaStream_t s, const AlsBuffers& b, int ndim, int mode, int R,
                float ridge_eps, bool last, double tol, double l2, int tik_order,
                double tik_lambda) {
  if (R > kMaxRank) return fail(TSR_E_UNSUPPORTED, "rank %d too large for the FP64 solve", R);
  const TraceSlot tr = trace_slot(ctx, TRACE_INVERSE, mode);
  const int lst = last ? 1 : 0;
  switch ((R + 15) / 16) {
#define TSR_CHOL(RB)                                                                       \
  chol_kernel<RB><<<1, kGjThreads, 0, s>>>(b, ndim, mode, R, ridge_eps, lst, tol, l2, tik_order, \
                                           tik_lambda, tr)
    case 1: TSR_CHOL(1); break;
    case 2: TSR_CHOL(2); break;
    case 3: TSR_CHOL(3); break;
    case 4: TSR_CHOL(4); break;
    case 5: TSR_CHOL(5); break;
    case 6: TSR_CHOL(6); break;
    default: TSR_CHOL(7); break;
#undef TSR_CHOL
  }
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_clamp_nonneg(tsr_ctx* ctx, cudaStream_t s, float* U, int64_t n) {
  if (n <= 0) return TSR_OK;
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(n, 256), 4 * (int64_t)ctx->sm_count);
  clamp_nonneg_kernel<<<grid, 256, 0, s>>>(U, n);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_any_negative(tsr_ctx* ctx, cudaStream_t s, const float* X, int64_t n, int* flag) {
  if (n <= 0) return TSR_OK;
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(n, 256), 4 * (int64_t)ctx->sm_count);
  any_negative_kernel<<<grid, 256, 0, s>>>(X, n, flag);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_fit(tsr_ctx* ctx, cudaStream_t s, const AlsBuffers& b, int ndim, int R, double tol) {
  fit_kernel<<<1, 32, 0, s>>>(b, tol);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

int launch_solve(tsr_ctx* ctx, cudaStream_t s, const AlsBuffers& b, const float* partials,
                 int splits, int64_t rows, int R, float* U, double* gram, bool last, int ndim,
                 double tol, float l1, int nonneg, uint8_t* bimg, int img_n_pad) {
  if (R > kMaxRank) return fail(TSR_E_UNSUPPORTED, "rank %d too large for the FP64 solve", R);
  // about 64 row chunks (one per CTA) for small modes, so that the Gram
  // atomics stay few; 16-row chunks grid-strided over at most 8 CTAs per SM
  // for large ones
  const int rpc = (int)std::max<int64_t>(1, std::min<int64_t>(16, ceil_div(rows, 64)));
  const unsigned grid =
      (unsigned)std::min<int64_t>(ceil_div(rows, rpc), 8 * (int64_t)ctx->sm_count);
  const int full = rpc * R;
  const int groups = solve_groups(full, R);
  const size_t smem = (size_t)(R * R + 2 * full + (size_t)groups * full) * sizeof(double);
  if (smem > 200 * 1024) return fail(TSR_E_UNSUPPORTED, "rank %d too large for the FP64 solve", R);
  const int lst = last ? 1 : 0;
  // the mode is the Gram slot this solve accumulates into
  const TraceSlot tr = trace_slot(ctx, TRACE_SOLVE, (int)((gram - b.grams) / ((int64_t)R * R)));
#define TSR_SOLVE(RB)                                                                    \
  TSR_CUDA(launch_pdl(solve_kernel<RB>, dim3(grid), dim3(256), smem, s, b, partials, splits, \
                      rows, R, rpc, U, gram, lst, ndim, tol, l1, nonneg, bimg, img_n_pad, tr))
  switch ((R + 15) / 16) {
    case 1: TSR_SOLVE(1); break;
    case 2: TSR_SOLVE(2); break;
    case 3: TSR_SOLVE(3); break;
    case 4: TSR_SOLVE(4); break;
    case 5: TSR_SOLVE(5); break;
    case 6: TSR_SOLVE(6); break;
    default: TSR_SOLVE(7); break;
  }
#undef TSR_SOLVE
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

}  // namespace tsr

// FP64 Gram / Cholesky / solve / fit kernels of the ALS sweep.
#pragma once
#include "common.cuh"

namespace tsr {

constexpr int kMaxRank = 112;  // two R x R FP64 matrices fit in shared memory

// Device-resident ALS bookkeeping mirroring cp/core.rs:101-166.
struct AlsState {
  double xnorm_sq;      // ||X||^2 (FP64)
  double inner;         // <X, Xhat> accumulated by the last mode's solve
  double xhat_sq;       // ||Xhat||^2 = sum(H_last o Gram_last), same solve
  double prev_fit;
  double fit;
  double final_change;
  int iter;             // iterations completed
  int osc;              // oscillation_count
  int reason;           // tsr_reason
  int done;             // stop flag: converged, oscillation or error
  unsigned status;      // DevStatus bits
  int ridge_used;
  int fit_pending;      // the last solve of a sweep ran; its fit is not formed yet
  int pad;
};

// Upper triangle of U[r0:r1]^T U[r0:r1] added into `gram` (row a, column
// c >= a) with one FP64 atomic per entry per CTA of 256 threads. Thread
// (ty, tx) of a 16 x 16 grid owns entries (ty + 16a, tx + 16b); rows are
// staged through shared memory (Us: kGramChunk * 16 * RB doubles) in chunks,
// so a row costs 2*RB shared loads for RB*RB FMAs. Products of fp32 values
// are exact in FP64.
constexpr int kGramChunk = 32;
template <int RB>
__device__ __forceinline__ void gram_rows_accumulate(const float* __restrict__ U, int64_t r0,
                                                     int64_t r1, int R, double* __restrict__ gram,
                                                     double* Us) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[RB][RB];
#pragma unroll
  for (int ai = 0; ai < RB; ++ai)
#pragma unroll
    for (int bj = 0; bj < RB; ++bj) acc[ai][bj] = 0.0;
  const int LD = 16 * RB;
  for (int64_t c0 = r0; c0 < r1; c0 += kGramChunk) {
    const int nr = (int)(r1 - c0 < kGramChunk ? r1 - c0 : kGramChunk);
    __syncthreads();
#pragma unroll 4
    for (int k = threadIdx.x; k < nr * LD; k += 256) {
      const int i = k / LD, c = k % LD;
      Us[k] = c < R ? (double)__ldg(U + (c0 + i) * R + c) : 0.0;
    }
    __syncthreads();
    for (int i = 0; i < nr; ++i) {
      double x[RB], y[RB];
#pragma unroll
      for (int ai = 0; ai < RB; ++ai) x[ai] = Us[i * LD + ty + 16 * ai];
#pragma unroll
      for (int bj = 0; bj < RB; ++bj) y[bj] = Us[i * LD + tx + 16 * bj];
#pragma unroll
      for (int ai = 0; ai < RB; ++ai)
#pragma unroll
        for (int bj = 0; bj < RB; ++bj) acc[ai][bj] += x[ai] * y[bj];
    }
  }
#pragma unroll
  for (int ai = 0; ai < RB; ++ai)
#pragma unroll
    for (int bj = 0; bj < RB; ++bj) {
      const int a = ty + 16 * ai, c = tx + 16 * bj;
      if (a < R && c < R && c >= a) atomicAdd(gram + a * R + c, acc[ai][bj]);
    }
}

// the state occupies the first 256 bytes of its buffer, the fit history follows
static_assert(sizeof(AlsState) <= 256, "AlsState must fit its 256-byte slot");

struct AlsBuffers {
  double* grams;    // [N][R][R]   U_m^T U_m
  double* hadam;    // [N][R][R]   Hadamard of the other Grams (G_n)
  double* ginv;     // [R][R]      G_n^{-1} of the current mode
  AlsState* state;
  double* history;  // [max_iters]
};

// 16 x 16 Gauss-Jordan inverse held by one warp: lane owns P[r][c] for
// r = (lane >> 4) + 2q (q < 8), c = lane & 15. Pivot rows/columns move by
// shuffles; returns false on a pivot that is not positive or not finite.
__device__ __forceinline__ bool warp_gj16(double (&v)[8], int lane) {
  const int c = lane & 15, r0 = lane >> 4;
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int krow_lane = (k & 1) * 16;  // lanes holding row k
    const double p = __shfl_sync(0xffffffffu, v[k >> 1], krow_lane + k);
    const double pkc = __shfl_sync(0xffffffffu, v[k >> 1], krow_lane + c);
    double prk[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) prk[q] = __shfl_sync(0xffffffffu, v[q], r0 * 16 + k);
    ok = ok && (p > 0.0) && isfinite(p);
    const double inv = __drcp_rn(p);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int r = r0 + 2 * q;
      if (r == k)
        v[q] = (c == k) ? inv : v[q] * inv;
      else if (c == k)
        v[q] = -prk[q] * inv;
      else
        v[q] = v[q] - prk[q] * (pkc * inv);
    }
  }
  return ok;
}

void init_als_attributes();
// Upper triangle of U^T U (FP64) accumulated into gram; zero_first memsets it.
int launch_gram(tsr_ctx* ctx, cudaStream_t s, const float* U, int64_t rows, int R,
                double* gram, bool zero_first);
// ||X||^2 (FP64) added into *out (which the caller zeroes).
int launch_norm_sq(tsr_ctx* ctx, cudaStream_t s, const float* X, int64_t n, double* out);
// Hadamard of all Grams except `mode`, its inverse (ridge retry), and the
// zeroing of gram[mode] (and, when `last`, state->inner) before the solve.
// For mode 0 it first forms the fit of the previous sweep, when one is pending.
// l2 >= 0 is added to the Hadamard's diagonal before the inverse (the ridge of
// cp_als_constrained, core.rs:336-343); the stored Hadamard (used by the fit)
// stays unshifted.
// tik_order > 0 adds tik_lambda times the finite-difference penalty of
// apply_tikhonov_to_gram (helpers.rs:630-700) instead.
int launch_chol(tsr_ctx* ctx, cudaStream_t s, const AlsBuffers& b, int ndim, int mode, int R,
                float ridge_eps, bool last, double tol, double l2 = 0.0, int tik_order = 0,
                double tik_lambda = 0.0);
// orthonormalize_factor (helpers.rs:582-607) after this mode's solve: the
// factor U (rows x R, in place) becomes Q = U R^-1 with U^T U = R^T R
// (Cholesky in FP64 of the Gram the solve accumulated; Q's R has a positive
// diagonal), gram is recomputed as Q^T Q and, for the last mode, <M, Q> and
// ||Xhat||^2 are re-formed from the split partials. A Gram that is not
// positive definite (linearly dependent columns) stops the run with DS_NOT_SPD.
int launch_orthonormalize(tsr_ctx* ctx, cudaStream_t s, const AlsBuffers& b, int ndim, int mode,
                          int R, int64_t rows, float* U, double* gram, bool last,
                          const float* partials, int splits);
// Clamp n floats at zero (non-negative initial factors, core.rs:271-276).
int launch_clamp_nonneg(tsr_ctx* ctx, cudaStream_t s, float* U, int64_t n);
// Sets *flag to 1 if any of the n values is negative (helpers.rs:705-716).
int launch_any_negative(tsr_ctx* ctx, cudaStream_t s, const float* X, int64_t n, int* flag);
// The pending fit of the last sweep (fit, history, stopping rules).
int launch_fit(tsr_ctx* ctx, cudaStream_t s, const AlsBuffers& b, int ndim, int R, double tol);
// U_mode = (sum of split partials) . G^{-1} and its Gram U^T U added into
// `gram` (zeroed by this mode's launch_chol); `last` also accumulates <M, U>
// and marks the sweep's fit pending. Each new fp32 entry is soft-thresholded
// by l1 when l1 > 0 and clamped at zero when nonneg (core.rs:350-359) before
// it is stored and enters the Gram and the fit.
// With bimg set, each new entry's bf16 hi/lo halves are also written into that
// B image (mttkrp3.cu layout, n_pad img_n_pad) for the next MTTKRP.
int launch_solve(tsr_ctx* ctx, cudaStream_t s, const AlsBuffers& b, const float* partials,
                 int splits, int64_t rows, int R, float* U, double* gram, bool last, int ndim,
                 double tol, float l1 = 0.f, int nonneg = 0, uint8_t* bimg = nullptr,
                 int img_n_pad = 0);

}  // namespace tsr

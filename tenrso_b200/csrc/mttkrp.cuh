// Host-side entry points of the dense MTTKRP kernels (split-K partials).
#pragma once
#include "kr.cuh"

namespace tsr {

struct SplitPlan {
  int splits = 1;
  int64_t k_per_split = 0;
  int bn = 64;  // FP32 path: output columns per CTA tile (32 or 64)
  int run_length = 0;  // > 0 selects the run-scaled kernel (runs of this length), either path
};

void init_tc_attributes();
void init_simt_attributes();

// FP32 SIMT kernel (mttkrp_simt.cu).
// L > 0: the unfolding's columns come in runs of L (the fastest other mode);
// where the run-scaled kernel applies (L a multiple of 4, R <= 64, its
// shared-memory tile fits) the plan selects it (run_length = L) and
// k_per_split then counts 32-column steps over all runs.
SplitPlan plan_simt(const tsr_ctx* ctx, int64_t rows, int64_t K, int R, int64_t L = 0);
int launch_mttkrp_simt(tsr_ctx* ctx, const float* A, const Unfolding& u, const KRSpec& kr,
                       const SplitPlan& plan, float* partials);
int launch_mttkrp_reduce(tsr_ctx* ctx, const float* partials, int splits, int64_t n, float* out);
// Same for a rows x R result, each column r scaled by w[r] when w is given.
int launch_mttkrp_reduce_scaled(tsr_ctx* ctx, const float* partials, int splits, int64_t rows,
                                int R, const float* w, float* out);

// BF16x3 tcgen05 kernel (mttkrp_tc.cu). The unfolding halves hi/lo are bf16
// with row stride u.ld (a multiple of 8 elements, 16 bytes).
bool tc_supported(const Unfolding& u, int R);
SplitPlan plan_tc(const tsr_ctx* ctx, const Unfolding& u, int R);
// a_resident: hi / lo were written before the kernel that precedes this
// launch in the stream (see ModeOperand::resident).
int launch_mttkrp_tc(tsr_ctx* ctx, const __nv_bfloat16* hi, const __nv_bfloat16* lo,
                     const Unfolding& u, const KRSpec& kr, const SplitPlan& plan,
                     float* partials, bool a_resident = false);

// Single-layout BF16x3 MTTKRP of a 3-way tensor (mttkrp3.cu): X split once
// into bf16 hi/lo halves in its own row-major layout, read by every mode;
// the contracted factor comes as a prebuilt swizzled "B image".
struct Dense3 {
  int64_t I, J, K;
  int R, n_pad;  // n_pad: 32 (R <= 32) or 64
  const __nv_bfloat16* hi;
  const __nv_bfloat16* lo;
  uint8_t* bimg[3];  // [1]: image of U1 (L = J, mode 2), [2]: of U2 (L = K, modes 0 and 1)
};
void init_mttkrp3_attributes();
bool dense3_supported(int ndim, const int64_t* shape, int R);
int dense3_n_pad(int R);
size_t bimage_bytes(int64_t L, int n_pad);
int64_t dense3_rows(const Dense3& d, int mode);
// X (n floats, n % 4 == 0) -> hi / lo; ||X||^2 (FP64) added into *norm_sq.
int launch_split_bf16(tsr_ctx* ctx, cudaStream_t s, const float* X, int64_t n, __nv_bfloat16* hi,
                      __nv_bfloat16* lo, double* norm_sq);
// The whole B image of U (L x R), zero padding included.
// L_img > L: the image covers L_img rows, those from L on zero.
int launch_bimage(tsr_ctx* ctx, cudaStream_t s, const float* U, int64_t L, int R, int n_pad,
                  uint8_t* img, int64_t L_img = 0);
// SplitPlan: splits, k_per_split = runs per split, run_length = contracted length.
SplitPlan plan_mttkrp3(const tsr_ctx* ctx, const Dense3& d, int mode);
// Partials [splits][rows][R] of mode `mode`; the weights come from ft.
int launch_mttkrp3(tsr_ctx* ctx, cudaStream_t s, const Dense3& d, int mode, const FactorTable& ft,
                   const SplitPlan& plan, float* partials, bool a_resident);

// Two-sided contraction of X seen as an A x C matrix (its bf16 halves,
// row-major): T += X W (A x R) and P += X^T V (C x R) in one read of X, for
// R <= 32. W (C x R) and V (A x R) come as B images with n_pad 32 covering
// twosided_pad(C) and twosided_pad(A) rows. T and P are added into (fp32
// atomics): zero them first.
struct TwoSided {
  const __nv_bfloat16* hi;
  const __nv_bfloat16* lo;
  int64_t A, C;
  int R;
  const uint8_t* wimg;
  const uint8_t* vimg;
  float* T;
  float* P;
};
// B images (n_pad rows of hi halves, n_pad of lo halves per 64-row block) of
// Khatri-Rao products, built on the fly: row k of image w is the product of
// im[w].U[f][k_f, :] over the row-major multi-index (k_0, ..., k_{nf-1}) of k
// over the factors' row counts; rows from L on are zero. chunks = image
// bytes / 16 (bimage_bytes of the padded row count).
struct KRImage {
  int nf;
  const float* U[kMaxModes];
  int size[kMaxModes];
  int L;
  int chunks;
  uint8_t* img;
};
struct KRImages {
  KRImage im[2];
  int n;  // images in use (1 or 2)
  int R, n_pad;
  float* zero;      // also zero-filled by the launch: zero_n4 float4s (16-byte aligned)
  int64_t zero_n4;
};
// pdl: programmatic dependent launch (the kernel waits for its predecessor
// before writing, then lets its dependent start).
int launch_kr_images(tsr_ctx* ctx, cudaStream_t s, const KRImages& a, bool pdl = false);
bool twosided_supported(int64_t A, int64_t C, int R);
int64_t twosided_pad(int64_t L);
// Launched with programmatic dependent launch: the prologue overlaps the
// predecessor, whose writes are awaited before any operand is read.
int launch_twosided(tsr_ctx* ctx, cudaStream_t s, const TwoSided& a);

// Materialised two-factor Khatri-Rao product (the public khatri_rao API).
int launch_khatri_rao(tsr_ctx* ctx, const float* A, int64_t I, const float* B, int64_t J,
                      int64_t K, float* C);

// Partial buffer size in floats for a plan.
inline size_t partial_floats(const SplitPlan& p, int64_t rows, int R) {
  return (size_t)p.splits * rows * R;
}

}  // namespace tsr

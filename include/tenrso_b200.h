/*
 * tenrso_b200 — C ABI of a B200-native (sm_100a) CP-ALS hot path for tenrso.
 *
 * Every entry point replaces one tenrso function on the CP-ALS path and is
 * cited below by its file:line inside the tenrso repository. Plain pointers
 * and sizes only. Unless a name ends in `_dev`, tensor/factor/output pointers
 * are HOST memory and the call blocks until the result is on the host, as the
 * synchronous Rust functions do; `_dev` variants take device pointers and are
 * stream-ordered on the context's stream.
 *
 * Layouts: dense tensors are row-major (C order) unless a strides array is
 * given; factor matrices are row-major I_m x R; outputs are row-major.
 *
 * Errors: every function returns a tsr_status. tsr_last_error() returns the
 * message of the calling thread's last failure, worded as tenrso words it
 * (e.g. "Mode 5 out of bounds for tensor with rank 2"), so a Rust shim can
 * re-raise it through anyhow::bail! unchanged.
 */
#ifndef TENRSO_B200_H
#define TENRSO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tsr_status {
  TSR_OK = 0,
  TSR_E_MODE_OOB = 1,        /* mttkrp.rs:87-93 "Mode {} out of bounds ..." */
  TSR_E_NFACTORS = 2,        /* mttkrp.rs:95-101 "Number of factor matrices ..." */
  TSR_E_RANK_MISMATCH = 3,   /* mttkrp.rs:106-112 "Factor matrix {} has {} columns ..." */
  TSR_E_ROWS_MISMATCH = 4,   /* mttkrp.rs:113-121 "Factor matrix {} has {} rows ..." */
  TSR_E_INVALID_RANK = 5,    /* cp/types.rs:15 CpError::InvalidRank */
  TSR_E_INVALID_TOL = 6,     /* cp/types.rs:18 CpError::InvalidTolerance */
  TSR_E_NOT_SPD = 7,         /* cp/types.rs:21 CpError::LinalgError */
  TSR_E_TIMEOUT = 8,         /* a bounded device-side wait gave up */
  TSR_E_CUDA = 9,            /* CUDA runtime/driver failure */
  TSR_E_INVALID_ARG = 10,    /* null pointer, bad size, unsupported layout */
  TSR_E_NEED_2_FACTORS = 11, /* mttkrp.rs:196-198 "Need at least 2 factor matrices for MTTKRP" */
  TSR_E_TILE_SIZE = 12,      /* mttkrp.rs:402-404 "Tile size must be greater than 0" */
  TSR_E_MODE_ORDER = 13,     /* csf.rs:143-156 CsfError::InvalidModeOrder */
  TSR_E_UNSUPPORTED = 14,    /* shape/rank outside what the kernels implement */
  TSR_E_COLS_MISMATCH = 15,  /* khatri_rao.rs:63-67 "Number of columns must match" */
  TSR_E_SHAPE = 16,          /* cp/types.rs:24 CpError::ShapeMismatch / coo.rs errors */
  TSR_E_INDEX_OOB = 17,      /* coo.rs:130-137 CooError::IndexOutOfBounds */
  TSR_E_NONNEG_VIOLATION = 18, /* cp/types.rs:30-31 CpError::NonnegativeViolation */
  TSR_E_INVALID_REGULARIZATION = 19, /* cp/types.rs:33-34 CpError::InvalidRegularization */
  TSR_E_BLOCK_SHAPE = 20     /* hicoo.rs:43-44 HiCooError::InvalidBlockShape */
} tsr_status;

/* Arithmetic of the dense MTTKRP. FP32: IEEE fp32 FMA on the SIMT pipes.
 * BF16X3: operands split as x = hi + lo (both bf16), three tcgen05 bf16 MMAs
 * (hi*hi + hi*lo + lo*hi) with fp32 accumulation in tensor memory. */
typedef enum tsr_precision { TSR_PREC_FP32 = 0, TSR_PREC_BF16X3 = 1 } tsr_precision;

/* cp/types.rs:319-328 ConvergenceReason */
/* InitStrategy (crates/tenrso-decomp/src/cp/types.rs:39-59). */
typedef enum tsr_init_strategy {
  TSR_INIT_RANDOM = 0,
  TSR_INIT_RANDOM_NORMAL = 1,
  TSR_INIT_SVD = 2,
  TSR_INIT_NNSVD = 3,
  TSR_INIT_LEVERAGE_SCORE = 4
} tsr_init_strategy;

typedef enum tsr_reason {
  TSR_REASON_MAX_ITERATIONS = 0,
  TSR_REASON_FIT_TOLERANCE = 1,
  TSR_REASON_OSCILLATION = 2,
  TSR_REASON_TIME_LIMIT = 3
} tsr_reason;

/* cp/types.rs:329-344 ConvergenceInfo + CpDecomp::{fit, iters} (types.rs:350-368).
 * fit_history is caller-owned with room for max_iters values (may be NULL). */
typedef struct tsr_cp_info {
  double fit;
  int32_t iters;
  int32_t reason; /* tsr_reason */
  int32_t oscillated;
  int32_t oscillation_count;
  double final_fit_change;
  double* fit_history;
  int32_t ridge_used; /* 1: the eps*rank*10 ridge of cp/helpers.rs:477-490 engaged;
                         2: that ridge scaled by the Gram's mean diagonal was needed */
  int32_t reserved;
} tsr_cp_info;

typedef struct tsr_ctx tsr_ctx;

/* ---- context ----------------------------------------------------------- */
const char* tsr_last_error(void);
const char* tsr_status_string(int status);
const char* tsr_version(void);
/* stream may be NULL (the context creates its own) or a cudaStream_t. */
int tsr_ctx_create(int device, void* stream, tsr_ctx** out);
int tsr_ctx_destroy(tsr_ctx* ctx);
int tsr_ctx_synchronize(tsr_ctx* ctx);
/* Kernels launched through this context since creation (a counter). */
int64_t tsr_ctx_launch_count(const tsr_ctx* ctx);
/* Clock-cycle budget of each bounded pipeline wait in the tensor-core MTTKRP
 * kernels (cycles <= 0 restores the default, about one second). A wait that
 * runs out makes the kernel drain its copies, free its tensor memory and
 * return; the call then fails with TSR_E_TIMEOUT and the context stays usable.
 * No tenrso counterpart (failure-path testing aid). */
int tsr_ctx_set_wait_budget(tsr_ctx* ctx, int64_t cycles);
/* Kernel timeline tracing of the CP-ALS sweep (measurement aid, no tenrso
 * counterpart). capacity > 0 allocates that many slots and turns tracing on
 * (0 turns it off); while on, every dense cp_als call is captured afresh and
 * each of its MTTKRP, inverse and solve launches records the first CTA entry
 * and the last CTA exit (%globaltimer, ns). tsr_ctx_read_trace copies up to
 * `capacity` records of the last call: start/end ns, kind (0 MTTKRP,
 * 1 inverse, 2 solve) and mode, and the number written into *count. */
int tsr_ctx_set_trace(tsr_ctx* ctx, int capacity);
int tsr_ctx_read_trace(tsr_ctx* ctx, int capacity, int64_t* start_ns, int64_t* end_ns,
                       int* kind, int* mode, int* count);

/* ---- Khatri-Rao: crates/tenrso-kernels/src/khatri_rao.rs:56-89 ----------
 * out (I*J x K) with row a*J + b = A[a,:] * B[b,:]. Host pointers. */
int tsr_khatri_rao_f32(tsr_ctx* ctx, const float* a, int64_t a_rows, int64_t a_cols,
                       const float* b, int64_t b_rows, int64_t b_cols, float* out);

/* ---- dense MTTKRP: crates/tenrso-kernels/src/mttkrp.rs:74-146 -----------
 * tensor: ndim dims, shape[ndim]; strides[ndim] in elements (NULL = row-major).
 * factors[m]: factor_rows[m] x factor_cols[m] row-major (ndim_factors of them).
 * out: shape[mode] x R row-major. Validation order and messages follow
 * mttkrp.rs:86-122. */
int tsr_mttkrp_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                   const int64_t* strides, const float* const* factors, int n_factors,
                   const int64_t* factor_rows, const int64_t* factor_cols, int mode,
                   int precision, float* out);
/* mttkrp_blocked / mttkrp_blocked_parallel (mttkrp.rs:395-498, 529-609): the
 * tile size only regroups the sum; validated (> 0) then the same kernel runs. */
int tsr_mttkrp_blocked_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                           const int64_t* strides, const float* const* factors, int n_factors,
                           const int64_t* factor_rows, const int64_t* factor_cols, int mode,
                           int64_t tile_size, int precision, float* out);
/* mttkrp_all_modes (crates/tenrso-kernels/src/utils.rs:282-307): out[m] gets
 * shape[m] x R for every mode m, the tensor is uploaded once. */
int tsr_mttkrp_all_modes_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                             const float* const* factors, int64_t rank, int precision,
                             float* const* out);
/* Device-resident MTTKRP: d_tensor row-major contiguous on the device,
 * d_factors[m] device pointers (row-major shape[m] x rank), d_out device. */
int tsr_mttkrp_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim, const int64_t* shape,
                       const float* const* d_factors, int64_t rank, int mode, int precision,
                       float* d_out);

/* Kernel-only timing of the dense MTTKRP (the roofline figure): the unfolding
 * is prepared once, then `iters` launches of the MTTKRP kernel are timed with
 * CUDA events on the context's stream, optionally writing a buffer larger
 * than L2 between launches. No tenrso counterpart (measurement aid). */
int tsr_profile_mttkrp_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim,
                               const int64_t* shape, const float* const* d_factors, int64_t rank,
                               int mode, int precision, int iters, int flush_l2,
                               double* ms_per_launch, int64_t* splits_out);

/* The FP64 inverse the CP-ALS solve applies (the step that replaces the
 * per-row scirs2_linalg::lstsq of solve_least_squares, cp/helpers.rs:455-495,
 * with the same ridge retry): `gram` (rank x rank, row-major, symmetric, host)
 * is inverted `iters` times by the sweep's inverse kernel, the result copied
 * to `inverse` (host), *ridge_used set to 0 (none), 1 (eps*rank*10) or 2
 * (scaled by the mean diagonal), and *ms_per_launch to the mean device time
 * of one launch (CUDA events, warm). TSR_E_NOT_SPD when every ridge fails.
 * No tenrso counterpart (test and measurement aid). */
int tsr_gram_inverse_f64(tsr_ctx* ctx, const double* gram, int64_t rank, int iters,
                         double* inverse, int* ridge_used, double* ms_per_launch);

/* Allocation-free MTTKRP of mode 0 (FP32 split-K path). No tenrso
 * counterpart: it exists for callers that cannot call cudaMalloc, such as a
 * library whose host application's caching allocator owns all device memory,
 * or a service that sizes every device buffer before it starts. It takes a
 * stream instead of a tsr_ctx and keeps its split partials in a fixed 16 MiB
 * device array that every GPU loading the library holds until exit; it calls
 * no cudaMalloc/cudaFree. Device pointers, row-major layouts as
 * tsr_mttkrp_dev_f32; needs prod(shape[1:]) % 4 == 0 and a 16-byte aligned
 * tensor, and rejects with TSR_E_UNSUPPORTED any problem whose split partials
 * (shape[0] x rank x the kernel's split count) exceed the array's 4 Mi
 * floats. The stream must belong to the current device (TSR_E_INVALID_ARG
 * otherwise); negative sizes are rejected, and an empty tensor gives a zero
 * output. The first call on a device resolves the array's device address
 * (cudaGetSymbolAddress) and sets the kernels' attributes. All calls share
 * the array, so calls that overlap on the GPU race and must be serialised by
 * the caller. */
int tsr_mttkrp_mode0_noalloc_f32(void* stream, const float* d_tensor, int ndim,
                                 const int64_t* shape, const float* const* d_factors,
                                 int64_t rank, float* d_out);

/* ---- CP-ALS: crates/tenrso-decomp/src/cp/core.rs:59-182 -----------------
 * Same loop, validation (rank in [1, min I_n], tol in [0,1)), fit, oscillation
 * and convergence rules. init_factors: concatenated row-major I_0xR, I_1xR, ...
 * (the injected initialisation tenrso cannot seed); NULL = U(0,1) from the
 * library's SplitMix64 stream `seed` (InitStrategy::Random, helpers.rs:215-222).
 * time_limit_s < 0 means None. out_factors: concatenated like init_factors. */
int tsr_cp_als_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                   int64_t rank, int max_iters, double tol, const float* init_factors,
                   uint64_t seed, int precision, double time_limit_s, float* out_factors,
                   tsr_cp_info* info);
/* Device-resident CP-ALS: d_tensor (row-major), d_init and d_out_factors are
 * device pointers (concatenated factors); info stays on the host. */
int tsr_cp_als_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim, const int64_t* shape,
                       int64_t rank, int max_iters, double tol, const float* d_init,
                       int precision, double time_limit_s, float* d_out_factors,
                       tsr_cp_info* info);

/* The f64 instantiation of the drop-in: mttkrp<f64> (mttkrp.rs:74-146) and
 * cp_als<f64> (cp/core.rs:59-182) with FP64 tensor, factors, MTTKRP, Gram,
 * solve and fit (host buffers; the tensor row-major). Arguments, validation
 * and messages as tsr_mttkrp_f32 / tsr_cp_als_f32; init_factors NULL draws
 * InitStrategy::Random from the library's seeded stream `seed` in FP64. */
int tsr_mttkrp_f64(tsr_ctx* ctx, const double* tensor, int ndim, const int64_t* shape,
                   const double* const* factors, int n_factors, const int64_t* factor_rows,
                   const int64_t* factor_cols, int mode, double* out);
int tsr_cp_als_f64(tsr_ctx* ctx, const double* tensor, int ndim, const int64_t* shape,
                   int64_t rank, int max_iters, double tol, const double* init_factors,
                   uint64_t seed, double time_limit_s, double* out_factors, tsr_cp_info* info);

/* Constraints of cp_als_constrained (crates/tenrso-decomp/src/cp/types.rs:199-225,
 * core.rs:225-400) in the form the sweep applies them:
 *   l2  effective_l2() (types.rs:298-303): added to the diagonal of the Gram
 *       Hadamard before the solve (core.rs:336-343);
 *   l1  effective_l1() (types.rs:306-308): soft threshold of each new factor
 *       entry after the solve (core.rs:350-353, helpers.rs:610-623);
 *   nonnegative: initial factors and every new factor clamped at zero
 *       (core.rs:271-276, 356-359);
 *   validate_nonneg_input: with nonnegative, a tensor holding a negative
 *       entry is rejected with TSR_E_NONNEG_VIOLATION (core.rs:265-267,
 *       helpers.rs:705-716).
 *   orthogonal: each new factor (after the threshold and the projection)
 *       replaced by the Q of its QR factorization (core.rs:361-364,
 *       helpers.rs:582-607), taken with a positive diagonal in R (Cholesky of
 *       U^T U in FP64); linearly dependent columns give TSR_E_NOT_SPD;
 *   tikhonov_order > 0: tikhonov_lambda times apply_tikhonov_to_gram's
 *       finite-difference penalty added to the Gram instead of l2
 *       (core.rs:327-344).
 * l2, l1 or tikhonov_lambda negative or not finite gives
 * TSR_E_INVALID_REGULARIZATION. */
typedef struct tsr_cp_constraints {
  double l2;
  double l1;
  int nonnegative;
  int validate_nonneg_input;
  int orthogonal;         /* QR-orthonormalize each updated factor (core.rs:361-364) */
  int tikhonov_order;     /* > 0: RegularizationType::Tikhonov{lambda, order}'s */
  double tikhonov_lambda; /*   finite-difference penalty (helpers.rs:630-700) */
} tsr_cp_constraints;

/* cp_als_constrained (core.rs:225-400) on the dense path; arguments as
 * tsr_cp_als_f32, plus the constraints (NULL = none, i.e. cp_als). */
int tsr_cp_als_constrained_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                               int64_t rank, int max_iters, double tol,
                               const float* init_factors, uint64_t seed,
                               const tsr_cp_constraints* constraints, int precision,
                               double time_limit_s, float* out_factors, tsr_cp_info* info);
/* Device-resident form; arguments as tsr_cp_als_dev_f32 plus the constraints. */
int tsr_cp_als_constrained_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim,
                                   const int64_t* shape, int64_t rank, int max_iters,
                                   double tol, const float* d_init,
                                   const tsr_cp_constraints* constraints, int precision,
                                   double time_limit_s, float* d_out_factors,
                                   tsr_cp_info* info);

/* cp_als_accelerated (crates/tenrso-decomp/src/cp/advanced.rs:51-213): the
 * CP-ALS sweep with the line search of line_search_cp (cp/helpers.rs:130-189)
 * and the adaptive extrapolation from the second iteration on. Arguments as
 * tsr_cp_als_f32; tol must lie in (0, 1) (TSR_E_INVALID_TOL otherwise), rank 0
 * is TSR_E_INVALID_RANK. The result has no weights; info->ridge_used reports
 * the solve's ridge retry. */
int tsr_cp_als_accelerated_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                               int64_t rank, int max_iters, double tol,
                               const float* init_factors, uint64_t seed, int precision,
                               double time_limit_s, float* out_factors, tsr_cp_info* info);
/* Device-resident form; arguments as tsr_cp_als_dev_f32. */
int tsr_cp_als_accelerated_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim,
                                   const int64_t* shape, int64_t rank, int max_iters, double tol,
                                   const float* d_init, int precision, double time_limit_s,
                                   float* d_out_factors, tsr_cp_info* info);

/* One ALS factor update on device data, the building block of a sharded
 * sweep: U = M G^-1 for the rows x rank fp32 MTTKRP rows d_M and the FP64
 * R x R Hadamard d_hadamard (solve_least_squares, cp/helpers.rs:455-495, with
 * its eps*rank*10 ridge retry), the full FP64 Gram U^T U of the new rows into
 * d_gram and <M, U> (FP64) into *inner_out. rows may be 0 (d_gram = 0). */
int tsr_als_solve_dev_f32(tsr_ctx* ctx, const float* d_M, int64_t rows, int64_t rank,
                          const double* d_hadamard, float* d_U, double* d_gram,
                          double* inner_out, int* ridge_used);

/* initialize_factors (crates/tenrso-decomp/src/cp/helpers.rs:192-377) for
 * every InitStrategy: out_factors receives the concatenated I_n x rank fp32
 * factors. Random and RandomNormal draw from the library's seeded stream
 * `seed` (tenrso's thread_rng cannot be seeded); Svd, Nnsvd and
 * LeverageScore take the leading singular vectors of each unfolding (FP64 on
 * the device, mode sizes up to 1024, each u_r oriented so that its
 * largest-magnitude entry is positive) and pad columns past the unfolding's
 * rank with N(0, 0.01) draws from the same seeded stream. The factors feed
 * tsr_cp_als_f32 (and its variants) as init_factors. */
int tsr_cp_init_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                    int64_t rank, int strategy, uint64_t seed, float* out_factors);
int tsr_cp_init_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim, const int64_t* shape,
                        int64_t rank, int strategy, uint64_t seed, float* d_out_factors);

/* ---- sparse: crates/tenrso-sparse --------------------------------------
 * COO entries are `indices` (nnz x ndim, row-major int64) and `values`
 * (nnz float32). Validation follows CooTensor::new (coo.rs:101-149). */
typedef struct tsr_sparse tsr_sparse;

/* CooTensor::sort (coo.rs:239-257): stable lexicographic sort, in place. */
int tsr_coo_sort_f32(tsr_ctx* ctx, int64_t* indices, float* values, int64_t nnz, int ndim,
                     const int64_t* shape);
/* CooTensor::deduplicate (coo.rs:320-347): sort, then sum equal coordinates
 * left to right in fp32 (insertion order); rewrites the first *nnz_out entries. */
int tsr_coo_deduplicate_f32(tsr_ctx* ctx, int64_t* indices, float* values, int64_t nnz, int ndim,
                            const int64_t* shape, int64_t* nnz_out);
/* CsfTensor::from_coo (csf.rs:137-264), bit-exact arrays: fptr is
 * ndim x (nnz+1) and fids ndim x max(nnz,1) (row l = level l); lens[2l] and
 * lens[2l+1] receive len(fptr[l]) and len(fids[l]); vals_out gets nnz values
 * (none for ndim == 1, as the reference). Every fptr level holds nnz offsets. */
int tsr_csf_from_coo_f32(tsr_ctx* ctx, const int64_t* indices, const float* values, int64_t nnz,
                         int ndim, const int64_t* shape, const int64_t* mode_order,
                         int n_mode_order, int64_t* fptr, int64_t* fids, float* vals_out,
                         int64_t* lens);
/* Device-resident sparse tensor: one CSF per root mode, mode_order = [n, the
 * other modes in ascending size]. Duplicates are kept (as from_coo). */
int tsr_sparse_create_f32(tsr_ctx* ctx, const int64_t* indices, const float* values, int64_t nnz,
                          int ndim, const int64_t* shape, tsr_sparse** out);
/* Same from device COO arrays (indices validated on the device). */
int tsr_sparse_create_dev_f32(tsr_ctx* ctx, const int64_t* d_indices, const float* d_values,
                              int64_t nnz, int ndim, const int64_t* shape, tsr_sparse** out);
/* CooTensor::deduplicate on device arrays (in place, first *nnz_out entries). */
int tsr_coo_deduplicate_dev_f32(tsr_ctx* ctx, int64_t* d_indices, float* d_values, int64_t nnz,
                                int ndim, const int64_t* shape, int64_t* nnz_out);
/* Seeded synthetic input (no tenrso counterpart): `nnz` distinct coordinates
 * of per-mode Zipf(s_exp) indices over seeded permutations, as a raw COO in
 * draw order (duplicates included) written to d_indices/d_values (room for
 * `capacity` entries); *n_raw_out receives the raw entry count. Identical to
 * tenrso_b200.synth.zipf_coo. */
int tsr_synth_zipf_coo_dev(tsr_ctx* ctx, int ndim, const int64_t* shape, int64_t nnz,
                           uint64_t seed, double s_exp, int64_t capacity, int64_t* d_indices,
                           float* d_values, int64_t* n_raw_out);
int tsr_sparse_destroy(tsr_sparse* sp);
int tsr_sparse_info(const tsr_sparse* sp, int mode, int64_t* nnz, int64_t* n_roots,
                    int64_t* n_fibers);
/* Sparse MTTKRP (no tenrso implementation; csf.rs:42 names it): the dense
 * mttkrp math (mttkrp.rs:851-875) over the nonzeros. out: shape[mode] x rank. */
int tsr_mttkrp_csf_f32(tsr_ctx* ctx, const tsr_sparse* sp, const float* const* factors,
                       int64_t rank, int mode, float* out);
int tsr_mttkrp_csf_dev_f32(tsr_ctx* ctx, const tsr_sparse* sp, const float* const* d_factors,
                           int64_t rank, int mode, float* d_out);
/* Kernel timing of the CSF MTTKRP (measurement aid, no tenrso counterpart). */
int tsr_profile_mttkrp_csf_dev_f32(tsr_ctx* ctx, const tsr_sparse* sp,
                                   const float* const* d_factors, int64_t rank, int mode,
                                   int iters, int flush_l2, double* ms_per_launch);
/* Sparse CP-ALS (tenrso has none): cp_als's loop (cp/core.rs:59-182) with the
 * CSF MTTKRP; FP32 factors, FP64 Gram/solve/fit. */
int tsr_cp_als_sparse_f32(tsr_ctx* ctx, const tsr_sparse* sp, int64_t rank, int max_iters,
                          double tol, const float* init_factors, uint64_t seed,
                          double time_limit_s, float* out_factors, tsr_cp_info* info);
int tsr_cp_als_sparse_dev_f32(tsr_ctx* ctx, const tsr_sparse* sp, int64_t rank, int max_iters,
                              double tol, const float* d_init, double time_limit_s,
                              float* d_out_factors, tsr_cp_info* info);

/* ---- HiCOO: crates/tenrso-sparse/src/hicoo.rs ---------------------------
 * HiCooTensor::from_coo (hicoo.rs:118-203): entries split into block
 * coordinates i / b and local coordinates i % b, stably sorted by block
 * coordinate; nothing merged. Block sides up to 256 (u8 local coordinates on
 * the device; larger sides give TSR_E_UNSUPPORTED). Errors: a block_shape
 * whose length differs from ndim or that holds a zero is TSR_E_BLOCK_SHAPE
 * with hicoo.rs's messages; shape and index checks as CooTensor::new. */
typedef struct tsr_hicoo tsr_hicoo;
int tsr_hicoo_create_f32(tsr_ctx* ctx, const int64_t* indices, const float* values, int64_t nnz,
                         int ndim, const int64_t* shape, const int64_t* block_shape,
                         int n_block_shape, tsr_hicoo** out);
int tsr_hicoo_destroy(tsr_hicoo* h);
/* nnz() and num_blocks() (hicoo.rs:229-238). */
int tsr_hicoo_info(const tsr_hicoo* h, int64_t* nnz, int64_t* num_blocks);
/* block_coords (num_blocks x ndim), block_ptrs (num_blocks + 1), local_coords
 * (nnz x ndim) and values (hicoo.rs:249-271) copied to host arrays; any may
 * be NULL. */
int tsr_hicoo_export(tsr_ctx* ctx, const tsr_hicoo* h, int64_t* block_coords,
                     int64_t* block_ptrs, int64_t* local_coords, float* values);
/* Sparse MTTKRP on the HiCOO layout (no tenrso implementation; hicoo.rs:30-34
 * names it): out (shape[mode] x rank) = sum over entries of
 * v * prod_{m != mode} U_m[i_m, :]. Factors are host arrays (I_m x rank). */
int tsr_mttkrp_hicoo_f32(tsr_ctx* ctx, const tsr_hicoo* h, const float* const* factors,
                         int64_t rank, int mode, float* out);
int tsr_mttkrp_hicoo_dev_f32(tsr_ctx* ctx, const tsr_hicoo* h, const float* const* d_factors,
                             int64_t rank, int mode, float* d_out);

/* ---- n-mode products: crates/tenrso-kernels/src/nmode.rs ----------------
 * nmode_product (nmode.rs:72-131): out = tensor x_mode matrix, matrix rows x
 * cols (row-major) with cols == shape[mode]; out has shape[mode] replaced by
 * rows. Errors: "Mode {} out of bounds for tensor with rank {}"
 * (TSR_E_MODE_OOB), "Matrix columns ({}) must match tensor mode-{} size ({})"
 * (TSR_E_COLS_MISMATCH). fp32 in, fp32 accumulate (the reference sums in T). */
int tsr_nmode_product_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                          const float* matrix, int64_t rows, int64_t cols, int mode, float* out);
int tsr_nmode_product_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim, const int64_t* shape,
                              const float* d_matrix, int64_t rows, int64_t cols, int mode,
                              float* d_out);
/* nmode_products_seq (nmode.rs:241-254) / tucker_operator_ordered
 * (nmode.rs:517-531): products in the given order; cols[t] equals that
 * mode's size at step t. out_shape gets the result's shape; out may be NULL
 * to ask for the shape only. */
int tsr_nmode_products_seq_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                               int n, const int* modes, const float* const* mats,
                               const int64_t* rows, const int64_t* cols, float* out,
                               int64_t* out_shape);
/* tucker_operator (nmode.rs:442-480): a mode -> matrix map applied in
 * ascending order of rows / mode size (ties by mode index). */
int tsr_tucker_operator_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                            int n, const int* modes, const float* const* mats,
                            const int64_t* rows, const int64_t* cols, float* out,
                            int64_t* out_shape);
/* tucker_reconstruct (nmode.rs:576-611): core x_0 U_0 ... x_{N-1} U_{N-1};
 * "Number of factor matrices ({}) must match core rank ({})" (TSR_E_NFACTORS),
 * "Factor matrix {} has {} columns, expected {} (core mode-{} size)"
 * (TSR_E_RANK_MISMATCH). */
int tsr_tucker_reconstruct_f32(tsr_ctx* ctx, const float* core, int ndim,
                               const int64_t* core_shape, int n_factors,
                               const float* const* factors, const int64_t* rows,
                               const int64_t* cols, float* out, int64_t* out_shape);

/* ---- CP reconstruction and its adjoint ----------------------------------
 * tenrso_kernels::cp_reconstruct (crates/tenrso-kernels/src/outer.rs:223-274):
 * out (row-major, prod of factor_rows) = sum_r w_r U_0[:,r] o ... o U_{N-1}[:,r].
 * weights may be NULL (all ones). Errors as outer.rs:231-255. */
int tsr_cp_reconstruct_f32(tsr_ctx* ctx, const float* const* factors, int n_factors,
                           const int64_t* factor_rows, const int64_t* factor_cols,
                           const float* weights, int64_t n_weights, float* out);
int tsr_cp_reconstruct_dev_f32(tsr_ctx* ctx, const float* const* d_factors, int ndim,
                               const int64_t* shape, int64_t rank, const float* d_weights,
                               float* d_out);
/* Forward of the reconstruction loss (no tenrso counterpart): d_out = alpha *
 * (Xhat - X) (alpha = 2 gives dL/dXhat of ||X - Xhat||^2) and, when sq_err is
 * not NULL, *sq_err = sum (Xhat - X)^2 in FP64 (the call then synchronizes).
 * d_out may alias d_tensor. */
int tsr_cp_residual_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim, const int64_t* shape,
                            const float* const* d_factors, int64_t rank, const float* d_weights,
                            float alpha, float* d_out, double* sq_err);
/* CpReconstructionGrad::compute_factor_gradients (crates/tenrso-ad/src/grad.rs:81-120),
 * the VjpOp rule of the reconstruction: out_grads[n] (shape[n] x rank) =
 * unfold(G, n) . KR_{m != n}(U_m) . diag(weights), computed as an MTTKRP of G
 * whose Khatri-Rao rows are never stored. Errors as grad.rs:84-91, 137-139. */
int tsr_cp_reconstruction_grad_f32(tsr_ctx* ctx, const float* grad_output, int grad_ndim,
                                   const int64_t* shape, const float* const* factors,
                                   int n_factors, const int64_t* factor_rows,
                                   const int64_t* factor_cols, const float* weights,
                                   int64_t n_weights, int precision, float* const* out_grads);
int tsr_cp_reconstruction_grad_dev_f32(tsr_ctx* ctx, const float* d_grad_output, int ndim,
                                       const int64_t* shape, const float* const* d_factors,
                                       int64_t rank, const float* d_weights, int precision,
                                       float* const* d_out_grads);
/* A device tensor prepared for repeated MTTKRPs (no tenrso counterpart): its
 * per-mode unfoldings in `precision` are built once and owned by the object;
 * d_tensor stays the caller's and must not change while the object lives. */
typedef struct tsr_dense tsr_dense;
int tsr_dense_create_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim, const int64_t* shape,
                             int precision, tsr_dense** out);
int tsr_dense_destroy(tsr_dense* X);
/* Loss ||X - [[U]]||^2 + reg * sum_n ||U_n||_F^2 and every dL/dU_n (no tenrso
 * counterpart; the gradient equals grad.rs's rule applied to G = 2(Xhat - X)
 * plus 2 reg U_n), evaluated through Gram identities without forming Xhat:
 * one MTTKRP of X per mode plus FP64 R x R work (three or more modes, rank
 * <= 32: BF16x3 one two-sided contraction reading X once, FP32 two
 * MTTKRPs, of X and of its transpose made when the tensor is prepared;
 * BF16x3 rank <= 64: three single-layout passes). d_grads[n]: shape[n] x rank.
 * loss may be NULL: no synchronization, and a device wait that ran out
 * (TSR_E_TIMEOUT) is reported by the context's next synchronizing call;
 * otherwise the call synchronizes and reports it. */
int tsr_cp_loss_grad_dev_f32(tsr_ctx* ctx, const tsr_dense* X, const float* const* d_factors,
                             int64_t rank, double reg, float* const* d_grads, double* loss);

/* ---- batched CP-ALS (no tenrso counterpart; each instance is cp_als,
 * crates/tenrso-decomp/src/cp/core.rs:59-182, from injected factors) -------
 * A device-resident batch of n_inst dense 3-way tensors: shapes is n_inst x 3,
 * ranks n_inst (1 <= rank <= min(shape), rank <= 16), tensors[b] a host
 * row-major fp32 tensor. Factors of the whole batch are one packed array:
 * instance b at offsets[b] (tsr_batch_factor_layout) holds A | B | C, each
 * row-major with row stride rank. All instances run in one persistent
 * launch per run (a CUDA graph captured on first use and replayed). */
typedef struct tsr_batch tsr_batch;
int tsr_batch_create_f32(tsr_ctx* ctx, int n_inst, const int64_t* shapes, const int64_t* ranks,
                         const float* const* tensors, tsr_batch** out);
int tsr_batch_destroy(tsr_batch* batch);
int tsr_batch_factor_layout(const tsr_batch* batch, int64_t* total_floats, int64_t* offsets);
/* Launch configuration: threads per instance CTA (128, 256 or 512), sweeps
 * per launch (0 = all iterations in one launch), resident CTAs per SM (1-4).
 * tsr_batch_autotune chooses it by timing; set/get override or read it. */
int tsr_batch_set_config(tsr_batch* batch, int threads, int sweeps_per_launch, int ctas_per_sm);
int tsr_batch_get_config(const tsr_batch* batch, int* threads, int* sweeps_per_launch,
                         int* ctas_per_sm);
/* Times the candidate configurations on this batch (max_iters sweeps each,
 * from d_init) and keeps the fastest; the result is cached in the JSON file
 * cache_path (NULL = no cache) under the device name and the batch's shape
 * signature, and read back from there on later calls. */
int tsr_batch_autotune(tsr_ctx* ctx, tsr_batch* batch, int max_iters, const float* d_init,
                       const char* cache_path, int* from_cache);
/* cp_als on every instance: max_iters, tol as cp_als; init = packed initial
 * factors (host; NULL = U(0,1) from the seeded stream seed + instance);
 * out = packed factors (host); infos = n_inst results (fit_history pointers
 * may be NULL). */
int tsr_cp_als_batched_f32(tsr_ctx* ctx, tsr_batch* batch, int max_iters, double tol,
                           const float* init, uint64_t seed, float* out, tsr_cp_info* infos);
/* Device-resident form: d_init / d_out packed device arrays (may alias);
 * infos may be NULL (then the call does not synchronize). */
int tsr_cp_als_batched_dev_f32(tsr_ctx* ctx, tsr_batch* batch, int max_iters, double tol,
                               const float* d_init, float* d_out, tsr_cp_info* infos);

#ifdef __cplusplus
}
#endif

#endif /* TENRSO_B200_H */

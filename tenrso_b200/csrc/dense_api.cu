// Host mirror of tenrso's dense CP-ALS entry points over the C ABI:
//   tenrso_kernels::khatri_rao       khatri_rao.rs:56-89
//   tenrso_kernels::mttkrp (+blocked, all_modes)  mttkrp.rs:74-146, 395-498; utils.rs:282-307
//   tenrso_decomp::cp_als            cp/core.rs:59-182
// Validation order and messages follow the cited lines so that a Rust shim can
// surface them through anyhow / CpError unchanged.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>

#include "als.cuh"
#include "csf.cuh"
#include "dense.cuh"

namespace tsr {


// mttkrp.rs:86-122 then the KR helper's bail (mttkrp.rs:196-198).
int validate_mttkrp(int ndim, const int64_t* shape, int n_factors, const int64_t* frows,
                    const int64_t* fcols, int mode) {
  if (mode < 0 || mode >= ndim)
    return fail(TSR_E_MODE_OOB, "Mode %d out of bounds for tensor with rank %d", mode, ndim);
  if (n_factors != ndim)
    return fail(TSR_E_NFACTORS, "Number of factor matrices (%d) must match tensor rank (%d)",
                n_factors, ndim);
  int64_t R = fcols[0];
  for (int i = 0; i < ndim; ++i) {
    if (fcols[i] != R)
      return fail(TSR_E_RANK_MISMATCH, "Factor matrix %d has %lld columns, expected %lld", i,
                  (long long)fcols[i], (long long)R);
    if (frows[i] != shape[i])
      return fail(TSR_E_ROWS_MISMATCH,
                  "Factor matrix %d has %lld rows, expected %lld (tensor mode-%d size)", i,
                  (long long)frows[i], (long long)shape[i], i);
  }
  if (ndim < 2) return fail(TSR_E_NEED_2_FACTORS, "Need at least 2 factor matrices for MTTKRP");
  if (ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d exceeds the supported %d", ndim, kMaxModes);
  return TSR_OK;
}

int check_sizes(int ndim, const int64_t* shape, int64_t rank) {
  for (int d = 0; d < ndim; ++d)
    if (shape[d] < 0)
      return fail(TSR_E_INVALID_ARG, "mode %d has a negative size (%lld)", d, (long long)shape[d]);
  if (rank < 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  return TSR_OK;
}

int64_t numel(int ndim, const int64_t* shape) {
  int64_t n = 1;
  for (int d = 0; d < ndim; ++d) n *= shape[d];
  return n;
}

static bool is_row_major(int ndim, const int64_t* shape, const int64_t* strides) {
  if (!strides) return true;
  int64_t s = 1;
  for (int d = ndim - 1; d >= 0; --d) {
    if (shape[d] != 1 && strides[d] != s) return false;
    s *= shape[d];
  }
  return true;
}

// ndarray's as_standard_layout (mttkrp.rs:172-173): pack a strided host view.
static void pack_host(const float* src, int ndim, const int64_t* shape, const int64_t* strides,
               float* dst) {
  int64_t n = numel(ndim, shape);
  std::vector<int64_t> idx(ndim, 0);
  for (int64_t k = 0; k < n; ++k) {
    int64_t off = 0;
    for (int d = 0; d < ndim; ++d) off += idx[d] * strides[d];
    dst[k] = src[off];
    for (int d = ndim - 1; d >= 0; --d) {
      if (++idx[d] < shape[d]) break;
      idx[d] = 0;
    }
  }
}

// Upload a host tensor (any strides) into a device slot as row-major fp32.
int upload_tensor(tsr_ctx* ctx, const float* host, int ndim, const int64_t* shape,
                  const int64_t* strides, float** d_out) {
  int64_t n = numel(ndim, shape);
  void* d;
  TSR_TRY(slot_get(ctx, SLOT_TENSOR, sizeof(float) * n, &d));
  if (is_row_major(ndim, shape, strides)) {
    TSR_CUDA(cudaMemcpyAsync(d, host, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
  } else {
    void* stage;
    TSR_TRY(pinned_get(ctx, sizeof(float) * n, &stage));
    TSR_CUDA(cudaStreamSynchronize(ctx->stream));
    pack_host(host, ndim, shape, strides, (float*)stage);
    TSR_CUDA(cudaMemcpyAsync(d, stage, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
  }
  *d_out = (float*)d;
  return TSR_OK;
}

int upload_factors(tsr_ctx* ctx, int ndim, const int64_t* shape, const float* const* factors,
                   int64_t R, FactorTable* ft) {
  int64_t total = 0;
  for (int m = 0; m < ndim; ++m) total += shape[m] * R;
  void* d;
  TSR_TRY(slot_get(ctx, SLOT_FACTORS, sizeof(float) * total, &d));
  float* p = (float*)d;
  for (int m = 0; m < ndim; ++m) {
    TSR_CUDA(cudaMemcpyAsync(p, factors[m], sizeof(float) * shape[m] * R, cudaMemcpyHostToDevice,
                             ctx->stream));
    ft->ptr[m] = p;
    ft->rows[m] = shape[m];
    p += shape[m] * R;
  }
  return TSR_OK;
}

// SplitMix64 U(0,1) stream identical to tenrso_b200.synth.uniform.
uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
void seeded_uniform(uint64_t seed, uint64_t stream, int64_t n, float* out) {
  const uint64_t golden = 0x9E3779B97F4A7C15ull;
  uint64_t key = mix64(seed * 0x100000001B3ull + stream * 0x2545F4914F6CDD1Dull + golden);
  for (int64_t i = 0; i < n; ++i) {
    uint64_t r = mix64(key + (uint64_t)i * golden);
    out[i] = (float)((double)(r >> 11) * (1.0 / 9007199254740992.0));
  }
}

// Per-mode operand of the MTTKRP: unfolding copies in the precision needed.
void mode_operand_bytes(const Unfolding& u, int precision, size_t* a_bytes, size_t* b_bytes) {
  if (precision == TSR_PREC_BF16X3) {
    *a_bytes = *b_bytes = 2 * (size_t)u.rows * u.ld;
  } else {
    *a_bytes = (u.mode == 0 && u.ld == u.cols) ? 0 : sizeof(float) * (size_t)u.rows * u.ld;
    *b_bytes = 0;
  }
}

int prepare_mode_into(tsr_ctx* ctx, const float* dX, int ndim, const int64_t* shape, int mode,
                      int precision, void* buf_a, void* buf_b, ModeOperand* op) {
  op->u = make_unfolding(ndim, shape, mode);
  const Unfolding& u = op->u;
  if (precision == TSR_PREC_BF16X3) {
    TSR_TRY(launch_unfold_bf16x2(ctx, dX, shape, u, (__nv_bfloat16*)buf_a,
                                 (__nv_bfloat16*)buf_b));
    op->hi = (const __nv_bfloat16*)buf_a;
    op->lo = (const __nv_bfloat16*)buf_b;
    return TSR_OK;
  }
  // mode 0 of a row-major tensor is already its unfolding when rows are aligned
  if (mode == 0 && u.ld == u.cols) {
    op->f32 = dX;
    return TSR_OK;
  }
  TSR_TRY(launch_unfold_f32(ctx, dX, shape, u, (float*)buf_a));
  op->f32 = (const float*)buf_a;
  return TSR_OK;
}

int prepare_mode(tsr_ctx* ctx, const float* dX, int ndim, const int64_t* shape, int mode,
                 int precision, int slot_index, ModeOperand* op) {
  size_t ab, bb;
  mode_operand_bytes(make_unfolding(ndim, shape, mode), precision, &ab, &bb);
  void *a = nullptr, *b = nullptr;
  if (ab) TSR_TRY(slot_get(ctx, SLOT_UNFOLD0 + slot_index, ab, &a));
  if (bb) TSR_TRY(slot_get(ctx, SLOT_UNFOLD_LO + slot_index, bb, &b));
  return prepare_mode_into(ctx, dX, ndim, shape, mode, precision, a, b, op);
}

// Split-K partial MTTKRP of one mode into `partials` (allocated here).
// Run length of the FP32 operand for the run-scaled kernel (the fastest other
// mode), or 0 when its rows are not 16-byte aligned.
int64_t simt_run_len(const ModeOperand& op) {
  if (!op.f32 || ((uintptr_t)op.f32 & 15) != 0 || (op.u.ld & 3) != 0 || op.u.n_other < 1)
    return 0;
  return op.u.other_size[op.u.n_other - 1];
}

int run_mttkrp_partials(tsr_ctx* ctx, const ModeOperand& op, const FactorTable& ft, int R,
                        int precision, float** partials, int* splits) {
  KRSpec kr = make_krspec(op.u, ft, R);
  SplitPlan plan;
  bool tc = precision == TSR_PREC_BF16X3;
  if (tc && !tc_supported(op.u, R))
    return fail(TSR_E_UNSUPPORTED, "BF16X3 path needs rank <= 256 (got %d)", R);
  plan = tc ? plan_tc(ctx, op.u, R)
            : plan_simt(ctx, op.u.rows, op.u.cols, R, simt_run_len(op));
  void* p;
  TSR_TRY(slot_get(ctx, SLOT_PARTIALS, sizeof(float) * partial_floats(plan, op.u.rows, R), &p));
  if (tc)
    TSR_TRY(launch_mttkrp_tc(ctx, op.hi, op.lo, op.u, kr, plan, (float*)p, op.resident));
  else
    TSR_TRY(launch_mttkrp_simt(ctx, op.f32, op.u, kr, plan, (float*)p));
  *partials = (float*)p;
  *splits = plan.splits;
  return TSR_OK;
}

int check_precision(int precision) {
  if (precision != TSR_PREC_FP32 && precision != TSR_PREC_BF16X3)
    return fail(TSR_E_INVALID_ARG, "unknown precision %d", precision);
  return TSR_OK;
}

// The single-layout BF16x3 operand of a 3-way tensor for a standalone MTTKRP
// of `mode`: X's hi/lo halves and the B image of the contracted factor (U1
// for mode 2, U2 otherwise), in the context's slots.
static bool dense3_usable(int ndim, const int64_t* shape, int R, int precision, const float* dX) {
  return precision == TSR_PREC_BF16X3 && dense3_supported(ndim, shape, R) &&
         ((uintptr_t)dX & 15) == 0;
}

static int prepare_dense3(tsr_ctx* ctx, const float* dX, const int64_t* shape, int R,
                          const FactorTable& ft, int mode, Dense3* d) {
  std::memset(d, 0, sizeof(*d));
  d->I = shape[0];
  d->J = shape[1];
  d->K = shape[2];
  d->R = R;
  d->n_pad = dense3_n_pad(R);
  const size_t n = (size_t)(d->I * d->J * d->K);
  void *hp, *lp, *ip, *np;
  TSR_TRY(slot_get(ctx, SLOT_D3_HI, sizeof(__nv_bfloat16) * n, &hp));
  TSR_TRY(slot_get(ctx, SLOT_D3_LO, sizeof(__nv_bfloat16) * n, &lp));
  const int c = mode == 2 ? 1 : 2;
  const int64_t L = c == 1 ? d->J : d->K;
  TSR_TRY(slot_get(ctx, SLOT_D3_IMG, bimage_bytes(L, d->n_pad), &ip));
  TSR_TRY(slot_get(ctx, SLOT_MISC2, sizeof(double), &np));  // ||X||^2, not needed here
  d->hi = (const __nv_bfloat16*)hp;
  d->lo = (const __nv_bfloat16*)lp;
  d->bimg[c] = (uint8_t*)ip;
  TSR_TRY(launch_split_bf16(ctx, ctx->stream, dX, (int64_t)n, (__nv_bfloat16*)hp,
                            (__nv_bfloat16*)lp, (double*)np));
  TSR_TRY(launch_bimage(ctx, ctx->stream, ft.ptr[c], L, R, d->n_pad, d->bimg[c]));
  return TSR_OK;
}

// Device MTTKRP for one mode into d_out (I_mode x R).
int mttkrp_device(tsr_ctx* ctx, const float* dX, int ndim, const int64_t* shape,
                  const FactorTable& ft, int R, int mode, int precision, float* d_out) {
  if (dense3_usable(ndim, shape, R, precision, dX)) {
    Dense3 d;
    TSR_TRY(prepare_dense3(ctx, dX, shape, R, ft, mode, &d));
    const SplitPlan plan = plan_mttkrp3(ctx, d, mode);
    void* p;
    TSR_TRY(slot_get(ctx, SLOT_PARTIALS,
                     sizeof(float) * (size_t)plan.splits * dense3_rows(d, mode) * R, &p));
    TSR_TRY(launch_mttkrp3(ctx, ctx->stream, d, mode, ft, plan, (float*)p, false));
    return launch_mttkrp_reduce(ctx, (float*)p, plan.splits, shape[mode] * R, d_out);
  }
  ModeOperand op;
  TSR_TRY(prepare_mode(ctx, dX, ndim, shape, mode, precision, 0, &op));
  float* partials;
  int splits;
  TSR_TRY(run_mttkrp_partials(ctx, op, ft, R, precision, &partials, &splits));
  TSR_TRY(launch_mttkrp_reduce(ctx, partials, splits, op.u.rows * R, d_out));
  return TSR_OK;
}

// ---------------------------------------------------------------------------
// CP-ALS driver (cp/core.rs:59-182) on a device-resident tensor.
//
// One ALS sweep runs on two streams so that the FP64 inverse overlaps the
// MTTKRP: the main stream carries MTTKRP_n -> solve_n (which also forms the
// Gram of the new U_n and, for the last mode, the fit), the aux stream
// inverse_n, which starts when solve_{n-1} has finished (inverse_0 first
// forms the previous sweep's fit, off the main stream). Up to 16 sweeps are
// captured into one CUDA graph, replayed until max_iters sweeps ran; every kernel
// returns at entry once the device-side stop flag is set, which reproduces the
// reference's early exits without host round trips.
// ---------------------------------------------------------------------------
struct SweepArgs {
  const float* dX;
  int ndim;
  int64_t shape[kMaxModes];
  int R;
  int precision;
  double tol;
  float ridge;
  double l2;   // cp_als_constrained: Gram ridge, soft threshold, projection
  float l1;
  int nonneg;
  int orth;           // orthonormalize each updated factor (QR)
  int tik_order;      // Tikhonov penalty of order > 0 on the Gram
  double tik_lambda;
  FactorTable ft;
  const void* op_ptrs[3 * kMaxModes];
  float* partials;
  AlsBuffers b;
  const tsr_sparse* sp;  // sparse source (CSF MTTKRP) instead of the dense unfoldings
  double* acc64;         // sparse: FP64 accumulator of the CSF MTTKRP
  int d3_on;             // 3-way BF16x3: the single-layout MTTKRP on d3
  Dense3 d3;
  long long wait_budget;  // baked into the captured MTTKRP launches
};

static int enqueue_sweep(tsr_ctx* ctx, const SweepArgs& a, const std::vector<ModeOperand>& ops) {
  cudaStream_t A = ctx->stream, B = ctx->aux;
  TSR_CUDA(cudaEventRecord(ctx->ev[0], A));
  TSR_CUDA(cudaStreamWaitEvent(B, ctx->ev[0], 0));
  for (int n = 0; n < a.ndim; ++n) {
    const bool last = n == a.ndim - 1;
    TSR_TRY(launch_chol(ctx, B, a.b, a.ndim, n, a.R, a.ridge, last, a.tol, a.l2, a.tik_order,
                        a.tik_lambda));
    TSR_CUDA(cudaEventRecord(ctx->ev[1 + 2 * n], B));
    float* partials = a.partials;
    int splits = 1;
    uint8_t* img = nullptr;  // the B image this mode's new factor feeds
    if (a.sp) {
      TSR_TRY(launch_mttkrp_csf(ctx, A, a.sp, a.ft, a.R, n, partials, a.acc64));
    } else if (a.d3_on) {
      const SplitPlan plan = plan_mttkrp3(ctx, a.d3, n);
      TSR_TRY(launch_mttkrp3(ctx, A, a.d3, n, a.ft, plan, partials, true));
      splits = plan.splits;
      img = n == 0 ? nullptr : a.d3.bimg[n];  // U1 feeds mode 2, U2 modes 0 and 1
    } else {
      TSR_TRY(run_mttkrp_partials(ctx, ops[n], a.ft, a.R, a.precision, &partials, &splits));
    }
    TSR_CUDA(cudaStreamWaitEvent(A, ctx->ev[1 + 2 * n], 0));
    TSR_TRY(launch_solve(ctx, A, a.b, partials, splits, a.shape[n], a.R,
                         const_cast<float*>(a.ft.ptr[n]), a.b.grams + (size_t)n * a.R * a.R,
                         last, a.ndim, a.tol, a.l1, a.nonneg, img, a.d3.n_pad));
    if (a.orth)  // core.rs:361-364, after the soft threshold and the projection
      TSR_TRY(launch_orthonormalize(ctx, A, a.b, a.ndim, n, a.R, a.shape[n],
                                    const_cast<float*>(a.ft.ptr[n]),
                                    a.b.grams + (size_t)n * a.R * a.R, last, partials, splits));
    if (!last) {  // the next inverse needs this mode's Gram
      TSR_CUDA(cudaEventRecord(ctx->ev[2 + 2 * n], A));
      TSR_CUDA(cudaStreamWaitEvent(B, ctx->ev[2 + 2 * n], 0));
    }
  }
  return TSR_OK;
}

int cp_als_device(tsr_ctx* ctx, const float* dX, const tsr_sparse* sp, int ndim,
                  const int64_t* shape, int64_t rank, int max_iters, double tol,
                  const float* d_init, int precision, double time_limit_s, float* d_out,
                  tsr_cp_info* info, const tsr_cp_constraints* cons = nullptr) {
  auto t_start = std::chrono::steady_clock::now();
  // core.rs:82-94
  if (rank == 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  for (int d = 0; d < ndim; ++d)
    if (rank > shape[d]) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  if (!(tol >= 0.0 && tol < 1.0)) return fail(TSR_E_INVALID_TOL, "Invalid tolerance: %g", tol);
  TSR_TRY(check_precision(precision));
  if (ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d exceeds the supported %d", ndim, kMaxModes);
  if (rank > kMaxRank)
    return fail(TSR_E_UNSUPPORTED, "rank %lld exceeds the supported %d", (long long)rank,
                kMaxRank);
  if (ndim < 2 && max_iters > 0)
    return fail(TSR_E_SHAPE, "Shape mismatch: Need at least 2 factor matrices for MTTKRP");
  if (cons) {  // types.rs:105-182 (validate), core.rs:262-267
    if (sp) return fail(TSR_E_UNSUPPORTED, "constraints apply to the dense CP-ALS only");
    if (!(cons->l2 >= 0.0) || !std::isfinite(cons->l2))
      return fail(TSR_E_INVALID_REGULARIZATION,
                  "Invalid regularization parameter: L2 lambda must be >= 0, got %g", cons->l2);
    if (!(cons->l1 >= 0.0) || !std::isfinite(cons->l1))
      return fail(TSR_E_INVALID_REGULARIZATION,
                  "Invalid regularization parameter: L1 lambda must be >= 0, got %g", cons->l1);
    if (cons->tikhonov_order < 0)
      return fail(TSR_E_INVALID_ARG, "negative Tikhonov order %d", cons->tikhonov_order);
    if (cons->tikhonov_order > 0 &&
        (!(cons->tikhonov_lambda >= 0.0) || !std::isfinite(cons->tikhonov_lambda)))
      return fail(TSR_E_INVALID_REGULARIZATION,
                  "Invalid regularization parameter: Tikhonov lambda must be >= 0, got %g",
                  cons->tikhonov_lambda);
  }
  const int R = (int)rank;
  const int64_t n = numel(ndim, shape);

  SweepArgs a;
  std::memset(&a, 0, sizeof(a));  // the bytes of `a` are the graph cache key
  a.dX = dX;
  a.ndim = ndim;
  for (int m = 0; m < ndim; ++m) a.shape[m] = shape[m];
  a.R = R;
  a.precision = precision;
  a.tol = tol;
  a.ridge = std::numeric_limits<float>::epsilon() * (float)(R * 10);
  a.sp = sp;
  a.wait_budget = ctx->wait_budget;
  if (cons) {
    a.l2 = cons->l2;
    a.l1 = (float)cons->l1;  // the threshold in the factors' type (core.rs:351)
    a.nonneg = cons->nonnegative ? 1 : 0;
    a.orth = cons->orthogonal ? 1 : 0;
    if (cons->tikhonov_order > 0) {  // core.rs:330-334: replaces the ridge
      a.tik_order = cons->tikhonov_order;
      a.tik_lambda = cons->tikhonov_lambda;
      a.l2 = 0.0;
    }
  }

  // factors live in d_out for the whole run (updated in place)
  int64_t ftotal = 0;
  for (int m = 0; m < ndim; ++m) {
    a.ft.ptr[m] = d_out + ftotal;
    a.ft.rows[m] = shape[m];
    ftotal += shape[m] * R;
  }
  if (d_init != d_out)
    TSR_CUDA(cudaMemcpyAsync(d_out, d_init, sizeof(float) * ftotal, cudaMemcpyDeviceToDevice,
                             ctx->stream));

  // every buffer is sized before any capture (no allocation inside a graph)
  const int hist_n = std::max(max_iters, 1);
  const size_t gbytes = sizeof(double) * (size_t)(2 * ndim + 1) * R * R;
  const size_t sbytes = 256 + sizeof(double) * hist_n;
  void *gp, *stp;
  TSR_TRY(slot_get(ctx, SLOT_GRAMS, gbytes, &gp));
  TSR_TRY(slot_get(ctx, SLOT_STATE, sbytes, &stp));
  a.b.grams = (double*)gp;
  a.b.hadam = a.b.grams + (size_t)ndim * R * R;
  a.b.ginv = a.b.hadam + (size_t)ndim * R * R;
  a.b.state = (AlsState*)stp;
  a.b.history = (double*)((char*)stp + 256);
  TSR_CUDA(cudaMemsetAsync(stp, 0, sbytes, ctx->stream));
  TSR_CUDA(cudaMemsetAsync(gp, 0, gbytes, ctx->stream));
  TSR_TRY(reset_status(ctx));  // the MTTKRP kernels' status word
  const bool tracing = ctx->trace_start != nullptr;
  if (tracing) {  // this call's launches take slots from 0
    ctx->trace_next = 0;
    TSR_CUDA(cudaMemsetAsync(ctx->trace_start, 0xFF, sizeof(unsigned long long) * ctx->trace_cap,
                             ctx->stream));
    TSR_CUDA(cudaMemsetAsync(ctx->trace_end, 0, sizeof(unsigned long long) * ctx->trace_cap,
                             ctx->stream));
  }
  if (cons && cons->nonnegative && cons->validate_nonneg_input) {
    // helpers.rs:705-716: one pass over X before any factor is touched
    TSR_TRY(launch_any_negative(ctx, ctx->stream, dX, n, &a.b.state->pad));
    int neg = 0;
    TSR_CUDA(cudaMemcpyAsync(&neg, &a.b.state->pad, sizeof(int), cudaMemcpyDeviceToHost,
                             ctx->stream));
    TSR_CUDA(cudaStreamSynchronize(ctx->stream));
    if (neg)
      return fail(TSR_E_NONNEG_VIOLATION,
                  "Non-negative constraint violated: input tensor contains negative values");
  }
  if (a.nonneg) TSR_TRY(launch_clamp_nonneg(ctx, ctx->stream, d_out, ftotal));

  // per-mode unfoldings, resident for the whole run (the reference re-unfolds
  // in every mttkrp call, mttkrp.rs:126)
  std::vector<ModeOperand> ops(ndim);
  size_t pmax = 0;
  // 3-way BF16x3: one bf16 hi/lo copy of X read by every mode (no unfoldings)
  // (the orthonormalisation rewrites a factor after its solve, so the solve's
  // B image would be stale: that run takes the per-mode unfoldings)
  const bool d3 = !sp && max_iters > 0 && precision == TSR_PREC_BF16X3 &&
                  dense3_supported(ndim, shape, R) && ((uintptr_t)dX & 15) == 0 &&
                  !(cons && cons->orthogonal);
  const bool fused_unfold = !d3 && !sp && max_iters > 0 && unfold3_supported(ndim, shape);
  if (d3) {
    Dense3& d = a.d3;
    a.d3_on = 1;
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
    d.bimg[0] = nullptr;
    d.bimg[1] = (uint8_t*)ip;
    d.bimg[2] = (uint8_t*)ip + img1;
    for (int m = 0; m < 3; ++m) {
      const SplitPlan p = plan_mttkrp3(ctx, d, m);
      pmax = std::max(pmax, (size_t)p.splits * dense3_rows(d, m) * R);
    }
    void* pp;
    TSR_TRY(slot_get(ctx, SLOT_PARTIALS, sizeof(float) * pmax, &pp));
    a.partials = (float*)pp;
    // the initial Grams on the aux stream beside the split pass; the B images
    // of the initial U1 and U2 (the solves rewrite them as the factors change)
    TSR_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
    TSR_CUDA(cudaStreamWaitEvent(ctx->aux, ctx->ev[0], 0));
    for (int m = 0; m < ndim; ++m)
      TSR_TRY(launch_gram(ctx, ctx->aux, a.ft.ptr[m], shape[m], R,
                          a.b.grams + (size_t)m * R * R, false));
    TSR_TRY(launch_bimage(ctx, ctx->aux, a.ft.ptr[1], d.J, R, d.n_pad, d.bimg[1]));
    TSR_TRY(launch_bimage(ctx, ctx->aux, a.ft.ptr[2], d.K, R, d.n_pad, d.bimg[2]));
    TSR_CUDA(cudaEventRecord(ctx->ev[1], ctx->aux));
    TSR_TRY(launch_split_bf16(ctx, ctx->stream, dX, n, (__nv_bfloat16*)hp, (__nv_bfloat16*)lp,
                              &a.b.state->xnorm_sq));
    TSR_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->ev[1], 0));
  } else if (max_iters > 0 && sp) {
    for (int m = 0; m < ndim; ++m) pmax = std::max(pmax, (size_t)shape[m] * R);
    void* pp;
    TSR_TRY(slot_get(ctx, SLOT_PARTIALS, sizeof(float) * pmax, &pp));
    a.partials = (float*)pp;
    void* ap;
    TSR_TRY(slot_get(ctx, SLOT_MISC1, sizeof(double) * pmax, &ap));
    a.acc64 = (double*)ap;
  } else if (max_iters > 0) {
    // 3-way tensors: every unfolding (and ||X||^2) in one pass over X
    void* uhi[3] = {nullptr, nullptr, nullptr};
    void* ulo[3] = {nullptr, nullptr, nullptr};
    for (int m = 0; m < ndim; ++m) {
      if (fused_unfold) {
        ops[m].u = make_unfolding(ndim, shape, m);
        size_t ab, bb;
        mode_operand_bytes(ops[m].u, precision, &ab, &bb);
        if (ab) TSR_TRY(slot_get(ctx, SLOT_UNFOLD0 + m, ab, &uhi[m]));
        if (bb) TSR_TRY(slot_get(ctx, SLOT_UNFOLD_LO + m, bb, &ulo[m]));
        if (precision == TSR_PREC_BF16X3) {
          ops[m].hi = (const __nv_bfloat16*)uhi[m];
          ops[m].lo = (const __nv_bfloat16*)ulo[m];
        } else {
          ops[m].f32 = m == 0 ? dX : (const float*)uhi[m];
        }
      } else {
        TSR_TRY(prepare_mode(ctx, dX, ndim, shape, m, precision, m, &ops[m]));
      }
      const bool tc = precision == TSR_PREC_BF16X3;
      SplitPlan p = tc ? plan_tc(ctx, ops[m].u, R)
                       : plan_simt(ctx, ops[m].u.rows, ops[m].u.cols, R, simt_run_len(ops[m]));
      pmax = std::max(pmax, partial_floats(p, ops[m].u.rows, R));
      ops[m].resident = true;  // prepared here, before the sweep is enqueued
      a.op_ptrs[3 * m] = ops[m].f32;
      a.op_ptrs[3 * m + 1] = ops[m].hi;
      a.op_ptrs[3 * m + 2] = ops[m].lo;
    }
    void* pp;
    TSR_TRY(slot_get(ctx, SLOT_PARTIALS, sizeof(float) * pmax, &pp));
    a.partials = (float*)pp;
    if (fused_unfold) {
      // the initial Grams run on the aux stream beside the unfold pass
      TSR_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
      TSR_CUDA(cudaStreamWaitEvent(ctx->aux, ctx->ev[0], 0));
      for (int m = 0; m < ndim; ++m)
        TSR_TRY(launch_gram(ctx, ctx->aux, a.ft.ptr[m], shape[m], R,
                            a.b.grams + (size_t)m * R * R, false));
      TSR_CUDA(cudaEventRecord(ctx->ev[1], ctx->aux));
      TSR_TRY(launch_unfold3(ctx, dX, shape, precision == TSR_PREC_BF16X3, uhi,
                             precision == TSR_PREC_BF16X3 ? ulo : nullptr,
                             &a.b.state->xnorm_sq));
      TSR_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->ev[1], 0));
    }
  }
  if (sp)  // sum of squared values, FP64, computed when the tensor was built
    TSR_CUDA(cudaMemcpyAsync(&a.b.state->xnorm_sq, &sp->norm_sq, sizeof(double),
                             cudaMemcpyHostToDevice, ctx->stream));
  else if (!fused_unfold && !d3)
    TSR_TRY(launch_norm_sq(ctx, ctx->stream, dX, n, &a.b.state->xnorm_sq));
  if (!fused_unfold && !d3)
    for (int m = 0; m < ndim; ++m)
      TSR_TRY(launch_gram(ctx, ctx->stream, a.ft.ptr[m], shape[m], R,
                          a.b.grams + (size_t)m * R * R, false));

  const bool time_limited = time_limit_s >= 0.0;
  bool stopped_by_time = false;
  if (!time_limited && max_iters > 0) {
    // Sweeps are captured kSweepsPerGraph at a time into one graph (a graph
    // launch per sweep costs more host and front-end time than the sweep's
    // launch gaps); whole chunks are replayed, then a graph of the remainder.
    constexpr int kSweepsPerGraph = 16;
    const int chunk = std::min(max_iters, kSweepsPerGraph);
    const int n_chunks = max_iters / chunk, rem = max_iters % chunk;
    auto graph_for = [&](int nsweeps, tsr_ctx::SweepGraph** out) -> int {
      std::vector<uint8_t> key((const uint8_t*)&a, (const uint8_t*)&a + sizeof(a));
      key.insert(key.end(), (const uint8_t*)&nsweeps, (const uint8_t*)&nsweeps + sizeof(nsweeps));
      // a traced call captures afresh, so its launches own this call's slots
      for (auto& g : ctx->sweep_graphs)
        if (g.exec && g.key == key && !tracing) {
          g.last_use = ++ctx->graph_clock;
          *out = &g;
          return TSR_OK;
        }
      if ((int)ctx->sweep_graphs.size() >= tsr_ctx::kMaxGraphs) {
        auto lru = std::min_element(
            ctx->sweep_graphs.begin(), ctx->sweep_graphs.end(),
            [](const tsr_ctx::SweepGraph& x, const tsr_ctx::SweepGraph& y) {
              return x.last_use < y.last_use;
            });
        if (lru->exec) cudaGraphExecDestroy(lru->exec);
        ctx->sweep_graphs.erase(lru);
      }
      cudaGraph_t g;
      const int64_t before = ctx->launches;
      TSR_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      int rc = TSR_OK;
      for (int i = 0; i < nsweeps && rc == TSR_OK; ++i) rc = enqueue_sweep(ctx, a, ops);
      cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
      if (rc != TSR_OK) return rc;
      TSR_CUDA(ce);
      tsr_ctx::SweepGraph sg;
      sg.launches = ctx->launches - before;
      ctx->launches = before;
      cudaError_t ie = cudaGraphInstantiate(&sg.exec, g, 0);
      cudaGraphDestroy(g);
      TSR_CUDA(ie);
      sg.key = std::move(key);
      sg.last_use = ++ctx->graph_clock;
      ctx->sweep_graphs.push_back(std::move(sg));
      *out = &ctx->sweep_graphs.back();
      return TSR_OK;
    };
    tsr_ctx::SweepGraph *gc = nullptr, *gr = nullptr;
    TSR_TRY(graph_for(chunk, &gc));
    if (rem > 0) TSR_TRY(graph_for(rem, &gr));  // evicts the least recently used, never gc
    for (int c = 0; c < n_chunks; ++c) {
      TSR_CUDA(cudaGraphLaunch(gc->exec, ctx->stream));
      ctx->launches += gc->launches;
    }
    if (rem > 0) {
      TSR_CUDA(cudaGraphLaunch(gr->exec, ctx->stream));
      ctx->launches += gr->launches;
    }
  } else {
    for (int iter = 0; iter < max_iters; ++iter) {
      AlsState hs;
      TSR_CUDA(cudaMemcpyAsync(&hs, a.b.state, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
      TSR_CUDA(cudaStreamSynchronize(ctx->stream));
      if (hs.done) break;
      // core.rs:118-124: checked at the start of every iteration
      const double el =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
      if (el > time_limit_s) {
        stopped_by_time = true;
        break;
      }
      TSR_TRY(enqueue_sweep(ctx, a, ops));
    }
  }
  if (max_iters > 0) TSR_TRY(launch_fit(ctx, ctx->stream, a.b, ndim, R, tol));
  // one read-back into pinned memory, one synchronization: the state with the
  // fit history behind it (SLOT_STATE: state at 0, history at 256) and the
  // MTTKRP kernels' status word
  const size_t hist_bytes = sizeof(double) * (size_t)std::max(max_iters, 0);
  void* rbp;
  TSR_TRY(readback_get(ctx, 256 + hist_bytes + 16, &rbp));
  uint8_t* rb = (uint8_t*)rbp;
  TSR_CUDA(cudaMemcpyAsync(rb, a.b.state, 256 + hist_bytes, cudaMemcpyDeviceToHost, ctx->stream));
  TSR_CUDA(cudaMemcpyAsync(rb + 256 + hist_bytes, ctx->d_status, sizeof(unsigned),
                           cudaMemcpyDeviceToHost, ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  AlsState hs;
  std::memcpy(&hs, rb, sizeof(hs));
  unsigned mst = 0;
  std::memcpy(&mst, rb + 256 + hist_bytes, sizeof(mst));
  if (mst) {
    TSR_TRY(reset_status(ctx));
    if (mst & DS_TIMEOUT) return fail(TSR_E_TIMEOUT, "device wait timed out in the MTTKRP kernel");
  }
  if (hs.status & DS_TIMEOUT)
    return fail(TSR_E_TIMEOUT, "device wait timed out in the CP-ALS sweep");
  if (hs.status & DS_NOT_SPD)
    return fail(TSR_E_NOT_SPD,
                "Linear algebra error: Gram matrix is not positive definite (ridge %g also "
                "failed)",
                (double)a.ridge);
  if (info) {
    info->fit = hs.fit;
    info->iters = hs.iter;
    info->reason = stopped_by_time ? TSR_REASON_TIME_LIMIT
                   : hs.done       ? hs.reason
                                   : TSR_REASON_MAX_ITERATIONS;
    info->oscillation_count = hs.osc;
    info->oscillated = hs.osc > 0;
    info->final_fit_change = hs.final_change;
    info->ridge_used = hs.ridge_used;
    if (info->fit_history && hs.iter > 0)
      std::memcpy(info->fit_history, rb + 256, sizeof(double) * std::min(hs.iter, max_iters));
  }
  return TSR_OK;
}

// cudaFuncSetAttribute acts on the current device's context, so the raised
// shared-memory limits are set once per device (guarded: several host threads
// may make their first call at the same time).
void init_kernel_attributes() {
  static std::mutex mu;
  static uint64_t done_mask = 0;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> lock(mu);
  if (done_mask & (1ull << dev)) return;
  init_tc_attributes();
  init_mttkrp3_attributes();
  init_simt_attributes();
  init_als_attributes();
  init_adjoint_attributes();
  init_csf_attributes();
  init_batched_attributes();
  init_accel_attributes();
  init_hicoo_attributes();
  init_init_attributes();
  init_f64_attributes();
  done_mask |= 1ull << dev;
}

}  // namespace tsr

using namespace tsr;

extern "C" {

int tsr_khatri_rao_f32(tsr_ctx* ctx, const float* a, int64_t I, int64_t Ka, const float* b,
                       int64_t J, int64_t Kb, float* out) {
  if (Ka != Kb)
    return fail(TSR_E_COLS_MISMATCH,
                "Number of columns must match: A has %lld columns, B has %lld columns",
                (long long)Ka, (long long)Kb);
  TSR_TRY(check_ctx(ctx));
  if (I * J * Ka == 0) return TSR_OK;
  void *da, *db, *dc;
  TSR_TRY(slot_get(ctx, SLOT_MISC0, sizeof(float) * I * Ka, &da));
  TSR_TRY(slot_get(ctx, SLOT_MISC1, sizeof(float) * J * Ka, &db));
  TSR_TRY(slot_get(ctx, SLOT_OUT, sizeof(float) * I * J * Ka, &dc));
  TSR_CUDA(cudaMemcpyAsync(da, a, sizeof(float) * I * Ka, cudaMemcpyHostToDevice, ctx->stream));
  TSR_CUDA(cudaMemcpyAsync(db, b, sizeof(float) * J * Ka, cudaMemcpyHostToDevice, ctx->stream));
  TSR_TRY(launch_khatri_rao(ctx, (const float*)da, I, (const float*)db, J, Ka, (float*)dc));
  TSR_CUDA(cudaMemcpyAsync(out, dc, sizeof(float) * I * J * Ka, cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

int tsr_mttkrp_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                   const int64_t* strides, const float* const* factors, int n_factors,
                   const int64_t* factor_rows, const int64_t* factor_cols, int mode,
                   int precision, float* out) {
  if (!shape || (n_factors > 0 && (!factors || !factor_rows || !factor_cols)))
    return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(validate_mttkrp(ndim, shape, n_factors, factor_rows, factor_cols, mode));
  TSR_TRY(check_precision(precision));
  TSR_TRY(check_sizes(ndim, shape, factor_cols[0]));
  TSR_TRY(check_ctx(ctx));
  const int R = (int)factor_cols[0];
  const int64_t nout = shape[mode] * R;
  if (nout == 0) return TSR_OK;
  if (numel(ndim, shape) == 0 || R == 0) {
    std::memset(out, 0, sizeof(float) * nout);
    return TSR_OK;
  }
  float* dX;
  TSR_TRY(upload_tensor(ctx, tensor, ndim, shape, strides, &dX));
  FactorTable ft{};
  TSR_TRY(upload_factors(ctx, ndim, shape, factors, R, &ft));
  void* dout;
  TSR_TRY(slot_get(ctx, SLOT_OUT, sizeof(float) * nout, &dout));
  TSR_TRY(mttkrp_device(ctx, dX, ndim, shape, ft, R, mode, precision, (float*)dout));
  TSR_CUDA(cudaMemcpyAsync(out, dout, sizeof(float) * nout, cudaMemcpyDeviceToHost, ctx->stream));
  return check_device_status(ctx);
}

int tsr_mttkrp_blocked_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                           const int64_t* strides, const float* const* factors, int n_factors,
                           const int64_t* factor_rows, const int64_t* factor_cols, int mode,
                           int64_t tile_size, int precision, float* out) {
  if (tile_size <= 0) return fail(TSR_E_TILE_SIZE, "Tile size must be greater than 0");
  return tsr_mttkrp_f32(ctx, tensor, ndim, shape, strides, factors, n_factors, factor_rows,
                        factor_cols, mode, precision, out);
}

int tsr_mttkrp_all_modes_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                             const float* const* factors, int64_t rank, int precision,
                             float* const* out) {
  if (!shape || !factors || !out) return fail(TSR_E_INVALID_ARG, "null argument");
  std::vector<int64_t> cols(ndim, rank);
  TSR_TRY(validate_mttkrp(ndim, shape, ndim, shape, cols.data(), 0));
  TSR_TRY(check_precision(precision));
  TSR_TRY(check_ctx(ctx));
  const int R = (int)rank;
  float* dX = nullptr;
  TSR_TRY(upload_tensor(ctx, tensor, ndim, shape, nullptr, &dX));
  FactorTable ft{};
  TSR_TRY(upload_factors(ctx, ndim, shape, factors, R, &ft));
  for (int m = 0; m < ndim; ++m) {
    void* dout;
    TSR_TRY(slot_get(ctx, SLOT_OUT, sizeof(float) * shape[m] * R, &dout));
    TSR_TRY(mttkrp_device(ctx, dX, ndim, shape, ft, R, m, precision, (float*)dout));
    TSR_CUDA(cudaMemcpyAsync(out[m], dout, sizeof(float) * shape[m] * R, cudaMemcpyDeviceToHost,
                             ctx->stream));
    TSR_TRY(check_device_status(ctx));
  }
  return TSR_OK;
}

int tsr_mttkrp_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim, const int64_t* shape,
                       const float* const* d_factors, int64_t rank, int mode, int precision,
                       float* d_out) {
  if (!shape || !d_factors || !d_tensor || !d_out) return fail(TSR_E_INVALID_ARG, "null argument");
  std::vector<int64_t> cols(ndim, rank);
  TSR_TRY(validate_mttkrp(ndim, shape, ndim, shape, cols.data(), mode));
  TSR_TRY(check_precision(precision));
  TSR_TRY(check_sizes(ndim, shape, rank));
  TSR_TRY(check_ctx(ctx));
  const int64_t nout = shape[mode] * rank;
  if (nout == 0) return TSR_OK;
  if (numel(ndim, shape) == 0) {  // an empty sum: the output is zero
    TSR_CUDA(cudaMemsetAsync(d_out, 0, sizeof(float) * nout, ctx->stream));
    return TSR_OK;
  }
  FactorTable ft{};
  for (int m = 0; m < ndim; ++m) {
    ft.ptr[m] = d_factors[m];
    ft.rows[m] = shape[m];
  }
  TSR_TRY(mttkrp_device(ctx, d_tensor, ndim, shape, ft, (int)rank, mode, precision, d_out));
  // a bounded wait that gave up is reported (this synchronizes the stream)
  return check_device_status(ctx);
}

int tsr_profile_mttkrp_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim,
                               const int64_t* shape, const float* const* d_factors, int64_t rank,
                               int mode, int precision, int iters, int flush_l2,
                               double* ms_per_launch, int64_t* splits_out) {
  if (!shape || !d_factors || !d_tensor || !ms_per_launch || iters <= 0)
    return fail(TSR_E_INVALID_ARG, "invalid argument");
  std::vector<int64_t> cols(ndim, rank);
  TSR_TRY(validate_mttkrp(ndim, shape, ndim, shape, cols.data(), mode));
  TSR_TRY(check_precision(precision));
  TSR_TRY(check_ctx(ctx));
  FactorTable ft{};
  for (int m = 0; m < ndim; ++m) {
    ft.ptr[m] = d_factors[m];
    ft.rows[m] = shape[m];
  }
  const bool d3 = dense3_usable(ndim, shape, (int)rank, precision, d_tensor);
  ModeOperand op;
  Dense3 d;
  SplitPlan plan3;
  float* partials3 = nullptr;
  if (d3) {
    TSR_TRY(prepare_dense3(ctx, d_tensor, shape, (int)rank, ft, mode, &d));
    plan3 = plan_mttkrp3(ctx, d, mode);
    void* p;
    TSR_TRY(slot_get(ctx, SLOT_PARTIALS,
                     sizeof(float) * (size_t)plan3.splits * dense3_rows(d, mode) * rank, &p));
    partials3 = (float*)p;
  } else {
    TSR_TRY(prepare_mode(ctx, d_tensor, ndim, shape, mode, precision, 0, &op));
  }
  cudaEvent_t a, b;
  TSR_CUDA(cudaEventCreate(&a));
  TSR_CUDA(cudaEventCreate(&b));
  double total = 0.0;
  int splits = 0;
  for (int i = 0; i < iters; ++i) {
    if (flush_l2) TSR_TRY(::tsr::flush_l2(ctx, ctx->stream));
    float* partials;
    TSR_CUDA(cudaEventRecord(a, ctx->stream));
    if (d3) {
      TSR_TRY(launch_mttkrp3(ctx, ctx->stream, d, mode, ft, plan3, partials3, true));
      splits = plan3.splits;
    } else {
      TSR_TRY(run_mttkrp_partials(ctx, op, ft, (int)rank, precision, &partials, &splits));
    }
    TSR_CUDA(cudaEventRecord(b, ctx->stream));
    TSR_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    TSR_CUDA(cudaEventElapsedTime(&ms, a, b));
    total += ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms_per_launch = total / iters;
  if (splits_out) *splits_out = splits;
  return check_device_status(ctx);
}

int tsr_gram_inverse_f64(tsr_ctx* ctx, const double* gram, int64_t rank, int iters,
                         double* inverse, int* ridge_used, double* ms_per_launch) {
  if (!gram || !inverse || iters < 1) return fail(TSR_E_INVALID_ARG, "invalid argument");
  if (rank < 1 || rank > kMaxRank)
    return fail(TSR_E_UNSUPPORTED, "rank %lld outside 1..%d", (long long)rank, kMaxRank);
  TSR_TRY(check_ctx(ctx));
  const int R = (int)rank;
  const size_t RR = (size_t)R * R;
  // a 2-mode ALS state: Gram_0 = G, and the inverse of mode 1 is that of the
  // Hadamard of the other Grams, i.e. of G itself
  void *gp, *stp;
  TSR_TRY(slot_get(ctx, SLOT_GRAMS, sizeof(double) * 5 * RR, &gp));
  TSR_TRY(slot_get(ctx, SLOT_STATE, 256 + sizeof(double), &stp));
  AlsBuffers b;
  b.grams = (double*)gp;
  b.hadam = b.grams + 2 * RR;
  b.ginv = b.hadam + 2 * RR;
  b.state = (AlsState*)stp;
  b.history = (double*)((char*)stp + 256);
  TSR_CUDA(cudaMemsetAsync(stp, 0, 256 + sizeof(double), ctx->stream));
  TSR_CUDA(cudaMemcpyAsync(b.grams, gram, sizeof(double) * RR, cudaMemcpyHostToDevice,
                           ctx->stream));
  const float ridge = std::numeric_limits<float>::epsilon() * (float)(R * 10);
  cudaEvent_t e0, e1;
  TSR_CUDA(cudaEventCreate(&e0));
  TSR_CUDA(cudaEventCreate(&e1));
  TSR_TRY(launch_chol(ctx, ctx->stream, b, 2, 1, R, ridge, false, 0.0));  // warm-up
  TSR_CUDA(cudaEventRecord(e0, ctx->stream));
  for (int i = 0; i < iters; ++i) TSR_TRY(launch_chol(ctx, ctx->stream, b, 2, 1, R, ridge, false, 0.0));
  TSR_CUDA(cudaEventRecord(e1, ctx->stream));
  AlsState hs;
  TSR_CUDA(cudaMemcpyAsync(&hs, b.state, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
  TSR_CUDA(cudaMemcpyAsync(inverse, b.ginv, sizeof(double) * RR, cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ms_per_launch) *ms_per_launch = ms / iters;
  if (ridge_used) *ridge_used = hs.ridge_used;
  if (hs.status & DS_NOT_SPD)
    return fail(TSR_E_NOT_SPD,
                "Linear algebra error: Gram matrix is not positive definite (ridge %g also "
                "failed)",
                (double)ridge);
  return TSR_OK;
}

}  // extern "C"

namespace tsr {
namespace {
// out = upper triangle of g mirrored to a full symmetric R x R matrix.
__global__ void symmetrize_kernel(const double* __restrict__ g, int R, double* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < R * R; e += gridDim.x * blockDim.x) {
    const int i = e / R, j = e % R;
    out[e] = i <= j ? g[i * R + j] : g[j * R + i];
  }
}
}  // namespace
}  // namespace tsr

extern "C" {

int tsr_als_solve_dev_f32(tsr_ctx* ctx, const float* d_M, int64_t rows, int64_t rank,
                          const double* d_hadamard, float* d_U, double* d_gram,
                          double* inner_out, int* ridge_used) {
  if (!d_hadamard || !d_gram || (rows > 0 && (!d_M || !d_U)))
    return fail(TSR_E_INVALID_ARG, "null argument");
  if (rows < 0) return fail(TSR_E_INVALID_ARG, "negative row count");
  if (rank < 1 || rank > kMaxRank)
    return fail(TSR_E_UNSUPPORTED, "rank %lld outside 1..%d", (long long)rank, kMaxRank);
  TSR_TRY(check_ctx(ctx));
  const int R = (int)rank;
  const size_t RR = (size_t)R * R;
  // a 2-mode ALS state whose Gram_0 is the given Hadamard: the inverse of
  // mode 1 is then that of the Hadamard itself, and the solve of mode 1
  // writes U = M G^-1, its Gram (into Gram_1) and <M, U>
  void *gp, *stp;
  TSR_TRY(slot_get(ctx, SLOT_GRAMS, sizeof(double) * 5 * RR, &gp));
  TSR_TRY(slot_get(ctx, SLOT_STATE, 256 + sizeof(double), &stp));
  AlsBuffers b;
  b.grams = (double*)gp;
  b.hadam = b.grams + 2 * RR;
  b.ginv = b.hadam + 2 * RR;
  b.state = (AlsState*)stp;
  b.history = (double*)((char*)stp + 256);
  TSR_CUDA(cudaMemsetAsync(stp, 0, 256 + sizeof(double), ctx->stream));
  TSR_CUDA(cudaMemcpyAsync(b.grams, d_hadamard, sizeof(double) * RR, cudaMemcpyDeviceToDevice,
                           ctx->stream));
  TSR_TRY(reset_status(ctx));
  const float ridge = std::numeric_limits<float>::epsilon() * (float)(R * 10);
  TSR_TRY(launch_chol(ctx, ctx->stream, b, 2, 1, R, ridge, true, 0.0));
  if (rows > 0)
    TSR_TRY(launch_solve(ctx, ctx->stream, b, d_M, 1, rows, R, d_U, b.grams + RR, true, 2, 0.0));
  symmetrize_kernel<<<(unsigned)ceil_div((int64_t)RR, 256), 256, 0, ctx->stream>>>(b.grams + RR,
                                                                                  R, d_gram);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  AlsState hs;
  TSR_CUDA(cudaMemcpyAsync(&hs, b.state, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  TSR_TRY(check_device_status(ctx));
  if (ridge_used) *ridge_used = hs.ridge_used;
  if (inner_out) *inner_out = rows > 0 ? hs.inner : 0.0;
  if (hs.status & DS_NOT_SPD)
    return fail(TSR_E_NOT_SPD,
                "Linear algebra error: Gram matrix is not positive definite (ridge %g also "
                "failed)",
                (double)ridge);
  return TSR_OK;
}

int tsr_cp_als_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim, const int64_t* shape,
                       int64_t rank, int max_iters, double tol, const float* d_init,
                       int precision, double time_limit_s, float* d_out_factors,
                       tsr_cp_info* info) {
  if (!shape || !d_tensor || !d_init || !d_out_factors)
    return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(check_ctx(ctx));
  return cp_als_device(ctx, d_tensor, nullptr, ndim, shape, rank, max_iters, tol, d_init,
                       precision, time_limit_s, d_out_factors, info);
}

int tsr_cp_als_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                   int64_t rank, int max_iters, double tol, const float* init_factors,
                   uint64_t seed, int precision, double time_limit_s, float* out_factors,
                   tsr_cp_info* info) {
  return tsr_cp_als_constrained_f32(ctx, tensor, ndim, shape, rank, max_iters, tol, init_factors,
                                    seed, nullptr, precision, time_limit_s, out_factors, info);
}

int tsr_cp_als_constrained_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim,
                                   const int64_t* shape, int64_t rank, int max_iters,
                                   double tol, const float* d_init,
                                   const tsr_cp_constraints* constraints, int precision,
                                   double time_limit_s, float* d_out_factors,
                                   tsr_cp_info* info) {
  if (!shape || !d_tensor || !d_init || !d_out_factors)
    return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(check_ctx(ctx));
  return cp_als_device(ctx, d_tensor, nullptr, ndim, shape, rank, max_iters, tol, d_init,
                       precision, time_limit_s, d_out_factors, info, constraints);
}

int tsr_cp_als_constrained_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                               int64_t rank, int max_iters, double tol,
                               const float* init_factors, uint64_t seed,
                               const tsr_cp_constraints* constraints, int precision,
                               double time_limit_s, float* out_factors, tsr_cp_info* info) {
  if (!shape || !tensor || !out_factors) return fail(TSR_E_INVALID_ARG, "null argument");
  if (rank == 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  for (int d = 0; d < ndim; ++d)
    if (rank > shape[d]) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  if (!(tol >= 0.0 && tol < 1.0)) return fail(TSR_E_INVALID_TOL, "Invalid tolerance: %g", tol);
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
  float* dX = nullptr;
  TSR_TRY(upload_tensor(ctx, tensor, ndim, shape, nullptr, &dX));
  void* df;
  TSR_TRY(slot_get(ctx, SLOT_OUT, sizeof(float) * ftotal, &df));
  TSR_CUDA(cudaMemcpyAsync(df, init, sizeof(float) * ftotal, cudaMemcpyHostToDevice, ctx->stream));
  TSR_TRY(cp_als_device(ctx, dX, nullptr, ndim, shape, rank, max_iters, tol, (const float*)df,
                        precision, time_limit_s, (float*)df, info, constraints));
  TSR_CUDA(cudaMemcpyAsync(out_factors, df, sizeof(float) * ftotal, cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

int tsr_cp_als_sparse_dev_f32(tsr_ctx* ctx, const tsr_sparse* sp, int64_t rank, int max_iters,
                              double tol, const float* d_init, double time_limit_s,
                              float* d_out_factors, tsr_cp_info* info) {
  if (!sp || !d_init || !d_out_factors) return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(check_ctx(ctx));
  return cp_als_device(ctx, nullptr, sp, sp->ndim, sp->shape, rank, max_iters, tol, d_init,
                       TSR_PREC_FP32, time_limit_s, d_out_factors, info);
}

int tsr_cp_als_sparse_f32(tsr_ctx* ctx, const tsr_sparse* sp, int64_t rank, int max_iters,
                          double tol, const float* init_factors, uint64_t seed,
                          double time_limit_s, float* out_factors, tsr_cp_info* info) {
  if (!sp || !out_factors) return fail(TSR_E_INVALID_ARG, "null argument");
  if (rank == 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  for (int d = 0; d < sp->ndim; ++d)
    if (rank > sp->shape[d])
      return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  if (!(tol >= 0.0 && tol < 1.0)) return fail(TSR_E_INVALID_TOL, "Invalid tolerance: %g", tol);
  TSR_TRY(check_ctx(ctx));
  int64_t ftotal = 0;
  for (int m = 0; m < sp->ndim; ++m) ftotal += sp->shape[m] * rank;
  std::vector<float> init_buf;
  const float* init = init_factors;
  if (!init) {
    init_buf.resize(ftotal);
    int64_t off = 0;
    for (int m = 0; m < sp->ndim; ++m) {
      seeded_uniform(seed, 200 + m, sp->shape[m] * rank, init_buf.data() + off);
      off += sp->shape[m] * rank;
    }
    init = init_buf.data();
  }
  void* df;
  TSR_TRY(slot_get(ctx, SLOT_OUT, sizeof(float) * ftotal, &df));
  TSR_CUDA(cudaMemcpyAsync(df, init, sizeof(float) * ftotal, cudaMemcpyHostToDevice, ctx->stream));
  TSR_TRY(cp_als_device(ctx, nullptr, sp, sp->ndim, sp->shape, rank, max_iters, tol,
                        (const float*)df, TSR_PREC_FP32, time_limit_s, (float*)df, info));
  TSR_CUDA(cudaMemcpyAsync(out_factors, df, sizeof(float) * ftotal, cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

}  // extern "C"

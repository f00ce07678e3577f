// Dense-tensor helpers shared by the CP-ALS driver and the reconstruction
// adjoint: argument validation in tenrso's wording, host staging, per-mode
// MTTKRP operands and the split-K MTTKRP launch.
#pragma once
#include "mttkrp.cuh"

namespace tsr {

// mttkrp.rs:86-122 then the KR helper's bail (mttkrp.rs:196-198).
int validate_mttkrp(int ndim, const int64_t* shape, int n_factors, const int64_t* frows,
                    const int64_t* fcols, int mode);
int check_precision(int precision);
// Negative mode sizes (TSR_E_INVALID_ARG) or rank (TSR_E_INVALID_RANK).
int check_sizes(int ndim, const int64_t* shape, int64_t rank);
int64_t numel(int ndim, const int64_t* shape);

// Host tensor (any strides) into the context's tensor slot as row-major fp32.
int upload_tensor(tsr_ctx* ctx, const float* host, int ndim, const int64_t* shape,
                  const int64_t* strides, float** d_out);
// Host factor matrices (I_m x R each) into the context's factor slot.
int upload_factors(tsr_ctx* ctx, int ndim, const int64_t* shape, const float* const* factors,
                   int64_t R, FactorTable* ft);

// Per-mode operand of the MTTKRP: the mode's unfolding in the precision the
// kernel reads (fp32, or the bf16 hi/lo halves).
struct ModeOperand {
  Unfolding u;
  const float* f32 = nullptr;
  const __nv_bfloat16* hi = nullptr;
  const __nv_bfloat16* lo = nullptr;
  // written before any kernel that precedes the MTTKRP in its stream (e.g.
  // prepared before a captured sweep): the MTTKRP may stream it before its
  // programmatic-launch wait
  bool resident = false;
};
// Bytes of the two buffers prepare_mode_into needs (0 = not needed).
void mode_operand_bytes(const Unfolding& u, int precision, size_t* a_bytes, size_t* b_bytes);
// Build the operand into caller-owned buffers (fp32 / hi in a, lo in b).
int prepare_mode_into(tsr_ctx* ctx, const float* dX, int ndim, const int64_t* shape, int mode,
                      int precision, void* buf_a, void* buf_b, ModeOperand* op);
// Same, with buffers from the context's unfolding slots (slot_index 0..7).
int prepare_mode(tsr_ctx* ctx, const float* dX, int ndim, const int64_t* shape, int mode,
                 int precision, int slot_index, ModeOperand* op);
// Run length of an FP32 operand for the run-scaled SIMT kernel (0: not usable).
int64_t simt_run_len(const ModeOperand& op);
// Split-K partial MTTKRP of one mode into the context's partial slot.
int run_mttkrp_partials(tsr_ctx* ctx, const ModeOperand& op, const FactorTable& ft, int R,
                        int precision, float** partials, int* splits);
// Device MTTKRP of one mode into d_out (I_mode x R).
int mttkrp_device(tsr_ctx* ctx, const float* dX, int ndim, const int64_t* shape,
                  const FactorTable& ft, int R, int mode, int precision, float* d_out);

// Reconstruction kernels (adjoint.cu): Xhat = [[w; U]] into out, or, when X
// is given, out = alpha * (Xhat - X) with sum (Xhat - X)^2 added to *sq_err.
int launch_reconstruct(tsr_ctx* ctx, const FactorTable& ft, int ndim, int R, const float* w,
                       const float* X, float alpha, double* sq_err, float* out);
void init_adjoint_attributes();
void init_batched_attributes();
void init_accel_attributes();
void init_init_attributes();
void init_f64_attributes();

// SplitMix64 U(0,1) stream identical to tenrso_b200.synth.uniform (the
// library's InitStrategy::Random).
void seeded_uniform(uint64_t seed, uint64_t stream, int64_t n, float* out);

}  // namespace tsr

// N-mode product (TTM) and the Tucker operators built on it:
// tenrso_kernels::nmode_product / nmode_products_seq / tucker_operator /
// tucker_operator_ordered / tucker_reconstruct
// (crates/tenrso-kernels/src/nmode.rs:72-131, 241-254, 442-480, 517-531,
// 576-611).
//
// Y = X x_k M for X of shape (I_0..I_{N-1}) and M (J x I_k): viewing X as
// A x I_k x B (A = prod of the modes before k, B = prod after),
//   Y[a, j, b] = sum_i M[j, i] X[a, i, b],
// i.e. the reference's unfold / M . X_(k) / fold, written as one strided
// batched product without materialising the unfolding. For B > 1 each a is a
// GEMM C_a (J x B) = M (J x I) . X_a (I x B); for the last mode (B = 1) the
// whole product is one GEMM Y (A x J) = X (A x I) . M^T.
//
// The kernel: 64 x 64 output tile per 256-thread CTA (4 x 4 per thread),
// 16-deep K slices staged in shared memory, fp32 FMA with fp32 accumulation
// (the reference's sum is in T), operands addressed by (row, column) strides
// so that both layouts share it.
#include <algorithm>
#include <vector>

#include "dense.cuh"

namespace tsr {

namespace {

struct GemmView {
  const float* a;  // op A (m x k): a[m * a_rs + k * a_cs]
  int64_t a_rs, a_cs;
  const float* b;  // op B (k x n): b[k * b_rs + n * b_cs] (+ batch * b_bs)
  int64_t b_rs, b_cs, b_bs;
  float* c;        // C (m x n): c[m * c_rs + n] (+ batch * c_bs)
  int64_t c_rs, c_bs;
  int64_t M, N, K;
  int64_t batch;
};

constexpr int TT_BM = 64, TT_BN = 64, TT_BK = 16;

__global__ void __launch_bounds__(256) ttm_gemm_kernel(GemmView g) {
  __shared__ float As[TT_BK][TT_BM + 4];
  __shared__ float Bs[TT_BK][TT_BN + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t m0 = (int64_t)blockIdx.y * TT_BM, n0 = (int64_t)blockIdx.x * TT_BN;
  for (int64_t z = blockIdx.z; z < g.batch; z += gridDim.z) {
  const float* bz = g.b + z * g.b_bs;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
  for (int64_t k0 = 0; k0 < g.K; k0 += TT_BK) {
    // A tile (BM x BK) and B tile (BK x BN): 1024 elements each, 4 per
    // thread; the thread index runs along the operand's contiguous side
    for (int e = threadIdx.x; e < TT_BM * TT_BK; e += 256) {
      int r, c;
      if (g.a_cs == 1) {
        r = e / TT_BK;
        c = e % TT_BK;
      } else {
        r = e % TT_BM;
        c = e / TT_BM;
      }
      const int64_t m = m0 + r, k = k0 + c;
      As[c][r] = (m < g.M && k < g.K) ? __ldg(g.a + m * g.a_rs + k * g.a_cs) : 0.f;
    }
    for (int e = threadIdx.x; e < TT_BK * TT_BN; e += 256) {
      int r, c;
      if (g.b_cs == 1) {
        r = e / TT_BN;
        c = e % TT_BN;
      } else {
        r = e % TT_BK;
        c = e / TT_BK;
      }
      const int64_t k = k0 + r, n = n0 + c;
      Bs[r][c] = (k < g.K && n < g.N) ? __ldg(bz + k * g.b_rs + n * g.b_cs) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TT_BK; ++kk) {
      float av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    __syncthreads();
  }
  float* cz = g.c + z * g.c_bs;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t m = m0 + ty + 16 * i;
    if (m >= g.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t n = n0 + tx + 16 * j;
      if (n < g.N) cz[m * g.c_rs + n] = acc[i][j];
    }
  }
  }
}

}  // namespace

// Y = X x_mode M on device buffers (X: shape, row-major; M: J x shape[mode],
// row-major; Y: shape with shape[mode] -> J).
int launch_ttm(tsr_ctx* ctx, cudaStream_t s, const float* X, int ndim, const int64_t* shape,
               const float* Mat, int64_t J, int mode, float* Y) {
  int64_t A = 1, B = 1;
  for (int m = 0; m < mode; ++m) A *= shape[m];
  for (int m = mode + 1; m < ndim; ++m) B *= shape[m];
  const int64_t I = shape[mode];
  if (A * B * J == 0) return TSR_OK;
  GemmView g;
  int64_t batch;
  if (B > 1) {
    // C_a (J x B) = M (J x I) . X_a (I x B)
    g.a = Mat;
    g.a_rs = I;
    g.a_cs = 1;
    g.b = X;
    g.b_rs = B;
    g.b_cs = 1;
    g.b_bs = I * B;
    g.c = Y;
    g.c_rs = B;
    g.c_bs = J * B;
    g.M = J;
    g.N = B;
    g.K = I;
    batch = A;
  } else {
    // Y (A x J) = X (A x I) . M^T
    g.a = X;
    g.a_rs = I;
    g.a_cs = 1;
    g.b = Mat;
    g.b_rs = 1;
    g.b_cs = I;
    g.b_bs = 0;
    g.c = Y;
    g.c_rs = J;
    g.c_bs = 0;
    g.M = A;
    g.N = J;
    g.K = I;
    batch = 1;
  }
  g.batch = batch;
  dim3 grid((unsigned)ceil_div(g.N, TT_BN), (unsigned)ceil_div(g.M, TT_BM),
            (unsigned)std::min<int64_t>(batch, 65535));
  if (grid.y > 65535u) return fail(TSR_E_UNSUPPORTED, "output too tall for one launch");
  ttm_gemm_kernel<<<grid, 256, 0, s>>>(g);
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

namespace {

// nmode.rs:86-101 (same messages).
int check_ttm(int ndim, const int64_t* shape, int64_t rows, int64_t cols, int mode) {
  if (mode < 0 || mode >= ndim)
    return fail(TSR_E_MODE_OOB, "Mode %d out of bounds for tensor with rank %d", mode, ndim);
  if (cols != shape[mode])
    return fail(TSR_E_COLS_MISMATCH, "Matrix columns (%lld) must match tensor mode-%d size (%lld)",
                (long long)cols, mode, (long long)shape[mode]);
  if (rows < 0) return fail(TSR_E_INVALID_ARG, "negative matrix row count");
  return TSR_OK;
}

// Apply a chain of n-mode products in the given order on the device:
// the result lands in a context slot; its shape in out_shape.
int ttm_chain(tsr_ctx* ctx, const float* dX, int ndim, const int64_t* shape, int n,
              const int* modes, const float* const* mats_host, const int64_t* rows,
              float** d_result, int64_t* out_shape) {
  cudaStream_t s = ctx->stream;
  std::vector<int64_t> cur(shape, shape + ndim);
  int64_t cap = numel(ndim, shape);
  for (int t = 0; t < n; ++t) {
    cur[modes[t]] = rows[t];
    cap = std::max<int64_t>(cap, numel(ndim, cur.data()));
  }
  std::copy(shape, shape + ndim, cur.begin());
  int64_t mtotal = 0;
  for (int t = 0; t < n; ++t) {
    mtotal += rows[t] * cur[modes[t]];
    cur[modes[t]] = rows[t];
  }
  std::copy(shape, shape + ndim, cur.begin());
  void *p0, *p1, *pm;
  TSR_TRY(slot_get(ctx, SLOT_MISC0, sizeof(float) * std::max<int64_t>(cap, 1), &p0));
  TSR_TRY(slot_get(ctx, SLOT_MISC1, sizeof(float) * std::max<int64_t>(cap, 1), &p1));
  TSR_TRY(slot_get(ctx, SLOT_MISC3, sizeof(float) * std::max<int64_t>(mtotal, 1), &pm));
  const float* src = dX;
  float* bufs[2] = {(float*)p0, (float*)p1};
  int which = 0;
  int64_t moff = 0;
  // each matrix's columns equal the mode size at the time it is applied
  // (a mode appears once in a map; an ordered list may repeat a mode)
  for (int t = 0; t < n; ++t) {
    const int64_t cols = cur[modes[t]];
    float* dm = (float*)pm + moff;
    TSR_CUDA(cudaMemcpyAsync(dm, mats_host[t], sizeof(float) * rows[t] * cols,
                             cudaMemcpyHostToDevice, s));
    moff += rows[t] * cols;
    float* dst = bufs[which];
    TSR_TRY(launch_ttm(ctx, s, src, ndim, cur.data(), dm, rows[t], modes[t], dst));
    cur[modes[t]] = rows[t];
    src = dst;
    which ^= 1;
  }
  if (n == 0) {
    TSR_CUDA(cudaMemcpyAsync(bufs[0], dX, sizeof(float) * numel(ndim, shape),
                             cudaMemcpyDeviceToDevice, s));
    src = bufs[0];
  }
  std::copy(cur.begin(), cur.end(), out_shape);
  *d_result = const_cast<float*>(src);
  return TSR_OK;
}

}  // namespace

}  // namespace tsr

using namespace tsr;

extern "C" {

int tsr_nmode_product_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim, const int64_t* shape,
                              const float* d_matrix, int64_t rows, int64_t cols, int mode,
                              float* d_out) {
  if (!shape || !d_tensor || !d_matrix || !d_out) return fail(TSR_E_INVALID_ARG, "null argument");
  if (ndim < 1 || ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d outside 1..%d", ndim, kMaxModes);
  TSR_TRY(check_sizes(ndim, shape, 1));
  TSR_TRY(check_ttm(ndim, shape, rows, cols, mode));
  TSR_TRY(check_ctx(ctx));
  return launch_ttm(ctx, ctx->stream, d_tensor, ndim, shape, d_matrix, rows, mode, d_out);
}

// nmode_product (nmode.rs:72-131) with host buffers: out has shape with
// shape[mode] replaced by rows.
int tsr_nmode_product_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                          const float* matrix, int64_t rows, int64_t cols, int mode, float* out) {
  if (!shape || !tensor || !matrix || !out) return fail(TSR_E_INVALID_ARG, "null argument");
  if (ndim < 1 || ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d outside 1..%d", ndim, kMaxModes);
  TSR_TRY(check_sizes(ndim, shape, 1));
  TSR_TRY(check_ttm(ndim, shape, rows, cols, mode));
  TSR_TRY(check_ctx(ctx));
  float* dX;
  TSR_TRY(upload_tensor(ctx, tensor, ndim, shape, nullptr, &dX));
  const float* mats[1] = {matrix};
  const int modes[1] = {mode};
  float* dY;
  int64_t oshape[kMaxModes];
  TSR_TRY(ttm_chain(ctx, dX, ndim, shape, 1, modes, mats, &rows, &dY, oshape));
  TSR_CUDA(cudaMemcpyAsync(out, dY, sizeof(float) * numel(ndim, oshape), cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

// n-mode products applied in the given order (nmode_products_seq,
// nmode.rs:241-254, and tucker_operator_ordered, :517-531): modes[t] and the
// rows[t] x cols[t] matrix mats[t]; cols[t] must equal that mode's size at
// step t. out_shape receives the result's shape; out (host) its values, or
// only the shape when out is NULL.
int tsr_nmode_products_seq_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                               int n, const int* modes, const float* const* mats,
                               const int64_t* rows, const int64_t* cols, float* out,
                               int64_t* out_shape) {
  if (!shape || !tensor || !out_shape || (n > 0 && (!modes || !mats || !rows || !cols)))
    return fail(TSR_E_INVALID_ARG, "null argument");
  if (ndim < 1 || ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d outside 1..%d", ndim, kMaxModes);
  TSR_TRY(check_sizes(ndim, shape, 1));
  std::vector<int64_t> cur(shape, shape + ndim);
  for (int t = 0; t < n; ++t) {
    TSR_TRY(check_ttm(ndim, cur.data(), rows[t], cols[t], modes[t]));
    cur[modes[t]] = rows[t];
  }
  std::copy(cur.begin(), cur.end(), out_shape);
  if (!out) return TSR_OK;
  TSR_TRY(check_ctx(ctx));
  float* dX;
  TSR_TRY(upload_tensor(ctx, tensor, ndim, shape, nullptr, &dX));
  float* dY;
  int64_t oshape[kMaxModes];
  TSR_TRY(ttm_chain(ctx, dX, ndim, shape, n, modes, mats, rows, &dY, oshape));
  TSR_CUDA(cudaMemcpyAsync(out, dY, sizeof(float) * numel(ndim, oshape), cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

// tucker_operator (nmode.rs:442-480): the products of a mode -> matrix map,
// applied in ascending order of rows / mode size (ties by mode index; the
// reference iterates a HashMap there, so its tie order is unspecified). Each
// mode may appear once; cols[t] must equal shape[modes[t]].
int tsr_tucker_operator_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                            int n, const int* modes, const float* const* mats,
                            const int64_t* rows, const int64_t* cols, float* out,
                            int64_t* out_shape) {
  if (!shape || !out_shape || (n > 0 && (!modes || !mats || !rows || !cols)))
    return fail(TSR_E_INVALID_ARG, "null argument");
  if (ndim < 1 || ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d outside 1..%d", ndim, kMaxModes);
  for (int t = 0; t < n; ++t)
    if (modes[t] < 0 || modes[t] >= ndim)
      return fail(TSR_E_MODE_OOB, "Mode %d out of bounds for tensor with rank %d", modes[t],
                  ndim);
  for (int t = 0; t < n; ++t)
    for (int u = 0; u < t; ++u)
      if (modes[u] == modes[t])
        return fail(TSR_E_INVALID_ARG, "mode %d appears twice in the factor map", modes[t]);
  std::vector<int> ord(n);
  for (int t = 0; t < n; ++t) ord[t] = t;
  std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
    const double rx = (double)rows[x] / (double)shape[modes[x]];
    const double ry = (double)rows[y] / (double)shape[modes[y]];
    return rx != ry ? rx < ry : modes[x] < modes[y];
  });
  std::vector<int> m2(n);
  std::vector<const float*> p2(n);
  std::vector<int64_t> r2(n), c2(n);
  for (int t = 0; t < n; ++t) {
    m2[t] = modes[ord[t]];
    p2[t] = mats[ord[t]];
    r2[t] = rows[ord[t]];
    c2[t] = cols[ord[t]];
  }
  return tsr_nmode_products_seq_f32(ctx, tensor, ndim, shape, n, m2.data(), p2.data(), r2.data(),
                                    c2.data(), out, out_shape);
}

// tucker_reconstruct (nmode.rs:576-611): core x_0 U_0 ... x_{N-1} U_{N-1}
// through tucker_operator; factor m is rows[m] x cols[m] with cols[m] equal
// to the core's mode-m size (same messages as the reference).
int tsr_tucker_reconstruct_f32(tsr_ctx* ctx, const float* core, int ndim,
                               const int64_t* core_shape, int n_factors,
                               const float* const* factors, const int64_t* rows,
                               const int64_t* cols, float* out, int64_t* out_shape) {
  if (!core_shape || !out_shape || (n_factors > 0 && (!factors || !rows || !cols)))
    return fail(TSR_E_INVALID_ARG, "null argument");
  if (n_factors != ndim)
    return fail(TSR_E_NFACTORS, "Number of factor matrices (%d) must match core rank (%d)",
                n_factors, ndim);
  for (int m = 0; m < ndim; ++m)
    if (cols[m] != core_shape[m])
      return fail(TSR_E_RANK_MISMATCH,
                  "Factor matrix %d has %lld columns, expected %lld (core mode-%d size)", m,
                  (long long)cols[m], (long long)core_shape[m], m);
  std::vector<int> modes(ndim);
  for (int m = 0; m < ndim; ++m) modes[m] = m;
  return tsr_tucker_operator_f32(ctx, core, ndim, core_shape, ndim, modes.data(), factors, rows,
                                 cols, out, out_shape);
}

}  // extern "C"

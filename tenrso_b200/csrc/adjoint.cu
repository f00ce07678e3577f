// CP reconstruction, its adjoint, and the loss/gradient of a CP model.
//
//   tenrso_kernels::cp_reconstruct                  crates/tenrso-kernels/src/outer.rs:223-274
//     Xhat = sum_r w_r U_0[:, r] o U_1[:, r] o ... o U_{N-1}[:, r]
//   CpReconstructionGrad::compute_factor_gradients  crates/tenrso-ad/src/grad.rs:81-120
//     dL/dU_n = unfold(G, n) . KR_{m != n}(U_m) . diag(w),  G = dL/dXhat
//   that is, the MTTKRP of G; the Khatri-Rao rows are formed on the fly by the
//   MTTKRP kernels and never stored (grad.rs:128-150 materialises them).
//
// The loss/gradient entry evaluates  L = ||X - [[U]]||^2 + reg * sum_n ||U_n||^2
// and all dL/dU_n without forming Xhat, from the Gram identities
//   ||Xhat||^2   = sum_{r,s} prod_n (U_n^T U_n)[r, s]
//   <X, Xhat>    = sum_{i,r} MTTKRP(X, 0)[i, r] U_0[i, r]
//   dL/dU_n      = 2 (U_n H_n - MTTKRP(X, n)) + 2 reg U_n,  H_n = *_{m != n} U_m^T U_m
// with the Grams, H_n, the loss and the U_n H_n product in FP64.
#include <cstring>

#include "als.cuh"
#include "dense.cuh"

// A dense tensor prepared for repeated MTTKRPs: its per-mode unfoldings (in
// the precision the MTTKRP reads) are built once and kept in HBM. The tensor
// itself stays the caller's and must not change while the object is in use.
struct tsr_dense {
  int ndim = 0;
  int64_t shape[tsr::kMaxModes] = {};
  int precision = 0;
  int device = 0;
  const float* dX = nullptr;
  void* owned[2 * tsr::kMaxModes + 4] = {};
  tsr::ModeOperand ops[tsr::kMaxModes];
  double* d_scalars = nullptr;  // [0] ||X||^2, [1] <X, Xhat>, [2] loss, [3] scratch
  // BF16x3 tensors of 3 or more modes whose trailing-two-modes view
  // (prod of the leading modes, I_{N-2}, I_{N-1}) suits the two-sided
  // contraction or the single-layout 3-way MTTKRP: X's bf16 halves in its own
  // layout (owned[2N], owned[2N+1])
  bool d3_on = false;
  bool d3_three = false;  // the view suits the single-layout 3-way MTTKRP
  bool d3_two = false;    // the view suits the two-sided contraction
  tsr::Dense3 d3{};
  // FP32 tensors of 3 or more modes: T and P as mode-0 MTTKRPs. vops[0] is X
  // as the 3-way tensor (A, I_{N-2}, I_{N-1}) (X itself, or a padded copy);
  // vops[1] is X's transpose (C x A, C = I_{N-2} I_{N-1}) as the tensor
  // (C, I_0, .., I_{N-3}). Buffers in owned[2N + 2], owned[2N + 3].
  bool v2_on = false;
  int64_t v2_shape[2] = {0, 0};
  tsr::ModeOperand vops[2];
};

namespace tsr {

namespace {

constexpr int RC_THREADS = 256;
constexpr int RC_TILE = 64;   // output tile: 64 rows x 64 columns, 4 x 4 per thread
constexpr int RC_CHUNK = 32;  // rank columns staged in shared memory per pass

// The row-major output seen as a P x Lc matrix: rows run over modes
// [0, split), columns over the trailing modes [split, N) (the last fastest),
// so element (p, c) sits at p * Lc + c. Both operands of the tile product are
// Khatri-Rao rows built from the factors inside the kernel.
struct ReconArgs {
  FactorTable ft;
  int ndim;
  int split;
  int R;
  int64_t P, Lc;
  const float* w;    // weights (R) or null for all ones
  const float* X;    // residual mode: the target tensor
  float* out;        // Xhat, or alpha * (Xhat - X)
  float alpha;
  double* sq_err;    // residual mode: sum of (Xhat - X)^2 added here
};

// Offsets (element index * R) of one KR row's factor entries, modes [m0, m1).
__device__ __forceinline__ void kr_offsets(const ReconArgs& a, int m0, int m1, int64_t idx,
                                           int64_t* off) {
  for (int m = m1 - 1; m >= m0; --m) {
    const int64_t n = a.ft.rows[m];
    const int64_t q = idx / n;
    off[m] = (idx - q * n) * a.R;
    idx = q;
  }
}

template <bool RESIDUAL, bool VEC4>
__global__ void __launch_bounds__(RC_THREADS)
reconstruct_kernel(ReconArgs a) {
  __shared__ __align__(16) float Ws[RC_CHUNK][RC_TILE];  // row operand, rank-major
  __shared__ __align__(16) float Vs[RC_CHUNK][RC_TILE];  // column operand, rank-major
  __shared__ int64_t row_off[kMaxModes][RC_TILE];
  __shared__ int64_t col_off[kMaxModes][RC_TILE];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t p0 = (int64_t)blockIdx.y * RC_TILE;
  const int64_t c0 = (int64_t)blockIdx.x * RC_TILE;
  if (threadIdx.x < RC_TILE) {
    int64_t off[kMaxModes];
    const int64_t p = p0 + threadIdx.x;
    kr_offsets(a, 0, a.split, p < a.P ? p : 0, off);
    for (int m = 0; m < a.split; ++m) row_off[m][threadIdx.x] = off[m];
  } else if (threadIdx.x < 2 * RC_TILE) {
    int64_t off[kMaxModes];
    const int64_t c = c0 + threadIdx.x - RC_TILE;
    kr_offsets(a, a.split, a.ndim, c < a.Lc ? c : 0, off);
    for (int m = a.split; m < a.ndim; ++m) col_off[m][threadIdx.x - RC_TILE] = off[m];
  }
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
  for (int r0 = 0; r0 < a.R; r0 += RC_CHUNK) {
    __syncthreads();
    // stage KR entries: thread e covers (row/col i, rank r) with r fastest
    for (int e = threadIdx.x; e < RC_TILE * RC_CHUNK; e += RC_THREADS) {
      const int i = e / RC_CHUNK, r = e % RC_CHUNK;
      const int rr = r0 + r;
      float wv = 0.f, vv = 0.f;
      if (rr < a.R) {
        wv = (p0 + i < a.P) ? (a.w ? __ldg(a.w + rr) : 1.f) : 0.f;
        for (int m = 0; m < a.split; ++m) wv *= __ldg(a.ft.ptr[m] + row_off[m][i] + rr);
        vv = (c0 + i < a.Lc) ? 1.f : 0.f;
        for (int m = a.split; m < a.ndim; ++m) vv *= __ldg(a.ft.ptr[m] + col_off[m][i] + rr);
      }
      Ws[r][i] = wv;
      Vs[r][i] = vv;
    }
    __syncthreads();
    const int rn = a.R - r0 < RC_CHUNK ? a.R - r0 : RC_CHUNK;
#pragma unroll 8
    for (int r = 0; r < rn; ++r) {
      const float4 wv = *reinterpret_cast<const float4*>(&Ws[r][ty * 4]);
      const float4 vv = *reinterpret_cast<const float4*>(&Vs[r][tx * 4]);
      const float wa[4] = {wv.x, wv.y, wv.z, wv.w};
      const float va[4] = {vv.x, vv.y, vv.z, vv.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(wa[i], va[j], acc[i][j]);
    }
  }
  double sq = 0.0;
  const int64_t c = c0 + tx * 4;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t p = p0 + ty * 4 + i;
    if (p >= a.P) continue;
    const int64_t base = p * a.Lc + c;
    if (VEC4 && c + 3 < a.Lc) {
      float4 v = make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
      if (RESIDUAL) {
        const float4 x = __ldg(reinterpret_cast<const float4*>(a.X + base));
        const float d0 = v.x - x.x, d1 = v.y - x.y, d2 = v.z - x.z, d3 = v.w - x.w;
        sq += (double)d0 * d0 + (double)d1 * d1 + (double)d2 * d2 + (double)d3 * d3;
        v = make_float4(a.alpha * d0, a.alpha * d1, a.alpha * d2, a.alpha * d3);
      }
      __stcs(reinterpret_cast<float4*>(a.out + base), v);
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (c + j >= a.Lc) break;
        float v = acc[i][j];
        if (RESIDUAL) {
          const float d = v - __ldg(a.X + base + j);
          sq += (double)d * d;
          v = a.alpha * d;
        }
        a.out[base + j] = v;
      }
    }
  }
  if (RESIDUAL) {
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(a.sq_err, sq);
  }
}

__device__ __forceinline__ double sym_at(const double* g, int R, int a, int c) {
  return a <= c ? g[a * R + c] : g[c * R + a];
}

// Gradient rows of one mode in Gram form:
//   out[i, :] = 2 (U[i, :] H - M[i, :] + reg U[i, :]),  H = *_{m != mode} Gram_m
// where M is the sum of the split MTTKRP partials. Mode 0 also accumulates
// <M, U> (= <X, Xhat>) into scal[1]. Shared (FP64): H (R x R), M (rows x R),
// and the per-group partial sums: `groups` threads share one element of M and
// each sums a strided subset of the splits with 8 loads in flight.
__device__ __forceinline__ void gram_grad_block(
    const double* __restrict__ grams, int ndim, int mode, const float* __restrict__ partials,
    int splits, int64_t rows, int R, int rows_per_cta, const float* __restrict__ U, double reg,
    float* __restrict__ out, double* scal, int64_t blk, double* sh) {
  const int RR = R * R;
  double* H = sh;
  double* Ms = sh + RR;
  for (int e = threadIdx.x; e < RR; e += blockDim.x) {
    const int a = e / R, c = e % R;
    double h = 1.0;
    for (int m = 0; m < ndim; ++m)
      if (m != mode) h *= sym_at(grams + (int64_t)m * RR, R, a, c);
    H[e] = h;
  }
  const int64_t r0 = blk * rows_per_cta;
  const int nr = (int)(rows - r0 < rows_per_cta ? rows - r0 : rows_per_cta);
  const int64_t pstride = rows * R;
  const int ne = nr * R;
  const int full = rows_per_cta * R;
  const int groups = full >= (int)blockDim.x ? 1 : (int)blockDim.x / full;
  double* red = Ms + full;  // [groups][ne]
  for (int t = threadIdx.x; t < ne * groups; t += blockDim.x) {
    const int e = t % ne, g = t / ne;
    const float* p = partials + r0 * R + e;
    double s = 0.0;
    int q = g;
    for (; q + 7 * groups < splits; q += 8 * groups) {
      float v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = __ldg(p + (int64_t)(q + u * groups) * pstride);
#pragma unroll
      for (int u = 0; u < 8; ++u) s += (double)v[u];
    }
    for (; q < splits; q += groups) s += (double)__ldg(p + (int64_t)q * pstride);
    red[g * ne + e] = s;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    double s = 0.0;
    for (int g = 0; g < groups; ++g) s += red[g * ne + e];
    Ms[e] = s;
  }
  __syncthreads();
  double ip = 0.0;
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    const int i = e / R, c = e % R;
    const float* urow = U + (r0 + i) * R;
    double s0 = 0.0, s1 = 0.0;
    int k = 0;
    for (; k + 2 <= R; k += 2) {
      s0 += (double)__ldg(urow + k) * H[k * R + c];
      s1 += (double)__ldg(urow + k + 1) * H[(k + 1) * R + c];
    }
    if (k < R) s0 += (double)__ldg(urow + k) * H[k * R + c];
    const double u = (double)__ldg(urow + c);
    out[(r0 + i) * R + c] = (float)(2.0 * ((s0 + s1) - Ms[e] + reg * u));
    ip += Ms[e] * u;
  }
  if (mode == 0) {
    for (int o = 16; o > 0; o >>= 1) ip += __shfl_down_sync(0xffffffffu, ip, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(scal + 1, ip);
  }
}

__global__ void __launch_bounds__(256)
gram_grad_kernel(const double* __restrict__ grams, int ndim, int mode,
                 const float* __restrict__ partials, int splits, int64_t rows, int R,
                 int rows_per_cta, const float* __restrict__ U, double reg,
                 float* __restrict__ out, double* scal) {
  extern __shared__ double sh[];
  gram_grad_block(grams, ndim, mode, partials, splits, rows, R, rows_per_cta, U, reg, out, scal,
                  blockIdx.x, sh);
}

// sum_{r,s} prod_n Gram_n[r, s] + reg sum_n tr(Gram_n) over one CTA of
// `blockDim.x` threads (a multiple of 32), valid in thread 0
__device__ __forceinline__ double gram_loss_part(const double* __restrict__ grams, int ndim, int R,
                                                 double reg) {
  const int RR = R * R;
  double s = 0.0;
  for (int e = threadIdx.x; e < RR; e += blockDim.x) {
    const int a = e / R, c = e % R;
    double h = 1.0, tr = 0.0;
    for (int m = 0; m < ndim; ++m) {
      const double g = sym_at(grams + (int64_t)m * RR, R, a, c);
      h *= g;
      if (a == c) tr += g;
    }
    s += h + reg * tr;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
  return t;
}

// The Grams of every mode in one launch (pre-zeroed): block b is block
// b - cta0[m] of mode m, rpc[m] rows each.
struct GramAll {
  const float* U[kMaxModes];
  int64_t rows[kMaxModes];
  int64_t rpc[kMaxModes];
  int cta0[kMaxModes + 1];
  int ndim, R;
  double* grams;
};

template <int RB>
__global__ void __launch_bounds__(256) gram_all_kernel(const __grid_constant__ GramAll g) {
  __shared__ double Us[kGramChunk * 16 * RB];
  const int b = blockIdx.x;
  int m = 0;
  while (m + 1 < g.ndim && b >= g.cta0[m + 1]) ++m;
  const int64_t r0 = (int64_t)(b - g.cta0[m]) * g.rpc[m];
  const int64_t r1 = g.rows[m] < r0 + g.rpc[m] ? g.rows[m] : r0 + g.rpc[m];
  gram_rows_accumulate<RB>(g.U[m], r0, r1, g.R, g.grams + (int64_t)m * g.R * g.R, Us);
}

// loss = ||X||^2 - 2 <X, Xhat> + sum_{r,s} prod_n Gram_n[r, s] + reg sum_n tr(Gram_n)
__global__ void gram_loss_kernel(const double* __restrict__ grams, int ndim, int R, double reg,
                                 double* scal) {
  const double t = gram_loss_part(grams, ndim, R, reg);
  if (threadIdx.x == 0) scal[2] = scal[0] - 2.0 * scal[1] + t;
}

// MTTKRPs from a partial contraction. A side holds S (rows a over nlead
// modes, row-major, fewer than 2^31 rows) with
//   S[a, r] = sum over the other modes of X[a, ...] prod_{other p} U_p[., r],
// and the mode-m MTTKRP of one of its modes is
//   M_m[i, r] = sum_{a : a_m = i} S[a, r] prod_{p in side, p != m} U_p[a_p, r].
// The leading modes 0..N-3 come from T (S over the leading modes, the
// trailing two contracted), the trailing two from P (S over (I_{N-2},
// I_{N-1}), the leading modes contracted). One launch for every requested
// mode: block b is row i of mode n (the modes' rows stacked in `out`), lane r
// of a group of R threads, the groups split the side's other indices; FP64
// sums, fp32 output.
struct TSideC {
  const float* S;
  int nlead;
  int arows;
  int size[kMaxModes];
  int stride[kMaxModes];
  const float* U[kMaxModes];
};

struct TContract {
  TSideC side[2];
  int R, nmodes;
  int side_of[kMaxModes];  // output mode -> side
  int pos[kMaxModes];      // output mode -> its index within the side
  int row0[kMaxModes + 1];
  float* out;
};

// Thread (g, r)'s share of M_m[i, r]: groups g < groups split the side's
// other indices (FP64).
__device__ __forceinline__ double t_contract_part(const TSideC& sd, int m, int i, int R, int g,
                                                  int groups, int r) {
  double s = 0.0;
  if (g >= groups) return s;
  if (sd.nlead == 2) {
    // the other mode's index is the loop index: four independent loads per step
    const int o = 1 - m;
    const int cnt = sd.size[o], so = sd.stride[o];
    const float* Sp = sd.S + (int64_t)i * sd.stride[m] * R + r;
    const float* Uo = sd.U[o] + r;
    int q = g;
    for (; q + 3 * groups < cnt; q += 4 * groups) {
      float sv[4], wv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        sv[u] = __ldg(Sp + (int64_t)(q + u * groups) * so * R);
        wv[u] = __ldg(Uo + (int64_t)(q + u * groups) * R);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) s += (double)sv[u] * (double)wv[u];
    }
    for (; q < cnt; q += groups)
      s += (double)__ldg(Sp + (int64_t)q * so * R) * (double)__ldg(Uo + (int64_t)q * R);
    return s;
  }
  const int count = sd.arows / sd.size[m];
  for (int q = g; q < count; q += groups) {
    int rem = q, a = i * sd.stride[m];
    double w = 1.0;
    for (int p = sd.nlead - 1; p >= 0; --p) {
      if (p == m) continue;
      const int ip = rem % sd.size[p];
      rem /= sd.size[p];
      a += ip * sd.stride[p];
      w *= (double)__ldg(sd.U[p] + (int64_t)ip * R + r);
    }
    s += (double)__ldg(sd.S + (int64_t)a * R + r) * w;
  }
  return s;
}

__global__ void __launch_bounds__(256) t_contract_kernel(const __grid_constant__ TContract c) {
  __shared__ double part[256];
  const int b = blockIdx.x;
  int n = 0;
  while (n + 1 < c.nmodes && b >= c.row0[n + 1]) ++n;
  const int R = c.R;
  const int groups = blockDim.x / R;
  part[threadIdx.x] = t_contract_part(c.side[c.side_of[n]], c.pos[n], b - c.row0[n], R,
                                      threadIdx.x / R, groups, threadIdx.x % R);
  __syncthreads();
  if (threadIdx.x < R) {
    double t = 0.0;
    for (int q = 0; q < groups; ++q) t += part[q * R + threadIdx.x];
    c.out[(int64_t)b * R + threadIdx.x] = (float)t;
  }
}

// The same contraction with the gradient row formed in place (R <= 32): block
// b is row i of mode n; with M_n[i, :] reduced in shared memory,
//   grad[i, c] = 2 (sum_k U_n[i, k] H_n[k, c] - M_n[i, c] + reg U_n[i, c]),
// H_n = *_{m != n} Gram_m formed by the block (FP64, the Grams stay in L1).
// Mode-0 rows add <M_0, U_0> (= <X, Xhat>) into scal[1]; the extra last
// block writes the Gram part of the loss into scal[3].
struct GradArgs {
  const double* grams;
  int ndim;
  double reg;
  float* G[kMaxModes];
  double* scal;
};

__global__ void __launch_bounds__(256)
t_contract_grad_kernel(const __grid_constant__ TContract c, const __grid_constant__ GradArgs ga) {
  __shared__ double part[256];
  __shared__ double H[32 * 32];
  __shared__ double Mrow[32];
  // programmatic launch: T, P and, through the earlier kernels' own waits,
  // the Grams are complete once the predecessor is
  grid_dep_wait();
  const int b = blockIdx.x;
  const int R = c.R;
  if (b >= c.row0[c.nmodes]) {
    const double t = gram_loss_part(ga.grams, ga.ndim, R, ga.reg);
    if (threadIdx.x == 0) ga.scal[3] = t;
    return;
  }
  int n = 0;
  while (n + 1 < c.nmodes && b >= c.row0[n + 1]) ++n;
  const TSideC& sd = c.side[c.side_of[n]];
  const int m = c.pos[n], i = b - c.row0[n];
  const int groups = blockDim.x / R;
  part[threadIdx.x] = t_contract_part(sd, m, i, R, threadIdx.x / R, groups, threadIdx.x % R);
  const int RR = R * R;
  for (int e = threadIdx.x; e < RR; e += blockDim.x) {
    const int a = e / R, cc = e % R;
    double h = 1.0;
    for (int q = 0; q < ga.ndim; ++q)
      if (q != n) h *= sym_at(ga.grams + (int64_t)q * RR, R, a, cc);
    H[e] = h;
  }
  __syncthreads();
  if (threadIdx.x < R) {
    double t = 0.0;
    for (int q = 0; q < groups; ++q) t += part[q * R + threadIdx.x];
    Mrow[threadIdx.x] = t;
  }
  __syncthreads();
  if (threadIdx.x < 32) {  // R <= 32: one warp
    const int cc = threadIdx.x;
    double ip = 0.0;
    if (cc < R) {
      const float* urow = sd.U[m] + (int64_t)i * R;
      double s0 = 0.0, s1 = 0.0;
      int k = 0;
      for (; k + 2 <= R; k += 2) {
        s0 += (double)__ldg(urow + k) * H[k * R + cc];
        s1 += (double)__ldg(urow + k + 1) * H[(k + 1) * R + cc];
      }
      if (k < R) s0 += (double)__ldg(urow + k) * H[k * R + cc];
      const double u = (double)__ldg(urow + cc);
      ga.G[n][(int64_t)i * R + cc] = (float)(2.0 * ((s0 + s1) - Mrow[cc] + ga.reg * u));
      ip = Mrow[cc] * u;
    }
    if (n == 0) {
      for (int o = 16; o > 0; o >>= 1) ip += __shfl_down_sync(0xffffffffu, ip, o);
      if (cc == 0) atomicAdd(ga.scal + 1, ip);
    }
  }
}

// side k of c over modes m0 .. m1-1 of the tensor, the partial contraction S
void set_side(TContract& c, int k, const float* S, const int64_t* shape, int m0, int m1,
              const float* const* U) {
  TSideC& sd = c.side[k];
  sd.S = S;
  sd.nlead = m1 - m0;
  int st = 1;
  for (int p = m1 - 1; p >= m0; --p) {
    sd.size[p - m0] = (int)shape[p];
    sd.stride[p - m0] = st;
    sd.U[p - m0] = U[p];
    st *= (int)shape[p];
  }
  sd.arows = st;
}

int64_t prod_range(const int64_t* shape, int m0, int m1) {
  int64_t p = 1;
  for (int m = m0; m < m1; ++m) p *= shape[m];
  return p;
}

// Shared validation of tenrso's cp_reconstruct (outer.rs:231-255).
int validate_reconstruct(int n_factors, const int64_t* fcols, int64_t n_weights, bool has_w) {
  if (n_factors <= 0)
    return fail(TSR_E_SHAPE, "Need at least one factor matrix for CP reconstruction");
  const int64_t R = fcols[0];
  for (int i = 0; i < n_factors; ++i)
    if (fcols[i] != R)
      return fail(TSR_E_RANK_MISMATCH, "Factor %d has %lld columns, expected %lld", i,
                  (long long)fcols[i], (long long)R);
  if (has_w && n_weights != R)
    return fail(TSR_E_SHAPE, "Weights length %lld must match rank %lld", (long long)n_weights,
                (long long)R);
  if (n_factors > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d exceeds the supported %d", n_factors,
                kMaxModes);
  return TSR_OK;
}

}  // namespace

void init_adjoint_attributes() {
  cudaFuncSetAttribute(gram_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

// Xhat (or alpha * (Xhat - X) with sum of squares) on the context's stream.
int launch_reconstruct(tsr_ctx* ctx, const FactorTable& ft, int ndim, int R, const float* w,
                       const float* X, float alpha, double* sq_err, float* out) {
  ReconArgs a;
  std::memset(&a, 0, sizeof(a));
  a.ft = ft;
  a.ndim = ndim;
  a.R = R;
  a.w = w;
  a.X = X;
  a.out = out;
  a.alpha = alpha;
  a.sq_err = sq_err;
  int64_t shape[kMaxModes];
  for (int m = 0; m < ndim; ++m) shape[m] = ft.rows[m];
  // the fewest trailing modes that fill a 64-wide column tile
  int split = ndim - 1;
  while (split > 0 && prod_range(shape, split, ndim) < RC_TILE) --split;
  if (prod_range(shape, split, ndim) < RC_TILE) split = 0;
  a.split = split;
  a.P = prod_range(shape, 0, split);
  a.Lc = prod_range(shape, split, ndim);
  if (a.P == 0 || a.Lc == 0) return TSR_OK;
  const int64_t gy = ceil_div(a.P, RC_TILE);
  if (gy > 65535) {
    // fold excess rows into columns: keep the grid's y extent legal
    while (split > 0 && ceil_div(prod_range(shape, 0, split), RC_TILE) > 65535) --split;
    a.split = split;
    a.P = prod_range(shape, 0, split);
    a.Lc = prod_range(shape, split, ndim);
  }
  const int64_t gx = ceil_div(a.Lc, RC_TILE);
  if (gx > 0x7fffffffLL)
    return fail(TSR_E_UNSUPPORTED, "tensor too large for the reconstruction kernel");
  const dim3 grid((unsigned)gx, (unsigned)ceil_div(a.P, RC_TILE));
  const bool vec = (a.Lc % 4 == 0) && !((uintptr_t)out & 15) && !((uintptr_t)X & 15);
  if (X) {
    if (vec) reconstruct_kernel<true, true><<<grid, RC_THREADS, 0, ctx->stream>>>(a);
    else reconstruct_kernel<true, false><<<grid, RC_THREADS, 0, ctx->stream>>>(a);
  } else {
    if (vec) reconstruct_kernel<false, true><<<grid, RC_THREADS, 0, ctx->stream>>>(a);
    else reconstruct_kernel<false, false><<<grid, RC_THREADS, 0, ctx->stream>>>(a);
  }
  ctx->launches++;
  TSR_CUDA(cudaGetLastError());
  return TSR_OK;
}

namespace {

// dL/dU_n for every mode of a device gradient tensor G (grad.rs:81-120).
int reconstruction_grad_device(tsr_ctx* ctx, const float* dG, int ndim, const int64_t* shape,
                               const FactorTable& ft, int R, const float* dw, int precision,
                               float* const* d_out) {
  for (int n = 0; n < ndim; ++n) {
    if (shape[n] == 0) continue;
    if (numel(ndim, shape) == 0 || R == 0) {
      TSR_CUDA(cudaMemsetAsync(d_out[n], 0, sizeof(float) * shape[n] * R, ctx->stream));
      continue;
    }
    ModeOperand op;
    TSR_TRY(prepare_mode(ctx, dG, ndim, shape, n, precision, 0, &op));
    float* partials;
    int splits;
    TSR_TRY(run_mttkrp_partials(ctx, op, ft, R, precision, &partials, &splits));
    TSR_TRY(launch_mttkrp_reduce_scaled(ctx, partials, splits, shape[n], R, dw, d_out[n]));
  }
  return TSR_OK;
}

int validate_grad(int g_ndim, const int64_t* shape, int n_factors, const int64_t* frows,
                  const int64_t* fcols) {
  // grad.rs:84-91
  if (g_ndim != n_factors)
    return fail(TSR_E_SHAPE, "Gradient rank %d doesn't match number of factors %d", g_ndim,
                n_factors);
  // grad.rs:137-139: the Khatri-Rao product of the other factors needs one
  if (n_factors < 2)
    return fail(TSR_E_NEED_2_FACTORS, "Need at least one factor for Khatri-Rao product");
  return validate_mttkrp(g_ndim, shape, n_factors, frows, fcols, 0);
}

}  // namespace

}  // namespace tsr

using namespace tsr;

extern "C" {

int tsr_cp_reconstruct_f32(tsr_ctx* ctx, const float* const* factors, int n_factors,
                           const int64_t* factor_rows, const int64_t* factor_cols,
                           const float* weights, int64_t n_weights, float* out) {
  if (n_factors > 0 && (!factors || !factor_rows || !factor_cols))
    return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(validate_reconstruct(n_factors, factor_cols, n_weights, weights != nullptr));
  if (!out) return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(check_ctx(ctx));
  const int64_t R = factor_cols[0];
  const int64_t total = numel(n_factors, factor_rows);
  if (total == 0) return TSR_OK;
  if (R == 0) {
    std::memset(out, 0, sizeof(float) * total);
    return TSR_OK;
  }
  FactorTable ft{};
  TSR_TRY(upload_factors(ctx, n_factors, factor_rows, factors, R, &ft));
  const float* dw = nullptr;
  if (weights) {
    void* p;
    TSR_TRY(slot_get(ctx, SLOT_MISC0, sizeof(float) * R, &p));
    TSR_CUDA(cudaMemcpyAsync(p, weights, sizeof(float) * R, cudaMemcpyHostToDevice, ctx->stream));
    dw = (const float*)p;
  }
  void* dout;
  TSR_TRY(slot_get(ctx, SLOT_OUT, sizeof(float) * total, &dout));
  TSR_TRY(launch_reconstruct(ctx, ft, n_factors, (int)R, dw, nullptr, 0.f, nullptr,
                             (float*)dout));
  TSR_CUDA(cudaMemcpyAsync(out, dout, sizeof(float) * total, cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

int tsr_cp_reconstruct_dev_f32(tsr_ctx* ctx, const float* const* d_factors, int ndim,
                               const int64_t* shape, int64_t rank, const float* d_weights,
                               float* d_out) {
  if (!d_factors || !shape || !d_out) return fail(TSR_E_INVALID_ARG, "null argument");
  std::vector<int64_t> cols(ndim > 0 ? ndim : 1, rank);
  TSR_TRY(validate_reconstruct(ndim, cols.data(), rank, false));
  TSR_TRY(check_ctx(ctx));
  const int64_t total = numel(ndim, shape);
  if (total == 0) return TSR_OK;
  if (rank == 0) {
    TSR_CUDA(cudaMemsetAsync(d_out, 0, sizeof(float) * total, ctx->stream));
    return TSR_OK;
  }
  FactorTable ft{};
  for (int m = 0; m < ndim; ++m) {
    ft.ptr[m] = d_factors[m];
    ft.rows[m] = shape[m];
  }
  return launch_reconstruct(ctx, ft, ndim, (int)rank, d_weights, nullptr, 0.f, nullptr, d_out);
}

int tsr_cp_residual_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim, const int64_t* shape,
                            const float* const* d_factors, int64_t rank, const float* d_weights,
                            float alpha, float* d_out, double* sq_err) {
  if (!d_tensor || !d_factors || !shape || !d_out) return fail(TSR_E_INVALID_ARG, "null argument");
  std::vector<int64_t> cols(ndim > 0 ? ndim : 1, rank);
  TSR_TRY(validate_reconstruct(ndim, cols.data(), rank, false));
  if (rank <= 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  TSR_TRY(check_ctx(ctx));
  void* p;
  TSR_TRY(slot_get(ctx, SLOT_MISC2, sizeof(double), &p));
  TSR_CUDA(cudaMemsetAsync(p, 0, sizeof(double), ctx->stream));
  FactorTable ft{};
  for (int m = 0; m < ndim; ++m) {
    ft.ptr[m] = d_factors[m];
    ft.rows[m] = shape[m];
  }
  TSR_TRY(launch_reconstruct(ctx, ft, ndim, (int)rank, d_weights, d_tensor, alpha, (double*)p,
                             d_out));
  if (sq_err) {
    TSR_CUDA(cudaMemcpyAsync(sq_err, p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return TSR_OK;
}

int tsr_cp_reconstruction_grad_f32(tsr_ctx* ctx, const float* grad_output, int grad_ndim,
                                   const int64_t* shape, const float* const* factors,
                                   int n_factors, const int64_t* factor_rows,
                                   const int64_t* factor_cols, const float* weights,
                                   int64_t n_weights, int precision, float* const* out_grads) {
  if (!shape || !grad_output || !out_grads || (n_factors > 0 && (!factors || !factor_rows ||
                                                                  !factor_cols)))
    return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(validate_grad(grad_ndim, shape, n_factors, factor_rows, factor_cols));
  const int64_t R = factor_cols[0];
  if (weights && n_weights != R)
    return fail(TSR_E_SHAPE, "Weights length %lld must match rank %lld", (long long)n_weights,
                (long long)R);
  TSR_TRY(check_precision(precision));
  TSR_TRY(check_ctx(ctx));
  float* dG;
  TSR_TRY(upload_tensor(ctx, grad_output, grad_ndim, shape, nullptr, &dG));
  FactorTable ft{};
  TSR_TRY(upload_factors(ctx, n_factors, shape, factors, R, &ft));
  const float* dw = nullptr;
  if (weights && R > 0) {
    void* p;
    TSR_TRY(slot_get(ctx, SLOT_MISC0, sizeof(float) * R, &p));
    TSR_CUDA(cudaMemcpyAsync(p, weights, sizeof(float) * R, cudaMemcpyHostToDevice, ctx->stream));
    dw = (const float*)p;
  }
  int64_t total = 0;
  for (int m = 0; m < n_factors; ++m) total += shape[m] * R;
  void* dout;
  TSR_TRY(slot_get(ctx, SLOT_OUT, sizeof(float) * (total > 0 ? total : 1), &dout));
  std::vector<float*> outs(n_factors);
  int64_t off = 0;
  for (int m = 0; m < n_factors; ++m) {
    outs[m] = (float*)dout + off;
    off += shape[m] * R;
  }
  TSR_TRY(reconstruction_grad_device(ctx, dG, grad_ndim, shape, ft, (int)R, dw, precision,
                                     outs.data()));
  for (int m = 0; m < n_factors; ++m)
    if (shape[m] * R > 0)
      TSR_CUDA(cudaMemcpyAsync(out_grads[m], outs[m], sizeof(float) * shape[m] * R,
                               cudaMemcpyDeviceToHost, ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

int tsr_cp_reconstruction_grad_dev_f32(tsr_ctx* ctx, const float* d_grad_output, int ndim,
                                       const int64_t* shape, const float* const* d_factors,
                                       int64_t rank, const float* d_weights, int precision,
                                       float* const* d_out_grads) {
  if (!shape || !d_grad_output || !d_factors || !d_out_grads)
    return fail(TSR_E_INVALID_ARG, "null argument");
  std::vector<int64_t> cols(ndim > 0 ? ndim : 1, rank);
  TSR_TRY(validate_grad(ndim, shape, ndim, shape, cols.data()));
  TSR_TRY(check_precision(precision));
  TSR_TRY(check_ctx(ctx));
  FactorTable ft{};
  for (int m = 0; m < ndim; ++m) {
    ft.ptr[m] = d_factors[m];
    ft.rows[m] = shape[m];
  }
  return reconstruction_grad_device(ctx, d_grad_output, ndim, shape, ft, (int)rank, d_weights,
                                    precision, d_out_grads);
}

int tsr_dense_create_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim, const int64_t* shape,
                             int precision, tsr_dense** out) {
  if (!d_tensor || !shape || !out) return fail(TSR_E_INVALID_ARG, "null argument");
  *out = nullptr;
  if (ndim < 2) return fail(TSR_E_NEED_2_FACTORS, "Need at least 2 factor matrices for MTTKRP");
  if (ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d exceeds the supported %d", ndim, kMaxModes);
  for (int m = 0; m < ndim; ++m)
    if (shape[m] <= 0) return fail(TSR_E_SHAPE, "mode %d has size %lld", m, (long long)shape[m]);
  TSR_TRY(check_precision(precision));
  TSR_TRY(check_ctx(ctx));
  tsr_dense* d = new tsr_dense();
  d->ndim = ndim;
  d->precision = precision;
  d->device = ctx->device;
  d->dX = d_tensor;
  for (int m = 0; m < ndim; ++m) d->shape[m] = shape[m];
  auto cleanup = [&](int rc) {
    tsr_dense_destroy(d);
    return rc;
  };
  for (int m = 0; m < ndim; ++m) {
    size_t ab, bb;
    mode_operand_bytes(make_unfolding(ndim, shape, m), precision, &ab, &bb);
    if (ab && cudaMalloc(&d->owned[2 * m], ab) != cudaSuccess)
      return cleanup(fail(TSR_E_CUDA, "cudaMalloc of %zu bytes failed", ab));
    if (bb && cudaMalloc(&d->owned[2 * m + 1], bb) != cudaSuccess)
      return cleanup(fail(TSR_E_CUDA, "cudaMalloc of %zu bytes failed", bb));
    int rc = prepare_mode_into(ctx, d_tensor, ndim, shape, m, precision, d->owned[2 * m],
                               d->owned[2 * m + 1], &d->ops[m]);
    if (rc != TSR_OK) return cleanup(rc);
  }
  if (cudaMalloc(&d->d_scalars, 4 * sizeof(double)) != cudaSuccess)
    return cleanup(fail(TSR_E_CUDA, "cudaMalloc of the loss scalars failed"));
  // BF16x3, 3+ modes: the trailing-two-modes view (with 3 modes the leading
  // side is mode 0 alone)
  const int64_t vshape[3] = {prod_range(shape, 0, ndim - 2), shape[ndim - 2], shape[ndim - 1]};
  d->d3_three = dense3_supported(3, vshape, 1);
  d->d3_two = twosided_supported(vshape[0], vshape[1] * vshape[2], 1);
  if (precision == TSR_PREC_BF16X3 && ndim >= 3 && (d->d3_three || d->d3_two) &&
      vshape[0] <= ((int64_t)1 << 30) &&
      ((uintptr_t)d_tensor & 15) == 0) {
    const int64_t n = numel(ndim, shape);
    void *hp, *lp;
    if (cudaMalloc(&hp, sizeof(__nv_bfloat16) * n) != cudaSuccess)
      return cleanup(fail(TSR_E_CUDA, "cudaMalloc of the bf16 halves failed"));
    d->owned[2 * kMaxModes] = hp;
    if (cudaMalloc(&lp, sizeof(__nv_bfloat16) * n) != cudaSuccess)
      return cleanup(fail(TSR_E_CUDA, "cudaMalloc of the bf16 halves failed"));
    d->owned[2 * kMaxModes + 1] = lp;
    int rc = launch_split_bf16(ctx, ctx->stream, d_tensor, n, (__nv_bfloat16*)hp,
                               (__nv_bfloat16*)lp, d->d_scalars + 3);
    if (rc != TSR_OK) return cleanup(rc);
    d->d3_on = true;
    d->d3.I = vshape[0];
    d->d3.J = vshape[1];
    d->d3.K = vshape[2];
    d->d3.hi = (const __nv_bfloat16*)hp;
    d->d3.lo = (const __nv_bfloat16*)lp;
  }
  if (precision == TSR_PREC_FP32 && ndim >= 3 && vshape[0] <= ((int64_t)1 << 30) &&
      vshape[1] * vshape[2] < INT32_MAX) {
    const int64_t v2[2] = {vshape[0], vshape[1] * vshape[2]};
    for (int m = 0; m < 2; ++m) {
      // operand m: the 2-way view's mode-m unfolding (X, or its transpose)
      size_t ab, bb;
      mode_operand_bytes(make_unfolding(2, v2, m), precision, &ab, &bb);
      void* buf = nullptr;
      if (ab) {
        if (cudaMalloc(&buf, ab) != cudaSuccess)
          return cleanup(fail(TSR_E_CUDA, "cudaMalloc of %zu bytes failed", ab));
        d->owned[2 * kMaxModes + 2 + m] = buf;
      }
      int rc = prepare_mode_into(ctx, d_tensor, 2, v2, m, precision, buf, nullptr, &d->vops[m]);
      if (rc != TSR_OK) return cleanup(rc);
    }
    // the same bytes read as mode-0 unfoldings of finer tensors (their row
    // strides equal the 2-way view's: round_up(cols, 8)), so that the FP32
    // kernel forms the Khatri-Rao rows from the factors and may take its
    // run-scaled form over the fastest other mode
    d->vops[0].u = make_unfolding(3, vshape, 0);
    int64_t tshape[kMaxModes];
    tshape[0] = v2[1];
    for (int p = 0; p < ndim - 2; ++p) tshape[1 + p] = shape[p];
    d->vops[1].u = make_unfolding(ndim - 1, tshape, 0);
    d->v2_on = true;
    d->v2_shape[0] = v2[0];
    d->v2_shape[1] = v2[1];
  }
  cudaError_t e = cudaMemsetAsync(d->d_scalars, 0, 4 * sizeof(double), ctx->stream);
  if (e != cudaSuccess) return cleanup(fail(TSR_E_CUDA, "%s", cudaGetErrorString(e)));
  int rc = launch_norm_sq(ctx, ctx->stream, d_tensor, numel(ndim, shape), d->d_scalars);
  if (rc != TSR_OK) return cleanup(rc);
  e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cleanup(fail(TSR_E_CUDA, "%s", cudaGetErrorString(e)));
  *out = d;
  return TSR_OK;
}

int tsr_dense_destroy(tsr_dense* d) {
  if (!d) return TSR_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(d->device);
  for (void* p : d->owned)
    if (p) cudaFree(p);
  if (d->d_scalars) cudaFree(d->d_scalars);
  cudaSetDevice(prev);
  delete d;
  return TSR_OK;
}

int tsr_cp_loss_grad_dev_f32(tsr_ctx* ctx, const tsr_dense* X, const float* const* d_factors,
                             int64_t rank, double reg, float* const* d_grads, double* loss) {
  if (!X || !d_factors || !d_grads) return fail(TSR_E_INVALID_ARG, "null argument");
  if (rank <= 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: %lld", (long long)rank);
  if (rank > kMaxRank)
    return fail(TSR_E_UNSUPPORTED, "rank %lld exceeds the supported %d", (long long)rank,
                kMaxRank);
  TSR_TRY(check_ctx(ctx));
  if (ctx->device != X->device)
    return fail(TSR_E_INVALID_ARG, "tensor prepared on device %d, context on device %d",
                X->device, ctx->device);
  const int N = X->ndim, R = (int)rank, RR = R * R;
  FactorTable ft{};
  for (int m = 0; m < N; ++m) {
    ft.ptr[m] = d_factors[m];
    ft.rows[m] = X->shape[m];
  }
  void* gp;
  TSR_TRY(slot_get(ctx, SLOT_GRAMS, sizeof(double) * N * RR, &gp));
  double* grams = (double*)gp;
  TSR_CUDA(cudaMemsetAsync(X->d_scalars + 1, 0, 2 * sizeof(double), ctx->stream));
  {
    // every mode's Gram in one launch
    TSR_CUDA(cudaMemsetAsync(grams, 0, sizeof(double) * N * RR, ctx->stream));
    GramAll ga{};
    ga.ndim = N;
    ga.R = R;
    ga.grams = grams;
    ga.cta0[0] = 0;
    for (int m = 0; m < N; ++m) {
      const int64_t rows = X->shape[m];
      int64_t ctas = std::min<int64_t>(ceil_div(rows, 16), 2 * ctx->sm_count);
      ga.rpc[m] = ceil_div(rows, ctas);
      ga.U[m] = d_factors[m];
      ga.rows[m] = rows;
      ga.cta0[m + 1] = ga.cta0[m] + (int)ceil_div(rows, ga.rpc[m]);
    }
    const unsigned g = (unsigned)ga.cta0[N];
    switch ((R + 15) / 16) {
      case 1: gram_all_kernel<1><<<g, 256, 0, ctx->stream>>>(ga); break;
      case 2: gram_all_kernel<2><<<g, 256, 0, ctx->stream>>>(ga); break;
      case 3: gram_all_kernel<3><<<g, 256, 0, ctx->stream>>>(ga); break;
      case 4: gram_all_kernel<4><<<g, 256, 0, ctx->stream>>>(ga); break;
      case 5: gram_all_kernel<5><<<g, 256, 0, ctx->stream>>>(ga); break;
      case 6: gram_all_kernel<6><<<g, 256, 0, ctx->stream>>>(ga); break;
      default: gram_all_kernel<7><<<g, 256, 0, ctx->stream>>>(ga); break;
    }
    ctx->launches++;
    TSR_CUDA(cudaGetLastError());
  }
  auto grad_of = [&](int n, const float* partials, int splits) -> int {
    const int64_t rows = X->shape[n];
    const int rpc =
        (int)std::max<int64_t>(1, std::min<int64_t>(16, ceil_div(rows, 2 * ctx->sm_count)));
    const int full = rpc * R;
    const int groups = full >= 256 ? 1 : 256 / full;
    const size_t smem = sizeof(double) * ((size_t)RR + full + (size_t)groups * full);
    if (smem > 200 * 1024)
      return fail(TSR_E_UNSUPPORTED, "rank %d too large for the gradient kernel", R);
    gram_grad_kernel<<<(unsigned)ceil_div(rows, rpc), 256, smem, ctx->stream>>>(
        grams, N, n, partials, splits, rows, R, rpc, d_factors[n], reg, d_grads[n],
        X->d_scalars);
    ctx->launches++;
    TSR_CUDA(cudaGetLastError());
    return TSR_OK;
  };
  auto finish = [&]() -> int {
    gram_loss_kernel<<<1, 256, 0, ctx->stream>>>(grams, N, R, reg, X->d_scalars);
    ctx->launches++;
    TSR_CUDA(cudaGetLastError());
    if (loss) {
      TSR_TRY(check_device_status(ctx));
      TSR_CUDA(cudaMemcpyAsync(loss, X->d_scalars + 2, sizeof(double), cudaMemcpyDeviceToHost,
                               ctx->stream));
      TSR_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return TSR_OK;
  };
  // From T (A x R: the leading modes, the trailing two contracted) and P
  // (C x R: the trailing two, the leading contracted): every mode's MTTKRP
  // and gradient rows and the Gram part of the loss in one programmatic
  // launch (R <= 32), then the loss when requested.
  auto contract_grad = [&](const float* T, const float* P) -> int {
    int total_rows = 0;
    for (int p = 0; p < N; ++p) total_rows += (int)X->shape[p];
    TContract c{};
    set_side(c, 0, T, X->shape, 0, N - 2, d_factors);
    set_side(c, 1, P, X->shape, N - 2, N, d_factors);
    c.R = R;
    c.nmodes = N;
    c.row0[0] = 0;
    for (int p = 0; p < N; ++p) {
      c.side_of[p] = p < N - 2 ? 0 : 1;
      c.pos[p] = p < N - 2 ? p : p - (N - 2);
      c.row0[p + 1] = c.row0[p] + (int)X->shape[p];
    }
    GradArgs g{};
    g.grams = grams;
    g.ndim = N;
    g.reg = reg;
    g.scal = X->d_scalars;
    for (int m = 0; m < N; ++m) g.G[m] = d_grads[m];
    TSR_CUDA(launch_pdl(t_contract_grad_kernel, dim3((unsigned)total_rows + 1), dim3(256), 0,
                        ctx->stream, c, g));
    ctx->launches++;
    TSR_CUDA(cudaGetLastError());
    if (loss) {
      TSR_TRY(check_device_status(ctx));
      double sc[4];
      TSR_CUDA(cudaMemcpyAsync(sc, X->d_scalars, sizeof(sc), cudaMemcpyDeviceToHost, ctx->stream));
      TSR_CUDA(cudaStreamSynchronize(ctx->stream));
      *loss = sc[0] - 2.0 * sc[1] + sc[3];
    }
    return TSR_OK;
  };
  if (X->d3_on && X->d3_two && twosided_supported(X->d3.I, X->d3.J * X->d3.K, R)) {
    // one read of X's bf16 halves: T = X_(lead) KR(trailing two) and
    // P = X_(lead)^T KR(leading) from the two-sided contraction, then every
    // mode's MTTKRP from T (modes 0..N-3) or P (modes N-2, N-1)
    const int64_t A = X->d3.I, C = X->d3.J * X->d3.K;
    const int64_t Ap = twosided_pad(A), Cp = twosided_pad(C);
    void *tp, *ip;
    // B images of V = KR(leading factors) and W = KR(trailing two), rows
    // formed on the fly
    const size_t vb = bimage_bytes(Ap, 32), wb = bimage_bytes(Cp, 32);
    TSR_TRY(slot_get(ctx, SLOT_D3_IMG, vb + wb, &ip));
    KRImages ki{};
    ki.n = 2;
    ki.R = R;
    ki.n_pad = 32;
    for (int w = 0; w < 2; ++w) {
      KRImage& im = ki.im[w];
      const int m0 = w == 0 ? 0 : N - 2, m1 = w == 0 ? N - 2 : N;
      im.nf = m1 - m0;
      for (int f = 0; f < im.nf; ++f) {
        im.U[f] = d_factors[m0 + f];
        im.size[f] = X->shape[m0 + f];
      }
      im.L = w == 0 ? A : C;
      im.chunks = (int)((w == 0 ? vb : wb) / 16);
      im.img = (uint8_t*)ip + (w == 0 ? 0 : vb);
    }
    // T and P (accumulated into by the two-sided kernel) are zeroed by the
    // same launch, whole float4s (the slot is padded to them)
    const int64_t tp_n4 = ceil_div((A + C) * R, 4);
    TSR_TRY(slot_get(ctx, SLOT_MISC0, sizeof(float) * 4 * tp_n4, &tp));
    ki.zero = (float*)tp;
    ki.zero_n4 = tp_n4;
    // programmatic launches from here to the end of the evaluation: each
    // kernel's launch and prologue overlap its predecessor, whose writes it
    // awaits before reading them
    TSR_TRY(launch_kr_images(ctx, ctx->stream, ki, true));
    TwoSided ts;
    ts.hi = X->d3.hi;
    ts.lo = X->d3.lo;
    ts.A = A;
    ts.C = C;
    ts.R = R;
    ts.vimg = (const uint8_t*)ip;
    ts.wimg = (const uint8_t*)ip + vb;
    ts.T = (float*)tp;
    ts.P = (float*)tp + A * R;
    TSR_TRY(launch_twosided(ctx, ctx->stream, ts));
    return contract_grad(ts.T, ts.P);
  }
  if (X->v2_on && R <= 32) {
    // FP32: T is the mode-0 MTTKRP of X as (A, I_{N-2}, I_{N-1}), P that of
    // X's transpose as (C, I_0, .., I_{N-3}): two passes over X's bytes
    // instead of one per mode, and half the FLOPs of N MTTKRPs
    const int64_t A = X->v2_shape[0], C = X->v2_shape[1];
    void* tp;
    TSR_TRY(slot_get(ctx, SLOT_MISC0, sizeof(float) * (A + C) * R, &tp));
    FactorTable f0{}, f1{};
    f0.ptr[0] = d_factors[0];  // the output mode's slot (not read)
    f0.rows[0] = A;
    f0.ptr[1] = d_factors[N - 2];
    f0.rows[1] = X->shape[N - 2];
    f0.ptr[2] = d_factors[N - 1];
    f0.rows[2] = X->shape[N - 1];
    f1.ptr[0] = d_factors[0];  // not read
    f1.rows[0] = C;
    for (int p = 0; p < N - 2; ++p) {
      f1.ptr[1 + p] = d_factors[p];
      f1.rows[1 + p] = X->shape[p];
    }
    float* T = (float*)tp;
    float* P = T + A * R;
    for (int v = 0; v < 2; ++v) {
      float* partials;
      int splits;
      TSR_TRY(run_mttkrp_partials(ctx, X->vops[v], v == 0 ? f0 : f1, R, TSR_PREC_FP32,
                                  &partials, &splits));
      TSR_TRY(launch_mttkrp_reduce(ctx, partials, splits, (v == 0 ? A : C) * R, v == 0 ? T : P));
    }
    return contract_grad(T, P);
  }
  if (X->d3_on && X->d3_three && R <= 64) {
    // three single-layout passes over X's bf16 halves instead of one MTTKRP
    // per mode: the view (A = prod of the leading modes, I_{N-2}, I_{N-1})
    Dense3 d = X->d3;
    d.R = R;
    d.n_pad = dense3_n_pad(R);
    const int64_t A = d.I;
    // Khatri-Rao of the leading factors (forward order): the view's U0
    void *kp, *kq, *tp, *mp, *ip;
    TSR_TRY(slot_get(ctx, SLOT_MISC1, sizeof(float) * A * R, &kp));
    TSR_TRY(slot_get(ctx, SLOT_MISC3, sizeof(float) * A * R, &kq));
    const float* kr = d_factors[0];
    int64_t krows = X->shape[0];
    float* bufs[2] = {(float*)kp, (float*)kq};
    for (int p = 1; p < N - 2; ++p) {
      float* dst = bufs[p & 1];
      TSR_TRY(launch_khatri_rao(ctx, kr, krows, d_factors[p], X->shape[p], R, dst));
      kr = dst;
      krows *= X->shape[p];
    }
    const size_t img1 = bimage_bytes(d.J, d.n_pad), img2 = bimage_bytes(d.K, d.n_pad);
    TSR_TRY(slot_get(ctx, SLOT_D3_IMG, img1 + img2, &ip));
    d.bimg[0] = nullptr;
    d.bimg[1] = (uint8_t*)ip;
    d.bimg[2] = (uint8_t*)ip + img1;
    TSR_TRY(launch_bimage(ctx, ctx->stream, d_factors[N - 2], d.J, R, d.n_pad, d.bimg[1]));
    TSR_TRY(launch_bimage(ctx, ctx->stream, d_factors[N - 1], d.K, R, d.n_pad, d.bimg[2]));
    FactorTable vt{};
    vt.ptr[0] = kr;
    vt.rows[0] = A;
    vt.ptr[1] = d_factors[N - 2];
    vt.rows[1] = d.J;
    vt.ptr[2] = d_factors[N - 1];
    vt.rows[2] = d.K;
    size_t pmax = 0;
    for (int v = 0; v < 3; ++v) {
      const SplitPlan pl = plan_mttkrp3(ctx, d, v);
      pmax = std::max(pmax, (size_t)pl.splits * dense3_rows(d, v) * R);
    }
    void* pp;
    TSR_TRY(slot_get(ctx, SLOT_PARTIALS, sizeof(float) * pmax, &pp));
    float* partials = (float*)pp;
    // T = the view's mode-0 MTTKRP (A x R), then the leading modes from it
    TSR_TRY(slot_get(ctx, SLOT_MISC0, sizeof(float) * A * R, &tp));
    {
      const SplitPlan pl = plan_mttkrp3(ctx, d, 0);
      TSR_TRY(launch_mttkrp3(ctx, ctx->stream, d, 0, vt, pl, partials, true));
      TSR_TRY(launch_mttkrp_reduce(ctx, partials, pl.splits, A * R, (float*)tp));
    }
    int lead_rows = 0;
    for (int p = 0; p < N - 2; ++p) lead_rows += (int)X->shape[p];
    TSR_TRY(slot_get(ctx, SLOT_MISC2, sizeof(float) * lead_rows * R, &mp));
    TContract c{};
    set_side(c, 0, (const float*)tp, X->shape, 0, N - 2, d_factors);
    c.R = R;
    c.nmodes = N - 2;
    c.row0[0] = 0;
    for (int p = 0; p < N - 2; ++p) {
      c.side_of[p] = 0;
      c.pos[p] = p;
      c.row0[p + 1] = c.row0[p] + (int)X->shape[p];
    }
    c.out = (float*)mp;
    t_contract_kernel<<<(unsigned)lead_rows, 256, 0, ctx->stream>>>(c);
    ctx->launches++;
    TSR_CUDA(cudaGetLastError());
    for (int m = 0; m < N - 2; ++m)
      TSR_TRY(grad_of(m, (const float*)mp + (int64_t)c.row0[m] * R, 1));
    // the trailing two modes straight from the view's modes 1 and 2
    for (int v = 1; v <= 2; ++v) {
      const SplitPlan pl = plan_mttkrp3(ctx, d, v);
      TSR_TRY(launch_mttkrp3(ctx, ctx->stream, d, v, vt, pl, partials, true));
      TSR_TRY(grad_of(N - 3 + v, partials, pl.splits));
    }
    return finish();
  }
  for (int n = 0; n < N; ++n) {
    float* partials;
    int splits;
    TSR_TRY(run_mttkrp_partials(ctx, X->ops[n], ft, R, X->precision, &partials, &splits));
    TSR_TRY(grad_of(n, partials, splits));
  }
  return finish();
}

}  // extern "C"

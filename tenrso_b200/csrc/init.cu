// CP factor initialisation: tenrso_decomp's initialize_factors
// (crates/tenrso-decomp/src/cp/helpers.rs:192-377) for every InitStrategy.
//
//   Random        U(0,1) per entry (helpers.rs:215-222)
//   RandomNormal  N(0,1) per entry (helpers.rs:223-231)
//   Svd           the leading left singular vectors of each unfolding X_(n),
//                 N(0, 0.01) columns past the unfolding's rank (:232-263)
//   Nnsvd         per component r the dominant sign part of (u_r, v_r),
//                 scaled by sqrt(s_r * |u_part| |v_part|) (:264-317)
//   LeverageScore u_r sqrt(s_r) sqrt(I_n * lev_i), lev the normalised row
//                 leverage scores of the leading singular vectors (:318-373)
//
// Random draws come from the library's seeded SplitMix64 stream (tenrso's
// thread_rng cannot be seeded): U(0,1) on stream 200 + n, N(0,1) on stream
// 400 + n (Box-Muller over streams 400 + n and 400 + n + 0x5151), the
// N(0, 0.01) padding columns on stream 500 + n.
//
// The singular vectors on the device: the FP64 Gram G = X_(n) X_(n)^T
// (I_n x I_n; the order of the unfolding's columns does not enter G), then a
// cyclic Jacobi eigensolver on G in round-robin order (I_n / 2 disjoint
// rotations per round, each round three launches: rotation angles, row
// update, column update with the eigenvector update), sweeps until the
// off-diagonal mass is below 1e-26 of the diagonal's. s_r = sqrt(lambda_r).
// v_r (needed by Nnsvd, only through the norms of its positive and negative
// parts) is X_(n)^T u_r / s_r, formed and reduced on the fly. SVD signs are
// arbitrary; each u_r is oriented so that its entry of largest magnitude is
// positive (Nnsvd's result does not depend on the sign).
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "dense.cuh"

namespace tsr {

namespace {

// ---- host generators --------------------------------------------------------

uint64_t mix64h(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double uniform_at(uint64_t seed, uint64_t stream, int64_t i) {
  const uint64_t golden = 0x9E3779B97F4A7C15ull;
  const uint64_t key = mix64h(seed * 0x100000001B3ull + stream * 0x2545F4914F6CDD1Dull + golden);
  return (double)(mix64h(key + (uint64_t)i * golden) >> 11) * (1.0 / 9007199254740992.0);
}

// N(0, sigma^2) doubles, identical to tenrso_b200.synth.normal(seed, stream) * sigma.
void seeded_normal(uint64_t seed, uint64_t stream, int64_t n, double sigma, double* out) {
  const double two_pi = 6.283185307179586;
  for (int64_t i = 0; i < n; ++i) {
    const double u1 = 1.0 - uniform_at(seed, stream, i);
    const double u2 = uniform_at(seed, stream + 0x5151, i);
    out[i] = sigma * std::sqrt(-2.0 * std::log(u1)) * std::cos(two_pi * u2);
  }
}

// ---- Gram of an unfolding ---------------------------------------------------

// G[i, i'] = sum_{a, b} X[a, i, b] X[a, i', b], X viewed as A x I x B
// (A = prod of the modes before n, B = prod after). 32 x 32 output tile per
// 256-thread CTA (2 x 2 per thread), FP64 accumulation over 32-wide chunks.
__global__ void __launch_bounds__(256) unfold_gram_kernel(const float* __restrict__ X, int64_t A,
                                                          int64_t I, int64_t B,
                                                          double* __restrict__ G) {
  __shared__ double xs[2][32][33];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t i0 = (int64_t)blockIdx.y * 32, k0 = (int64_t)blockIdx.x * 32;
  const int64_t J = A * B;
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (int64_t j0 = 0; j0 < J; j0 += 32) {
    // 32 rows x 32 columns of each operand: thread t loads 4 elements each
    for (int e = threadIdx.x; e < 2 * 32 * 32; e += 256) {
      const int w = e >> 10, r = (e >> 5) & 31, c = e & 31;
      const int64_t row = (w ? k0 : i0) + r, j = j0 + c;
      double v = 0.0;
      if (row < I && j < J) {
        const int64_t a = j / B, b = j % B;
        v = (double)__ldg(X + (a * I + row) * B + b);
      }
      xs[w][r][c] = v;
    }
    __syncthreads();
#pragma unroll 8
    for (int c = 0; c < 32; ++c) {
      const double x0 = xs[0][ty][c], x1 = xs[0][ty + 16][c];
      const double y0 = xs[1][tx][c], y1 = xs[1][tx + 16][c];
      acc[0][0] = fma(x0, y0, acc[0][0]);
      acc[0][1] = fma(x0, y1, acc[0][1]);
      acc[1][0] = fma(x1, y0, acc[1][0]);
      acc[1][1] = fma(x1, y1, acc[1][1]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int64_t i = i0 + ty + 16 * p, k = k0 + tx + 16 * q;
      if (i < I && k < I) G[i * I + k] = acc[p][q];
    }
}

// ---- cyclic Jacobi (round-robin pairs) ------------------------------------------

// Angles of this round's rotations: zero A[p][q] for each pair (p < q).
__global__ void jacobi_angles_kernel(const double* __restrict__ Am, int m,
                                     const int2* __restrict__ pairs, int npairs,
                                     double2* __restrict__ cs) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npairs) return;
  const int p = pairs[t].x, q = pairs[t].y;
  const double apq = Am[(int64_t)p * m + q], app = Am[(int64_t)p * m + p],
               aqq = Am[(int64_t)q * m + q];
  double c = 1.0, s = 0.0;
  if (fabs(apq) > 1e-300 && fabs(apq) > 1e-18 * sqrt(fabs(app * aqq))) {
    const double th = (aqq - app) / (2.0 * apq);
    double tn;
    if (fabs(th) > 1e150)
      tn = 0.5 / th;
    else
      tn = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
    c = 1.0 / sqrt(tn * tn + 1.0);
    s = tn * c;
  }
  cs[t] = make_double2(c, s);
}

// Rows p, q of A become c A_p - s A_q and s A_p + c A_q.
__global__ void jacobi_rows_kernel(double* __restrict__ Am, int m, const int2* __restrict__ pairs,
                                   int npairs, const double2* __restrict__ cs) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)npairs * m) return;
  const int i = (int)(t / m), k = (int)(t % m);
  const int p = pairs[i].x, q = pairs[i].y;
  const double c = cs[i].x, s = cs[i].y;
  const double ap = Am[(int64_t)p * m + k], aq = Am[(int64_t)q * m + k];
  Am[(int64_t)p * m + k] = c * ap - s * aq;
  Am[(int64_t)q * m + k] = s * ap + c * aq;
}

// Columns p, q of A and of V likewise.
__global__ void jacobi_cols_kernel(double* __restrict__ Am, double* __restrict__ V, int m,
                                   const int2* __restrict__ pairs, int npairs,
                                   const double2* __restrict__ cs) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)npairs * m) return;
  const int i = (int)(t % npairs), k = (int)(t / npairs);
  const int p = pairs[i].x, q = pairs[i].y;
  const double c = cs[i].x, s = cs[i].y;
  double* ar = Am + (int64_t)k * m;
  const double ap = ar[p], aq = ar[q];
  ar[p] = c * ap - s * aq;
  ar[q] = s * ap + c * aq;
  double* vr = V + (int64_t)k * m;
  const double vp = vr[p], vq = vr[q];
  vr[p] = c * vp - s * vq;
  vr[q] = s * vp + c * vq;
}

// out[0] = sum of squared off-diagonal entries, out[1] = sum of squared
// diagonal entries (out zeroed by the caller).
__global__ void jacobi_offdiag_kernel(const double* __restrict__ Am, int m, double* out) {
  double off = 0.0, dia = 0.0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)m * m;
       e += (int64_t)gridDim.x * blockDim.x) {
    const double v = Am[e];
    if (e / m == e % m)
      dia += v * v;
    else
      off += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) {
    off += __shfl_down_sync(0xffffffffu, off, o);
    dia += __shfl_down_sync(0xffffffffu, dia, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out, off);
    atomicAdd(out + 1, dia);
  }
}

// ---- factors from the singular vectors -------------------------------------------

// U[i, r] = +-V[i, col[r]] for r < k (the sign that makes the largest-|.|
// entry positive), one CTA per column; also writes the oriented column into
// Uo (I x k, FP64) for the later kernels.
__global__ void orient_kernel(const double* __restrict__ V, int m, int I,
                              const int* __restrict__ col, double* __restrict__ Uo, int k,
                              double* __restrict__ upn) {
  const int r = blockIdx.x;
  __shared__ double best_v[32];
  __shared__ int best_i[32];
  double bv = -1.0;
  int bi = 0x7fffffff;
  for (int i = threadIdx.x; i < I; i += blockDim.x) {
    const double a = fabs(V[(int64_t)i * m + col[r]]);
    if (a > bv || (a == bv && i < bi)) {
      bv = a;
      bi = i;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_down_sync(0xffffffffu, bv, o);
    const int oi = __shfl_down_sync(0xffffffffu, bi, o);
    if (ov > bv || (ov == bv && oi < bi)) {
      bv = ov;
      bi = oi;
    }
  }
  if ((threadIdx.x & 31) == 0) {
    best_v[threadIdx.x >> 5] = bv;
    best_i[threadIdx.x >> 5] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (best_v[w] > best_v[0] || (best_v[w] == best_v[0] && best_i[w] < best_i[0])) {
        best_v[0] = best_v[w];
        best_i[0] = best_i[w];
      }
  }
  __syncthreads();
  const double sg = V[(int64_t)best_i[0] * m + col[r]] < 0.0 ? -1.0 : 1.0;
  double up = 0.0, un = 0.0;
  for (int i = threadIdx.x; i < I; i += blockDim.x) {
    const double u = sg * V[(int64_t)i * m + col[r]];
    Uo[(int64_t)i * k + r] = u;
    if (u > 0.0) up += u * u;
    if (u < 0.0) un += u * u;
  }
  // norms^2 of the column's positive and negative parts (Nnsvd)
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) {
    up += __shfl_down_sync(0xffffffffu, up, o);
    un += __shfl_down_sync(0xffffffffu, un, o);
  }
  if ((threadIdx.x & 31) == 0) {
    best_v[threadIdx.x >> 5] = up;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += best_v[w];
    upn[2 * r] = t;
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) best_v[threadIdx.x >> 5] = un;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += best_v[w];
    upn[2 * r + 1] = t;
  }
}

// Norms^2 of the positive and negative parts of v_r = X_(n)^T u_r / s_r:
// one thread per unfolding column j (a, b), all k components; pn[2r] and
// pn[2r+1] accumulate (zeroed by the caller). Uo is I x k, sv the s_r.
__global__ void __launch_bounds__(256) vnorm_kernel(const float* __restrict__ X, int64_t A,
                                                    int64_t I, int64_t B,
                                                    const double* __restrict__ Uo, int k,
                                                    const double* __restrict__ sv,
                                                    double* __restrict__ pn) {
  extern __shared__ double us[];  // chunk of Uo rows: 64 x k
  const int64_t J = A * B;
  for (int r0 = 0; r0 < k; r0 += 16) {
    const int nr = min(16, k - r0);
    double pos[16], neg[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) pos[q] = neg[q] = 0.0;
    for (int64_t j0 = (int64_t)blockIdx.x * blockDim.x; j0 < J;
         j0 += (int64_t)gridDim.x * blockDim.x) {
      const int64_t j = j0 + threadIdx.x;
      const bool ok = j < J;
      const int64_t a = ok ? j / B : 0, b = ok ? j % B : 0;
      double w[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) w[q] = 0.0;
      for (int64_t i0 = 0; i0 < I; i0 += 64) {
        const int ni = (int)(I - i0 < 64 ? I - i0 : 64);
        __syncthreads();
        for (int e = threadIdx.x; e < ni * 16; e += blockDim.x) {
          const int ii = e / 16, q = e % 16;
          us[e] = q < nr ? Uo[(i0 + ii) * k + r0 + q] : 0.0;
        }
        __syncthreads();
        if (ok)
          for (int ii = 0; ii < ni; ++ii) {
            const double x = (double)__ldg(X + (a * I + i0 + ii) * B + b);
#pragma unroll
            for (int q = 0; q < 16; ++q) w[q] = fma(x, us[ii * 16 + q], w[q]);
          }
      }
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const double s = q < nr ? sv[r0 + q] : 0.0;
        const double v = (ok && s > 0.0) ? w[q] / s : 0.0;
        if (v > 0.0) pos[q] += v * v;
        if (v < 0.0) neg[q] += v * v;
      }
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      double p = pos[q], n = neg[q];
      for (int o = 16; o > 0; o >>= 1) {
        p += __shfl_down_sync(0xffffffffu, p, o);
        n += __shfl_down_sync(0xffffffffu, n, o);
      }
      if ((threadIdx.x & 31) == 0 && q < nr) {
        atomicAdd(pn + 2 * (r0 + q), p);
        atomicAdd(pn + 2 * (r0 + q) + 1, n);
      }
    }
  }
}

// The strategy's factor from the oriented singular vectors (one CTA; I x R
// outputs, FP64 arithmetic, fp32 result). pad holds the N(0, 0.01) draws for
// the columns k..R-1 (I x (R - k)).
__global__ void svd_factor_kernel(int strategy, const double* __restrict__ Uo, int I, int k,
                                  int R, const double* __restrict__ sv,
                                  const double* __restrict__ pn, const double* __restrict__ upn,
                                  const double* __restrict__ pad, float* __restrict__ out) {
  extern __shared__ double lev[];  // I leverage scores (LeverageScore only)
  __shared__ double red[32];
  if (strategy == TSR_INIT_LEVERAGE_SCORE) {
    // helpers.rs:331-349: lev_i = sum_{j<k} u_ij^2 / k, normalised by its sum
    // when that exceeds fp32 epsilon
    double part = 0.0;
    for (int i = threadIdx.x; i < I; i += blockDim.x) {
      double sc = 0.0;
      for (int j = 0; j < k; ++j) sc += Uo[(int64_t)i * k + j] * Uo[(int64_t)i * k + j];
      lev[i] = k > 0 ? sc / k : 0.0;
      part += lev[i];
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
      red[0] = t;
    }
    __syncthreads();
    const double total = red[0];
    if (total > 1.1920928955078125e-07)
      for (int i = threadIdx.x; i < I; i += blockDim.x) lev[i] /= total;
    __syncthreads();
  }
  for (int64_t e = threadIdx.x; e < (int64_t)I * R; e += blockDim.x) {
    const int i = (int)(e / R), r = (int)(e % R);
    double v;
    if (r < k) {
      const double u = Uo[(int64_t)i * k + r];
      if (strategy == TSR_INIT_SVD) {
        v = u;
      } else if (strategy == TSR_INIT_NNSVD) {
        // |u_pos| |v_pos| against |u_neg| |v_neg| (helpers.rs:277-300)
        const double pos_prod = sqrt(upn[2 * r]) * sqrt(pn[2 * r]);
        const double neg_prod = sqrt(upn[2 * r + 1]) * sqrt(pn[2 * r + 1]);
        if (pos_prod >= neg_prod)
          v = (u > 0.0 ? u : 0.0) * sqrt(sv[r] * pos_prod);
        else
          v = (u < 0.0 ? -u : 0.0) * sqrt(sv[r] * neg_prod);
      } else {  // LeverageScore
        v = u * sqrt(sv[r]) * sqrt(lev[i] * (double)I);
      }
    } else {
      const double z = pad[(int64_t)i * (R - k) + (r - k)];
      if (strategy == TSR_INIT_SVD)
        v = z;
      else if (strategy == TSR_INIT_NNSVD)
        v = fabs(z);
      else
        v = z * lev[i];
    }
    out[(int64_t)i * R + r] = (float)v;
  }
}

struct DevBuf {
  std::vector<void*> ptrs;
  template <class T>
  int get(T** p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess)
      return fail(TSR_E_CUDA, "cudaMalloc (%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    ptrs.push_back(q);
    *p = (T*)q;
    return TSR_OK;
  }
  ~DevBuf() {
    for (void* q : ptrs) cudaFree(q);
  }
};

constexpr int kMaxSvdRows = 1024;  // Jacobi on I_n x I_n: cubic in I_n

// Leading eigenpairs of G (I x I, device, overwritten): eigenvalues
// descending into lam (host, all I), eigenvector matrix V (device, m x m row
// major, column c = eigenvector of A's diagonal entry c) and the column of
// each rank position in order.
int jacobi_eigen(tsr_ctx* ctx, cudaStream_t s, DevBuf& buf, double* G, int I, double** Vout,
                 int* m_out, std::vector<double>* lam, std::vector<int>* order) {
  const int m = I + (I & 1);
  double *Am, *V, *off;
  TSR_TRY(buf.get(&Am, (size_t)m * m));
  TSR_TRY(buf.get(&V, (size_t)m * m));
  TSR_TRY(buf.get(&off, 2));
  TSR_CUDA(cudaMemsetAsync(Am, 0, sizeof(double) * m * m, s));
  TSR_CUDA(cudaMemcpy2DAsync(Am, sizeof(double) * m, G, sizeof(double) * I, sizeof(double) * I,
                             I, cudaMemcpyDeviceToDevice, s));
  std::vector<double> eye((size_t)m * m, 0.0);
  for (int i = 0; i < m; ++i) eye[(size_t)i * m + i] = 1.0;
  TSR_CUDA(cudaMemcpyAsync(V, eye.data(), sizeof(double) * m * m, cudaMemcpyHostToDevice, s));
  // round-robin pairing: player 0 fixed, the others rotate
  const int np = m / 2, rounds = m - 1;
  std::vector<int2> tab((size_t)rounds * np);
  std::vector<int> pl(m);
  std::iota(pl.begin(), pl.end(), 0);
  for (int r = 0; r < rounds; ++r) {
    for (int i = 0; i < np; ++i) {
      const int a = pl[i], b = pl[m - 1 - i];
      tab[(size_t)r * np + i] = make_int2(std::min(a, b), std::max(a, b));
    }
    std::rotate(pl.begin() + 1, pl.end() - 1, pl.end());
  }
  int2* pairs;
  double2* cs;
  TSR_TRY(buf.get(&pairs, tab.size()));
  TSR_TRY(buf.get(&cs, np));
  TSR_CUDA(cudaMemcpyAsync(pairs, tab.data(), sizeof(int2) * tab.size(), cudaMemcpyHostToDevice,
                           s));
  const unsigned g_rot = (unsigned)ceil_div(np, 128);
  const unsigned g_upd = (unsigned)ceil_div((int64_t)np * m, 256);
  for (int sweep = 0; sweep < 40; ++sweep) {
    double h[2];
    TSR_CUDA(cudaMemsetAsync(off, 0, 2 * sizeof(double), s));
    jacobi_offdiag_kernel<<<(unsigned)std::min<int64_t>(ceil_div((int64_t)m * m, 256), 1024), 256,
                            0, s>>>(Am, m, off);
    ctx->launches++;
    TSR_CUDA(cudaMemcpyAsync(h, off, sizeof(h), cudaMemcpyDeviceToHost, s));
    TSR_CUDA(cudaStreamSynchronize(s));
    if (!(h[0] > 1e-26 * h[1])) break;  // also stops on a zero matrix
    for (int r = 0; r < rounds; ++r) {
      const int2* pr = pairs + (size_t)r * np;
      jacobi_angles_kernel<<<g_rot, 128, 0, s>>>(Am, m, pr, np, cs);
      jacobi_rows_kernel<<<g_upd, 256, 0, s>>>(Am, m, pr, np, cs);
      jacobi_cols_kernel<<<g_upd, 256, 0, s>>>(Am, V, m, pr, np, cs);
      ctx->launches += 3;
    }
    TSR_CUDA(cudaGetLastError());
  }
  // eigenvalues: the diagonal (the padding index, if any, holds 0 and is dropped)
  std::vector<double> diag((size_t)m * m);
  TSR_CUDA(cudaMemcpy(diag.data(), Am, sizeof(double) * m * m, cudaMemcpyDeviceToHost));
  lam->assign(I, 0.0);
  for (int i = 0; i < I; ++i) (*lam)[i] = diag[(size_t)i * m + i];
  order->resize(I);
  std::iota(order->begin(), order->end(), 0);
  std::stable_sort(order->begin(), order->end(),
                   [&](int a, int b) { return (*lam)[a] > (*lam)[b]; });
  *Vout = V;
  *m_out = m;
  return TSR_OK;
}

}  // namespace

int init_factors_device(tsr_ctx* ctx, const float* dX, int ndim, const int64_t* shape, int R,
                        int strategy, uint64_t seed, float* d_out) {
  cudaStream_t s = ctx->stream;
  int64_t off = 0;
  for (int mode = 0; mode < ndim; ++mode) {
    const int64_t I = shape[mode];
    float* out = d_out + off;
    off += I * R;
    if (strategy == TSR_INIT_RANDOM || strategy == TSR_INIT_RANDOM_NORMAL) {
      std::vector<float> h((size_t)(I * R));
      if (strategy == TSR_INIT_RANDOM) {
        seeded_uniform(seed, 200 + mode, I * R, h.data());
      } else {
        std::vector<double> z((size_t)(I * R));
        seeded_normal(seed, 400 + mode, I * R, 1.0, z.data());
        for (size_t e = 0; e < z.size(); ++e) h[e] = (float)z[e];
      }
      TSR_CUDA(cudaMemcpyAsync(out, h.data(), sizeof(float) * I * R, cudaMemcpyHostToDevice, s));
      TSR_CUDA(cudaStreamSynchronize(s));
      continue;
    }
    if (I > kMaxSvdRows)
      return fail(TSR_E_UNSUPPORTED,
                  "SVD-based initialisation supports mode sizes up to %d (mode %d has %lld)",
                  kMaxSvdRows, mode, (long long)I);
    int64_t A = 1, B = 1;
    for (int m = 0; m < mode; ++m) A *= shape[m];
    for (int m = mode + 1; m < ndim; ++m) B *= shape[m];
    const int64_t J = A * B;
    DevBuf buf;
    double* G;
    TSR_TRY(buf.get(&G, (size_t)(I * I)));
    dim3 gg((unsigned)ceil_div(I, 32), (unsigned)ceil_div(I, 32));
    unfold_gram_kernel<<<gg, 256, 0, s>>>(dX, A, I, B, G);
    ctx->launches++;
    TSR_CUDA(cudaGetLastError());
    double* V;
    int m;
    std::vector<double> lam;
    std::vector<int> order;
    TSR_TRY(jacobi_eigen(ctx, s, buf, G, (int)I, &V, &m, &lam, &order));
    // the thin SVD of the I x J unfolding has min(I, J) components
    const int k = (int)std::min<int64_t>(R, std::min<int64_t>(I, J));
    std::vector<int> col(std::max(k, 1));
    std::vector<double> sv(std::max(k, 1));
    for (int r = 0; r < k; ++r) {
      col[r] = order[r];
      sv[r] = std::sqrt(std::max(lam[order[r]], 0.0));
    }
    int* dcol;
    double *dsv, *Uo, *pn, *upn, *dpad;
    TSR_TRY(buf.get(&dcol, col.size()));
    TSR_TRY(buf.get(&dsv, sv.size()));
    TSR_TRY(buf.get(&Uo, (size_t)I * std::max(k, 1)));
    TSR_TRY(buf.get(&pn, 2 * (size_t)std::max(k, 1)));
    TSR_TRY(buf.get(&upn, 2 * (size_t)std::max(k, 1)));
    TSR_TRY(buf.get(&dpad, (size_t)I * std::max(R - k, 1)));
    TSR_CUDA(cudaMemcpyAsync(dcol, col.data(), sizeof(int) * col.size(), cudaMemcpyHostToDevice, s));
    TSR_CUDA(cudaMemcpyAsync(dsv, sv.data(), sizeof(double) * sv.size(), cudaMemcpyHostToDevice, s));
    TSR_CUDA(cudaMemsetAsync(pn, 0, sizeof(double) * 2 * std::max(k, 1), s));
    std::vector<double> pad((size_t)I * std::max(R - k, 1), 0.0);
    if (R > k) {
      seeded_normal(seed, 500 + mode, I * (R - k), 0.01, pad.data());
      TSR_CUDA(cudaMemcpyAsync(dpad, pad.data(), sizeof(double) * pad.size(),
                               cudaMemcpyHostToDevice, s));
    }
    if (k > 0) {
      orient_kernel<<<k, 256, 0, s>>>(V, m, (int)I, dcol, Uo, k, upn);
      ctx->launches++;
      if (strategy == TSR_INIT_NNSVD) {
        const unsigned g = (unsigned)std::max<int64_t>(
            1, std::min<int64_t>(ceil_div(J, 256), 4 * (int64_t)ctx->sm_count));
        vnorm_kernel<<<g, 256, sizeof(double) * 64 * 16, s>>>(dX, A, I, B, Uo, k, dsv, pn);
        ctx->launches++;
      }
    }
    const size_t lev_bytes = strategy == TSR_INIT_LEVERAGE_SCORE ? sizeof(double) * I : 0;
    svd_factor_kernel<<<1, 1024, lev_bytes, s>>>(strategy, Uo, (int)I, k, R, dsv, pn, upn, dpad,
                                                  out);
    ctx->launches++;
    TSR_CUDA(cudaGetLastError());
    TSR_CUDA(cudaStreamSynchronize(s));
  }
  return TSR_OK;
}

void init_init_attributes() {
  cudaFuncSetAttribute(svd_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(sizeof(double) * kMaxSvdRows));
}

}  // namespace tsr

using namespace tsr;

extern "C" {

int tsr_cp_init_dev_f32(tsr_ctx* ctx, const float* d_tensor, int ndim, const int64_t* shape,
                        int64_t rank, int strategy, uint64_t seed, float* d_out_factors) {
  if (!shape || !d_out_factors) return fail(TSR_E_INVALID_ARG, "null argument");
  if (ndim < 1 || ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d outside 1..%d", ndim, kMaxModes);
  TSR_TRY(check_sizes(ndim, shape, rank));
  if (rank == 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: 0");
  if (strategy < TSR_INIT_RANDOM || strategy > TSR_INIT_LEVERAGE_SCORE)
    return fail(TSR_E_INVALID_ARG, "unknown initialisation strategy %d", strategy);
  if (strategy >= TSR_INIT_SVD && !d_tensor) return fail(TSR_E_INVALID_ARG, "null argument");
  TSR_TRY(check_ctx(ctx));
  return init_factors_device(ctx, d_tensor, ndim, shape, (int)rank, strategy, seed,
                             d_out_factors);
}

int tsr_cp_init_f32(tsr_ctx* ctx, const float* tensor, int ndim, const int64_t* shape,
                    int64_t rank, int strategy, uint64_t seed, float* out_factors) {
  if (!shape || !out_factors || !tensor) return fail(TSR_E_INVALID_ARG, "null argument");
  if (ndim < 1 || ndim > kMaxModes)
    return fail(TSR_E_UNSUPPORTED, "tensor rank %d outside 1..%d", ndim, kMaxModes);
  TSR_TRY(check_sizes(ndim, shape, rank));
  if (rank == 0) return fail(TSR_E_INVALID_RANK, "Invalid rank: 0");
  if (strategy < TSR_INIT_RANDOM || strategy > TSR_INIT_LEVERAGE_SCORE)
    return fail(TSR_E_INVALID_ARG, "unknown initialisation strategy %d", strategy);
  TSR_TRY(check_ctx(ctx));
  int64_t ftotal = 0;
  for (int m = 0; m < ndim; ++m) ftotal += shape[m] * rank;
  float* dX = nullptr;
  if (strategy >= TSR_INIT_SVD) TSR_TRY(upload_tensor(ctx, tensor, ndim, shape, nullptr, &dX));
  void* df;
  TSR_TRY(slot_get(ctx, SLOT_OUT, sizeof(float) * ftotal, &df));
  TSR_TRY(init_factors_device(ctx, dX, ndim, shape, (int)rank, strategy, seed, (float*)df));
  TSR_CUDA(cudaMemcpyAsync(out_factors, df, sizeof(float) * ftotal, cudaMemcpyDeviceToHost,
                           ctx->stream));
  TSR_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSR_OK;
}

}  // extern "C"

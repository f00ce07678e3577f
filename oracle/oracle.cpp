// TEST INFRASTRUCTURE ONLY — the oracle.
//
// A CPU restatement of tenrso's CP-ALS hot path, used by tests/ (as the
// checker) and by bench.py's cpu_baseline / --impl reference leg (as the timed
// CPU baseline). Nothing in the tenrso_b200 package links, loads or calls this
// file. Every function cites the tenrso source lines (paths relative to the
// tenrso repository root) whose loop order and arithmetic it restates.
//
// Two flavours exist for the dense kernels:
//   * "faithful": the reference's own loop order and sequential summation in T
//     (unfold copy, materialised forward Khatri-Rao, i/r/j triple loop).
//   * "fast": the same mathematics with a cache-friendly loop order and
//     OpenMP over output rows; used as the FP64 oracle at full sizes.
//
// Third-party arithmetic the reference delegates to crates that are not
// vendored (scirs2_linalg::lstsq, crates.io 0.3.0) is restated as a Cholesky
// solve of the symmetric Gram system with the reference's ridge fallback.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using i64 = int64_t;

// crates/tenrso-kernels/src/mttkrp.rs:149-177 (unfold_tensor): permutation
// [mode, others ascending], row-major reshape to I_mode x prod(others).
template <class T>
void unfold(const T* X, int ndim, const i64* shape, int mode, std::vector<T>& out) {
  i64 total = 1;
  for (int d = 0; d < ndim; ++d) total *= shape[d];
  out.resize(total);
  std::vector<i64> stride(ndim);
  stride[ndim - 1] = 1;
  for (int d = ndim - 2; d >= 0; --d) stride[d] = stride[d + 1] * shape[d + 1];
  std::vector<int> perm;
  perm.push_back(mode);
  for (int d = 0; d < ndim; ++d)
    if (d != mode) perm.push_back(d);
  std::vector<i64> idx(ndim, 0);  // index in permuted order
  for (i64 lin = 0; lin < total; ++lin) {
    i64 src = 0;
    for (int p = 0; p < ndim; ++p) src += idx[p] * stride[perm[p]];
    out[lin] = X[src];
    for (int p = ndim - 1; p >= 0; --p) {
      if (++idx[p] < shape[perm[p]]) break;
      idx[p] = 0;
    }
  }
}

// crates/tenrso-kernels/src/mttkrp.rs:209-240 (khatri_rao_two) and
// crates/tenrso-kernels/src/khatri_rao.rs:56-89: row = a_idx * J + b_idx,
// column-outer loop.
template <class T>
void khatri_rao_two(const T* A, i64 I, const T* B, i64 J, i64 K, T* C) {
  for (i64 k = 0; k < K; ++k)
    for (i64 a = 0; a < I; ++a)
      for (i64 b = 0; b < J; ++b) C[(a * J + b) * K + k] = A[a * K + k] * B[b * K + k];
}

// crates/tenrso-kernels/src/mttkrp.rs:182-206 (khatri_rao_except_mode):
// FORWARD order over the factors, skipping `mode`.
template <class T>
void kr_except(const T* const* U, int ndim, const i64* shape, i64 R, int mode, std::vector<T>& kr,
               i64& rows) {
  std::vector<T> cur, nxt;
  bool first = true;
  rows = 0;
  for (int m = 0; m < ndim; ++m) {
    if (m == mode) continue;
    if (first) {
      cur.assign(U[m], U[m] + shape[m] * R);
      rows = shape[m];
      first = false;
    } else {
      nxt.assign((size_t)(rows * shape[m] * R), T(0));
      khatri_rao_two(cur.data(), rows, U[m], shape[m], R, nxt.data());
      rows *= shape[m];
      cur.swap(nxt);
    }
  }
  kr.swap(cur);
}

// crates/tenrso-kernels/src/mttkrp.rs:74-146 (mttkrp), validation :86-122.
// Returns 0 or a negative code mirroring the reference's bail! cases.
template <class T>
int mttkrp_impl(const T* X, int ndim, const i64* shape, const T* const* U, i64 R, int mode, T* out,
                int faithful) {
  if (mode < 0 || mode >= ndim) return -1;  // "Mode {} out of bounds ..."
  if (ndim < 2) return -5;                  // "Need at least 2 factor matrices for MTTKRP"
  i64 In = shape[mode];
  i64 other = 1;
  for (int d = 0; d < ndim; ++d)
    if (d != mode) other *= shape[d];
  if (faithful) {
    std::vector<T> unf, kr;
    unfold(X, ndim, shape, mode, unf);
    i64 rows;
    kr_except(U, ndim, shape, R, mode, kr, rows);
    // HOT LOOP, mttkrp.rs:135-143: for i, for r, for j, sequential sum in T.
    for (i64 i = 0; i < In; ++i)
      for (i64 r = 0; r < R; ++r) {
        T sum = T(0);
        const T* urow = unf.data() + i * other;
        for (i64 j = 0; j < other; ++j) sum = sum + urow[j] * kr[j * R + r];
        out[i * R + r] = sum;
      }
    return 0;
  }
  // fast: same math, j-outer / r-inner loop order, KR rows formed on the fly
  // from per-mode indices (mttkrp_fused, mttkrp.rs:851-875), OpenMP on rows.
  std::vector<int> others;
  for (int d = 0; d < ndim; ++d)
    if (d != mode) others.push_back(d);
  std::vector<i64> xs(ndim);
  xs[ndim - 1] = 1;
  for (int d = ndim - 2; d >= 0; --d) xs[d] = xs[d + 1] * shape[d + 1];
  const int no = (int)others.size();
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < In; ++i) {
    std::vector<T> acc(R, T(0)), kr(R);
    std::vector<i64> idx(no, 0);
    for (i64 j = 0; j < other; ++j) {
      i64 off = i * xs[mode];
      for (int p = 0; p < no; ++p) off += idx[p] * xs[others[p]];
      T x = X[off];
      if (x != T(0)) {
        for (i64 r = 0; r < R; ++r) kr[r] = U[others[0]][idx[0] * R + r];
        for (int p = 1; p < no; ++p) {
          const T* row = U[others[p]] + idx[p] * R;
          for (i64 r = 0; r < R; ++r) kr[r] *= row[r];
        }
        for (i64 r = 0; r < R; ++r) acc[r] += x * kr[r];
      }
      for (int p = no - 1; p >= 0; --p) {
        if (++idx[p] < shape[others[p]]) break;
        idx[p] = 0;
      }
    }
    for (i64 r = 0; r < R; ++r) out[i * R + r] = acc[r];
  }
  return 0;
}

// crates/tenrso-decomp/src/cp/helpers.rs:434-452 (compute_gram_matrix).
template <class T>
void gram(const T* F, i64 rows, i64 R, T* G) {
  for (i64 a = 0; a < R; ++a)
    for (i64 b = 0; b < R; ++b) {
      T s = T(0);
      for (i64 k = 0; k < rows; ++k) s = s + F[k * R + a] * F[k * R + b];
      G[a * R + b] = s;
    }
}

// crates/tenrso-decomp/src/cp/helpers.rs:409-431 (compute_gram_hadamard):
// start from all-ones, multiply in every factor's Gram except skip_mode.
template <class T>
void gram_hadamard(const std::vector<std::vector<T>>& U, const i64* shape, int ndim, i64 R,
                   int skip, std::vector<T>& G) {
  G.assign(R * R, T(1));
  std::vector<T> g(R * R);
  for (int m = 0; m < ndim; ++m) {
    if (m == skip) continue;
    gram(U[m].data(), shape[m], R, g.data());
    for (i64 k = 0; k < R * R; ++k) G[k] = G[k] * g[k];
  }
}

// Cholesky factorisation in T; false when a pivot is not positive.
template <class T>
bool cholesky(std::vector<T>& A, i64 n) {
  for (i64 j = 0; j < n; ++j) {
    T d = A[j * n + j];
    for (i64 k = 0; k < j; ++k) d -= A[j * n + k] * A[j * n + k];
    if (!(d > T(0))) return false;
    d = std::sqrt(d);
    A[j * n + j] = d;
    for (i64 i = j + 1; i < n; ++i) {
      T s = A[i * n + j];
      for (i64 k = 0; k < j; ++k) s -= A[i * n + k] * A[j * n + k];
      A[i * n + j] = s / d;
    }
  }
  return true;
}

// crates/tenrso-decomp/src/cp/helpers.rs:455-495 (solve_least_squares):
// row i of the result solves G^T x = M[i,:]. lstsq (scirs2_linalg 0.3.0, not
// vendored) is restated as a Cholesky solve of the symmetric Gram; on failure
// the reference retries with eps*rank*10 added to the diagonal (:477-490).
// Returns 0, or -3 (LinalgError) when the ridged system also fails.
template <class T>
int solve_ls(const T* M, i64 rows, const std::vector<T>& G, i64 R, T* out) {
  std::vector<T> L(R * R);
  for (i64 a = 0; a < R; ++a)
    for (i64 b = 0; b < R; ++b) L[a * R + b] = G[b * R + a];  // gram.t()
  if (!cholesky(L, R)) {
    T eps = std::numeric_limits<T>::epsilon() * T(R * 10);
    for (i64 a = 0; a < R; ++a)
      for (i64 b = 0; b < R; ++b) L[a * R + b] = G[b * R + a];
    for (i64 k = 0; k < R; ++k) L[k * R + k] += eps;
    if (!cholesky(L, R)) return -3;
  }
  std::vector<T> y(R);
  for (i64 i = 0; i < rows; ++i) {
    const T* b = M + i * R;
    for (i64 a = 0; a < R; ++a) {
      T s = b[a];
      for (i64 k = 0; k < a; ++k) s -= L[a * R + k] * y[k];
      y[a] = s / L[a * R + a];
    }
    for (i64 a = R - 1; a >= 0; --a) {
      T s = y[a];
      for (i64 k = a + 1; k < R; ++k) s -= L[k * R + a] * out[i * R + k];
      out[i * R + a] = s / L[a * R + a];
    }
  }
  return 0;
}

// crates/tenrso-decomp/src/cp/helpers.rs:498-510 (compute_norm_squared):
// sequential sum of squares in T.
template <class T>
T norm_sq(const T* X, i64 n) {
  T s = T(0);
  for (i64 k = 0; k < n; ++k) s = s + X[k] * X[k];
  return s;
}

// crates/tenrso-decomp/src/cp/helpers.rs:533-555
// (compute_reconstruction_norm_squared).
template <class T>
T recon_norm_sq(const std::vector<std::vector<T>>& U, const i64* shape, int ndim, i64 R) {
  T total = T(0);
  for (i64 r = 0; r < R; ++r)
    for (i64 s = 0; s < R; ++s) {
      T cross = T(1);
      for (int m = 0; m < ndim; ++m) {
        T ip = T(0);
        for (i64 i = 0; i < shape[m]; ++i) ip = ip + U[m][i * R + r] * U[m][i * R + s];
        cross = cross * ip;
      }
      total = total + cross;
    }
  return total;
}

// crates/tenrso-decomp/src/cp/helpers.rs:513-530 (compute_fit) with the inner
// product of :558-579 (compute_inner_product = a full mttkrp on mode 0,
// summed r-outer / i-inner against U_0).
template <class T>
T compute_fit(const T* X, int ndim, const i64* shape, const std::vector<std::vector<T>>& U, i64 R,
              T xnorm_sq, int faithful) {
  T rn = recon_norm_sq(U, shape, ndim, R);
  std::vector<const T*> ptrs(ndim);
  for (int m = 0; m < ndim; ++m) ptrs[m] = U[m].data();
  std::vector<T> M0(shape[0] * R);
  mttkrp_impl(X, ndim, shape, ptrs.data(), R, 0, M0.data(), faithful);
  T ip = T(0);
  for (i64 r = 0; r < R; ++r)
    for (i64 i = 0; i < shape[0]; ++i) ip = ip + M0[i * R + r] * U[0][i * R + r];
  T err_sq = xnorm_sq + rn - T(2) * ip;
  T err = std::sqrt(std::max(err_sq, T(0)));
  T fit = T(1) - err / std::sqrt(xnorm_sq);
  return std::min(std::max(fit, T(0)), T(1));
}

// crates/tenrso-decomp/src/cp/core.rs:59-182 (cp_als) with the factors
// injected instead of thread_rng (helpers.rs:212-222 cannot be seeded).
// reason: 0 MaxIterations, 1 FitTolerance, 2 Oscillation.
template <class T>
int cp_als_impl(const T* X, int ndim, const i64* shape, i64 R, int max_iters, double tol,
                T* factors_io, T* fit_history, int* iters_out, int* reason_out, int* osc_out,
                T* final_change_out, T* fit_out, int faithful) {
  if (R == 0) return -10;  // CpError::InvalidRank
  for (int d = 0; d < ndim; ++d)
    if (R > shape[d]) return -10;
  if (!(tol >= 0.0 && tol < 1.0)) return -11;  // CpError::InvalidTolerance
  std::vector<std::vector<T>> U(ndim);
  {
    T* p = factors_io;
    for (int m = 0; m < ndim; ++m) {
      U[m].assign(p, p + shape[m] * R);
      p += shape[m] * R;
    }
  }
  i64 total = 1;
  for (int d = 0; d < ndim; ++d) total *= shape[d];
  T xn = norm_sq(X, total);
  T prev_fit = T(0), fit = T(0), final_change = T(0);
  int iters = 0, osc = 0, reason = 0;
  std::vector<T> M, G;
  std::vector<const T*> ptrs(ndim);
  for (int iter = 0; iter < max_iters; ++iter) {
    iters = iter + 1;
    for (int mode = 0; mode < ndim; ++mode) {
      for (int m = 0; m < ndim; ++m) ptrs[m] = U[m].data();
      M.assign(shape[mode] * R, T(0));
      mttkrp_impl(X, ndim, shape, ptrs.data(), R, mode, M.data(), faithful);
      gram_hadamard(U, shape, ndim, R, mode, G);
      int rc = solve_ls(M.data(), shape[mode], G, R, U[mode].data());
      if (rc) return rc;
    }
    fit = compute_fit(X, ndim, shape, U, R, xn, faithful);
    fit_history[iter] = fit;
    if (iter > 0 && fit < prev_fit) osc += 1;
    T change = std::abs(fit - prev_fit);
    final_change = change;
    if (iter > 0 && change < T(tol)) {
      reason = 1;
      break;
    }
    if (osc > 5 && iter > 10) {
      reason = 2;
      break;
    }
    prev_fit = fit;
  }
  T* p = factors_io;
  for (int m = 0; m < ndim; ++m) {
    std::copy(U[m].begin(), U[m].end(), p);
    p += shape[m] * R;
  }
  *iters_out = iters;
  *reason_out = reason;
  *osc_out = osc;
  *final_change_out = final_change;
  *fit_out = fit;
  return 0;
}

// crates/tenrso-sparse/src/coo.rs:239-257 (sort: stable sort of a permutation
// by lexicographic index) and :320-347 (deduplicate: consecutive equal indices
// summed left to right). idx is nnz x ndim row-major; rewritten in place.
// Returns the deduplicated nnz.
template <class T>
i64 coo_dedup(i64* idx, T* vals, i64 nnz, int ndim) {
  if (nnz <= 1) return nnz;
  std::vector<i64> perm(nnz);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](i64 a, i64 b) {
    const i64* ia = idx + a * ndim;
    const i64* ib = idx + b * ndim;
    for (int d = 0; d < ndim; ++d)
      if (ia[d] != ib[d]) return ia[d] < ib[d];
    return false;
  });
  std::vector<i64> si(nnz * ndim);
  std::vector<T> sv(nnz);
  for (i64 k = 0; k < nnz; ++k) {
    std::memcpy(&si[k * ndim], idx + perm[k] * ndim, sizeof(i64) * ndim);
    sv[k] = vals[perm[k]];
  }
  i64 w = 0;
  for (i64 r = 1; r < nnz; ++r) {
    if (std::memcmp(&si[w * ndim], &si[r * ndim], sizeof(i64) * ndim) == 0) {
      sv[w] = sv[w] + sv[r];
    } else {
      ++w;
      if (w != r) {
        std::memcpy(&si[w * ndim], &si[r * ndim], sizeof(i64) * ndim);
        sv[w] = sv[r];
      }
    }
  }
  i64 out = w + 1;
  std::memcpy(idx, si.data(), sizeof(i64) * out * ndim);
  std::memcpy(vals, sv.data(), sizeof(T) * out);
  return out;
}

}  // namespace

extern "C" {

int orc_mttkrp_f32(const float* X, int ndim, const int64_t* shape, const float* const* U, int64_t R,
                   int mode, float* out, int faithful) {
  return mttkrp_impl<float>(X, ndim, shape, U, R, mode, out, faithful);
}
int orc_mttkrp_f64(const double* X, int ndim, const int64_t* shape, const double* const* U,
                   int64_t R, int mode, double* out, int faithful) {
  return mttkrp_impl<double>(X, ndim, shape, U, R, mode, out, faithful);
}

void orc_khatri_rao_f64(const double* A, int64_t I, const double* B, int64_t J, int64_t K,
                        double* C) {
  khatri_rao_two<double>(A, I, B, J, K, C);
}

void orc_gram_f64(const double* F, int64_t rows, int64_t R, double* G) {
  gram<double>(F, rows, R, G);
}

int orc_cp_als_f32(const float* X, int ndim, const int64_t* shape, int64_t R, int max_iters,
                   double tol, float* factors_io, float* fit_history, int* iters, int* reason,
                   int* osc, float* final_change, float* fit, int faithful) {
  return cp_als_impl<float>(X, ndim, shape, R, max_iters, tol, factors_io, fit_history, iters,
                            reason, osc, final_change, fit, faithful);
}
int orc_cp_als_f64(const double* X, int ndim, const int64_t* shape, int64_t R, int max_iters,
                   double tol, double* factors_io, double* fit_history, int* iters, int* reason,
                   int* osc, double* final_change, double* fit, int faithful) {
  return cp_als_impl<double>(X, ndim, shape, R, max_iters, tol, factors_io, fit_history, iters,
                             reason, osc, final_change, fit, faithful);
}

// One mode update of the reference loop (core.rs:129-140) in T=double, used to
// check the GPU solve in isolation: U_mode <- mttkrp * gram_hadamard^-1.
int orc_solve_f64(const double* M, int64_t rows, const double* G, int64_t R, double* out) {
  std::vector<double> g(G, G + R * R);
  return solve_ls<double>(M, rows, g, R, out);
}

int64_t orc_coo_dedup_f32(int64_t* idx, float* vals, int64_t nnz, int ndim) {
  return coo_dedup<float>(idx, vals, nnz, ndim);
}

// crates/tenrso-sparse/src/csf.rs:137-264 (CsfTensor::from_coo). idx is
// nnz x ndim row-major. fptr is ndim x (nnz+1), fids ndim x nnz (row l holds
// level l); lens[2l] = len(fptr[l]), lens[2l+1] = len(fids[l]). vals gets the
// leaf values. Returns 0, or -20 when mode_order is not a permutation.
int orc_csf_from_coo_f32(const int64_t* idx, const float* vals_in, int64_t nnz, int ndim,
                         const int64_t* mode_order, int64_t* fptr, int64_t* fids, float* vals,
                         int64_t* lens) {
  {
    std::vector<int64_t> s(mode_order, mode_order + ndim);
    std::sort(s.begin(), s.end());
    for (int d = 0; d < ndim; ++d)
      if (s[d] != d) return -20;
  }
  const int64_t W = nnz + 1;
  if (nnz == 0) {  // csf.rs:158-168: fptr = [[0]; ndim], fids = [[]; ndim]
    for (int l = 0; l < ndim; ++l) {
      fptr[l * W] = 0;
      lens[2 * l] = 1;
      lens[2 * l + 1] = 0;
    }
    return 0;
  }
  std::vector<int64_t> perm(nnz);
  std::iota(perm.begin(), perm.end(), 0);
  // csf.rs:178-186: stable sort_by over mode_order.
  std::stable_sort(perm.begin(), perm.end(), [&](int64_t a, int64_t b) {
    for (int l = 0; l < ndim; ++l) {
      int64_t m = mode_order[l];
      int64_t x = idx[a * ndim + m], y = idx[b * ndim + m];
      if (x != y) return x < y;
    }
    return false;
  });
  auto key = [&](int64_t pos, int64_t mode) { return idx[perm[pos] * ndim + mode]; };
  // level 0, csf.rs:193-214
  int64_t np = 0, ni = 0;
  fptr[np++] = 0;
  {
    int64_t m = mode_order[0];
    int64_t i = 0;
    while (i < nnz) {
      int64_t v = key(i, m);
      fids[ni++] = v;
      int64_t j = i;
      while (j < nnz && key(j, m) == v) ++j;
      fptr[np] = fptr[np - 1] + (j - i);
      ++np;
      i = j;
    }
  }
  lens[0] = np;
  lens[1] = ni;
  int64_t nvals = 0;
  // levels 1..ndim-1, csf.rs:217-254
  for (int level = 1; level < ndim; ++level) {
    int64_t m = mode_order[level];
    const int64_t* prev = fptr + (level - 1) * W;
    int64_t prev_len = lens[2 * (level - 1)];
    int64_t* np_ = fptr + level * W;
    int64_t* ni_ = fids + level * nnz;
    int64_t cp = 0, ci = 0;
    np_[cp++] = 0;
    for (int64_t f = 0; f + 1 < prev_len; ++f) {
      int64_t start = prev[f], end = prev[f + 1];
      if (level == ndim - 1) {
        for (int64_t p = start; p < end; ++p) {
          ni_[ci++] = key(p, m);
          vals[nvals++] = vals_in[perm[p]];
        }
        np_[cp++] = nvals;
      } else {
        int64_t ls = start;
        while (ls < end) {
          int64_t v = key(ls, m);
          ni_[ci++] = v;
          int64_t le = ls;
          while (le < end && key(le, m) == v) ++le;
          np_[cp] = np_[cp - 1] + (le - ls);
          ++cp;
          ls = le;
        }
      }
    }
    lens[2 * level] = cp;
    lens[2 * level + 1] = ci;
  }
  return 0;
}

// Sparse MTTKRP has no reference implementation (tenrso-sparse mentions it
// only in doc comments, csf.rs:42). Its definition is the dense mttkrp math
// (mttkrp.rs:851-875) restricted to the nonzeros:
//   M[i_n, r] = sum_k v_k * prod_{m != n} U_m[i_m(k), r],
// accumulated here in double over COO entries in the given order.
void orc_coo_mttkrp_f64(const int64_t* idx, const double* vals, int64_t nnz, int ndim,
                        const int64_t* shape, const double* const* U, int64_t R, int mode,
                        double* out) {
  std::fill(out, out + shape[mode] * R, 0.0);
  std::vector<double> t(R);
  for (int64_t k = 0; k < nnz; ++k) {
    for (int64_t r = 0; r < R; ++r) t[r] = vals[k];
    for (int m = 0; m < ndim; ++m) {
      if (m == mode) continue;
      const double* row = U[m] + idx[k * ndim + m] * R;
      for (int64_t r = 0; r < R; ++r) t[r] *= row[r];
    }
    double* o = out + idx[k * ndim + mode] * R;
    for (int64_t r = 0; r < R; ++r) o[r] += t[r];
  }
}

// crates/tenrso-kernels/src/outer.rs:223-274 (cp_reconstruct): sum over r of
// the weighted outer product of the r-th factor columns; row-major output.
void orc_cp_reconstruct_f64(const double* const* U, int ndim, const int64_t* shape, int64_t R,
                            const double* weights, double* out) {
  int64_t total = 1;
  for (int d = 0; d < ndim; ++d) total *= shape[d];
#pragma omp parallel for schedule(static)
  for (int64_t lin = 0; lin < total; ++lin) {
    int64_t rem = lin;
    std::vector<int64_t> ix(ndim);
    for (int d = ndim - 1; d >= 0; --d) {
      ix[d] = rem % shape[d];
      rem /= shape[d];
    }
    double s = 0.0;
    for (int64_t r = 0; r < R; ++r) {
      double p = weights ? weights[r] : 1.0;
      for (int d = 0; d < ndim; ++d) p *= U[d][ix[d] * R + r];
      s += p;
    }
    out[lin] = s;
  }
}

// Sum over the slice {i_mode = index} of (X - Xhat)^2 in FP64, with Xhat the
// reconstruction of outer.rs:223-274 (no weights). Perturbing U_mode[index, r]
// changes Xhat only on this slice, so central differences of the loss
// ||X - Xhat||^2 in that entry need only this slice (test infrastructure for
// the finite-difference check of the reconstruction gradient, grad.rs:81-120).
double orc_cp_slice_sqerr_f64(const double* X, int ndim, const int64_t* shape,
                              const double* const* U, int64_t R, int mode, int64_t index) {
  int64_t total = 1;
  for (int d = 0; d < ndim; ++d) total *= shape[d];
  const int64_t n_slice = total / shape[mode];
  double acc = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : acc)
  for (int64_t t = 0; t < n_slice; ++t) {
    // decode t over the other modes (last fastest), then place `index`
    std::vector<int64_t> ix(ndim);
    int64_t rem = t;
    for (int d = ndim - 1; d >= 0; --d) {
      if (d == mode) continue;
      ix[d] = rem % shape[d];
      rem /= shape[d];
    }
    ix[mode] = index;
    int64_t lin = 0;
    for (int d = 0; d < ndim; ++d) lin = lin * shape[d] + ix[d];
    double s = 0.0;
    for (int64_t r = 0; r < R; ++r) {
      double p = 1.0;
      for (int d = 0; d < ndim; ++d) p *= U[d][ix[d] * R + r];
      s += p;
    }
    const double e = X[lin] - s;
    acc += e * e;
  }
  return acc;
}

// Restated CSF MTTKRP over the reference CSF layout (csf.rs:193-254: every
// fptr level holds nnz offsets), 3-way, root = mode_order[0]; no tenrso
// implementation exists (csf.rs:42). Per root: for each of its level-1 fibers
// t = sum_k v_k U_leaf[leaf_k], then acc += U_fiber[fiber id] (*) t; the root's
// row of out (zeroed here) receives acc. fp32 arithmetic, as the f32 path.
// threads > 1 splits the roots over OpenMP threads (each output row has one
// owner); threads == 1 runs the same loop serially.
void orc_csf_mttkrp_f32(int64_t n_roots, const int64_t* root_ptr, const int64_t* root_ids,
                        int64_t n_fibers, const int64_t* fib_ptr, const int64_t* fib_ids,
                        const int64_t* leaf_ids, const float* vals, const float* U_fiber,
                        const float* U_leaf, int64_t R, int64_t out_rows, float* out,
                        int threads) {
  std::fill(out, out + out_rows * R, 0.0f);
  auto body = [&](int64_t s, std::vector<float>& acc, std::vector<float>& t) {
    std::fill(acc.begin(), acc.end(), 0.0f);
    const int64_t k0 = root_ptr[s], k1 = root_ptr[s + 1];
    // first fiber of the root: fib_ptr[f] == k0
    int64_t f = std::lower_bound(fib_ptr, fib_ptr + n_fibers, k0) - fib_ptr;
    for (; f < n_fibers && fib_ptr[f] < k1; ++f) {
      const int64_t e1 = f + 1 < n_fibers ? fib_ptr[f + 1] : k1;
      std::fill(t.begin(), t.end(), 0.0f);
      for (int64_t k = fib_ptr[f]; k < e1 && k < k1; ++k) {
        const float* row = U_leaf + leaf_ids[k] * R;
        for (int64_t r = 0; r < R; ++r) t[r] += vals[k] * row[r];
      }
      const float* urow = U_fiber + fib_ids[f] * R;
      for (int64_t r = 0; r < R; ++r) acc[r] += urow[r] * t[r];
    }
    float* o = out + root_ids[s] * R;
    for (int64_t r = 0; r < R; ++r) o[r] += acc[r];
  };
  if (threads <= 1) {
    std::vector<float> acc(R), t(R);
    for (int64_t s = 0; s < n_roots; ++s) body(s, acc, t);
    return;
  }
#pragma omp parallel num_threads(threads)
  {
    std::vector<float> acc(R), t(R);
#pragma omp for schedule(dynamic, 16)
    for (int64_t s = 0; s < n_roots; ++s) body(s, acc, t);
  }
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"

"""TEST INFRASTRUCTURE ONLY — ctypes front end of the oracle (oracle.cpp).

The oracle is a CPU restatement of tenrso's CP-ALS hot path. Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
module, always as the checker or as the timed CPU baseline, never as the
product. Citations (paths inside the tenrso repository) are in oracle.cpp.

Parity anchors: the golden vectors in tenrso's own unit tests (Khatri-Rao
``khatri_rao.rs:41-55,479-554``; MTTKRP definition ``mttkrp.rs:1000-1043``;
Gram ``cp/tests.rs:26-35``; COO ``coo.rs:420-452``; CSF ``csf.rs:501-682``)
are replayed against this oracle in tests/test_oracle.py. The least-squares
solve (``scirs2_linalg::lstsq`` 0.3.0, a crates.io dependency that is not
vendored) is restated as a Cholesky solve; no reference test pins a solve
value, so that step is "parity unpinned".
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile."""
    if force or not os.path.exists(_LIB) or (
        os.path.getmtime(_LIB) < os.path.getmtime(os.path.join(_HERE, "oracle.cpp"))
    ):
        subprocess.run(["make", "-B", "-C", _HERE, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB)
        P = C.c_void_p
        I64 = C.c_int64
        L.orc_mttkrp_f32.argtypes = [P, C.c_int, P, P, I64, C.c_int, P, C.c_int]
        L.orc_mttkrp_f64.argtypes = [P, C.c_int, P, P, I64, C.c_int, P, C.c_int]
        L.orc_khatri_rao_f64.argtypes = [P, I64, P, I64, I64, P]
        L.orc_gram_f64.argtypes = [P, I64, I64, P]
        L.orc_cp_als_f32.argtypes = [P, C.c_int, P, I64, C.c_int, C.c_double, P, P, P, P, P, P, P,
                                     C.c_int]
        L.orc_cp_als_f64.argtypes = L.orc_cp_als_f32.argtypes
        L.orc_solve_f64.argtypes = [P, I64, P, I64, P]
        L.orc_coo_dedup_f32.argtypes = [P, P, I64, C.c_int]
        L.orc_coo_dedup_f32.restype = I64
        L.orc_csf_from_coo_f32.argtypes = [P, P, I64, C.c_int, P, P, P, P, P]
        L.orc_coo_mttkrp_f64.argtypes = [P, P, I64, C.c_int, P, P, I64, C.c_int, P]
        L.orc_csf_mttkrp_f32.argtypes = [I64, P, P, I64, P, P, P, P, P, P, I64, I64, P, C.c_int]
        L.orc_cp_reconstruct_f64.argtypes = [P, C.c_int, P, I64, P, P]
        L.orc_cp_slice_sqerr_f64.argtypes = [P, C.c_int, P, P, I64, C.c_int, I64]
        L.orc_cp_slice_sqerr_f64.restype = C.c_double
        L.orc_num_threads.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _ptr_array(arrs):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def num_threads() -> int:
    return lib().orc_num_threads()


def mttkrp(X: np.ndarray, factors, mode: int, faithful: bool = False) -> np.ndarray:
    """Restated ``tenrso_kernels::mttkrp`` (mttkrp.rs:74-146) in X's dtype."""
    dt = X.dtype
    assert dt in (np.float32, np.float64)
    X = np.ascontiguousarray(X)
    fs = [np.ascontiguousarray(f, dtype=dt) for f in factors]
    shape = np.asarray(X.shape, dtype=np.int64)
    R = fs[0].shape[1]
    out = np.zeros((X.shape[mode], R), dtype=dt)
    fn = lib().orc_mttkrp_f32 if dt == np.float32 else lib().orc_mttkrp_f64
    rc = fn(_ptr(X), X.ndim, _ptr(shape), _ptr_array(fs), R, mode, _ptr(out), int(faithful))
    if rc:
        raise ValueError(f"oracle mttkrp failed: {rc}")
    return out


def khatri_rao(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """Restated ``tenrso_kernels::khatri_rao`` (khatri_rao.rs:56-89)."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    assert A.shape[1] == B.shape[1]
    out = np.zeros((A.shape[0] * B.shape[0], A.shape[1]))
    lib().orc_khatri_rao_f64(_ptr(A), A.shape[0], _ptr(B), B.shape[0], A.shape[1], _ptr(out))
    return out


def gram(F: np.ndarray) -> np.ndarray:
    """Restated ``compute_gram_matrix`` (cp/helpers.rs:434-452)."""
    F = np.ascontiguousarray(F, dtype=np.float64)
    G = np.zeros((F.shape[1], F.shape[1]))
    lib().orc_gram_f64(_ptr(F), F.shape[0], F.shape[1], _ptr(G))
    return G


def solve(M: np.ndarray, G: np.ndarray) -> np.ndarray:
    """Restated ``solve_least_squares`` (cp/helpers.rs:455-495), FP64."""
    M = np.ascontiguousarray(M, dtype=np.float64)
    G = np.ascontiguousarray(G, dtype=np.float64)
    out = np.zeros_like(M)
    rc = lib().orc_solve_f64(_ptr(M), M.shape[0], _ptr(G), G.shape[0], _ptr(out))
    if rc:
        raise np.linalg.LinAlgError("oracle solve: Gram not positive definite")
    return out


REASONS = ("MaxIterations", "FitTolerance", "Oscillation", "TimeLimit")


def cp_als(X: np.ndarray, rank: int, max_iters: int, tol: float, init_factors,
           faithful: bool = False):
    """Restated ``tenrso_decomp::cp_als`` (cp/core.rs:59-182) from injected
    factors. Returns (factors, info dict)."""
    dt = X.dtype
    X = np.ascontiguousarray(X)
    shape = np.asarray(X.shape, dtype=np.int64)
    flat = np.concatenate([np.ascontiguousarray(f, dtype=dt).ravel() for f in init_factors])
    hist = np.zeros(max(max_iters, 1), dtype=dt)
    iters = C.c_int(0)
    reason = C.c_int(0)
    osc = C.c_int(0)
    ctype = C.c_float if dt == np.float32 else C.c_double
    change = ctype(0)
    fit = ctype(0)
    fn = lib().orc_cp_als_f32 if dt == np.float32 else lib().orc_cp_als_f64
    rc = fn(_ptr(X), X.ndim, _ptr(shape), rank, max_iters, float(tol), _ptr(flat), _ptr(hist),
            C.byref(iters), C.byref(reason), C.byref(osc), C.byref(change), C.byref(fit),
            int(faithful))
    if rc == -10:
        raise ValueError(f"Invalid rank: {rank}")
    if rc == -11:
        raise ValueError(f"Invalid tolerance: {tol}")
    if rc:
        raise np.linalg.LinAlgError(f"oracle cp_als failed: {rc}")
    out, off = [], 0
    for n in X.shape:
        out.append(flat[off:off + n * rank].reshape(n, rank).copy())
        off += n * rank
    info = dict(fit=float(fit.value), iters=iters.value, reason=REASONS[reason.value],
                oscillation_count=osc.value, oscillated=osc.value > 0,
                final_fit_change=float(change.value), fit_history=hist[:iters.value].copy())
    return out, info


def tikhonov_penalty(n: int, order: int) -> np.ndarray:
    """The matrix apply_tikhonov_to_gram (cp/helpers.rs:630-700) adds, per
    unit lambda: order 0 I; order 1 D1^T D1 (nothing for n < 2); order >= 2
    the reference's banded form with diagonal 1, 5, 6.., 5, 1, first
    off-diagonal -2, -4.., -4, -2, second off-diagonal 1 (I for n < 3)."""
    P = np.zeros((n, n))
    if order == 0:
        return np.eye(n)
    if order == 1:
        if n >= 2:
            for i in range(n):
                P[i, i] = 1.0 if i in (0, n - 1) else 2.0
                if i + 1 < n:
                    P[i, i + 1] = P[i + 1, i] = -1.0
        return P
    if n < 3:
        return np.eye(n)
    for i in range(n):
        P[i, i] = 1.0 if i in (0, n - 1) else (5.0 if i in (1, n - 2) else 6.0)
        if i + 1 < n:
            P[i, i + 1] = P[i + 1, i] = -2.0 if i in (0, n - 2) else -4.0
        if i + 2 < n:
            P[i, i + 2] = P[i + 2, i] = 1.0
    return P


def orthonormalize(F: np.ndarray) -> np.ndarray:
    """orthonormalize_factor (cp/helpers.rs:582-607): the thin Q of a QR
    factorization. scirs2-linalg's QR leaves the signs to its algorithm; Q is
    taken here with a positive diagonal in R (the unique such QR)."""
    q, r = np.linalg.qr(F)
    d = np.sign(np.diag(r))
    d[d == 0] = 1.0
    return q * d[None, :]


def cp_als_constrained(X: np.ndarray, rank: int, max_iters: int, tol: float, init_factors,
                       l2: float = 0.0, l1: float = 0.0, nonneg: bool = False,
                       orthogonal: bool = False, tikhonov=None):
    """Restated ``cp_als_constrained`` (cp/core.rs:225-400) in FP64 from
    injected factors, for small tensors: per mode MTTKRP (the restated C
    kernel), Hadamard of the other Grams, ridge l2 on its diagonal
    (core.rs:336-343), the restated solve, soft threshold by l1
    (helpers.rs:610-623), projection onto >= 0 (core.rs:356-359), the QR
    orthonormalization (core.rs:361-364); tikhonov = (lambda, order) with
    order > 0 replaces the ridge by lambda * tikhonov_penalty (core.rs:327-334);
    the fit and stopping rules of core.rs:366-392 (the same as cp_als). The
    input non-negativity check and the initial projection (core.rs:265-276)
    are applied too. Returns (factors, info dict)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    if nonneg and (X < 0).any():
        raise ValueError("Non-negative constraint violated: input tensor contains negative values")
    U = [np.array(f, dtype=np.float64) for f in init_factors]
    if nonneg:
        U = [np.maximum(f, 0.0) for f in U]
    xn = float(np.sum(X * X))
    prev_fit, fit, osc, change, reason = 0.0, 0.0, 0, 0.0, "MaxIterations"
    hist, iters = [], 0
    for it in range(max_iters):
        iters = it + 1
        for n in range(X.ndim):
            M = mttkrp(X, U, n)
            G = np.ones((rank, rank))
            for m in range(X.ndim):
                if m != n:
                    G *= gram(U[m])
            if tikhonov is not None and tikhonov[1] > 0:
                G += tikhonov[0] * tikhonov_penalty(rank, tikhonov[1])
            elif l2 > 0.0:
                G[np.diag_indices(rank)] += l2
            U[n] = solve(M, G)
            if l1 > 0.0:
                U[n] = np.where(U[n] > l1, U[n] - l1, np.where(U[n] < -l1, U[n] + l1, 0.0))
            if nonneg:
                U[n] = np.maximum(U[n], 0.0)
            if orthogonal:
                U[n] = orthonormalize(U[n])
        # compute_fit (helpers.rs:513-579)
        inner = float(np.sum(mttkrp(X, U, 0) * U[0]))
        H = np.ones((rank, rank))
        for f in U:
            H *= gram(f)
        err = np.sqrt(max(xn + float(H.sum()) - 2.0 * inner, 0.0))
        fit = min(max(1.0 - err / np.sqrt(xn), 0.0), 1.0)
        hist.append(fit)
        if it > 0 and fit < prev_fit:
            osc += 1
        change = abs(fit - prev_fit)
        if it > 0 and change < tol:
            reason = "FitTolerance"
            break
        if osc > 5 and it > 10:
            reason = "Oscillation"
            break
        prev_fit = fit
    info = dict(fit=fit, iters=iters, reason=reason, oscillation_count=osc, oscillated=osc > 0,
                final_fit_change=change, fit_history=np.asarray(hist))
    return U, info


def coo_deduplicate(idx: np.ndarray, vals: np.ndarray):
    """Restated ``CooTensor::deduplicate`` (coo.rs:320-347)."""
    idx = np.ascontiguousarray(idx, dtype=np.int64).copy()
    vals = np.ascontiguousarray(vals, dtype=np.float32).copy()
    n = lib().orc_coo_dedup_f32(_ptr(idx), _ptr(vals), idx.shape[0], idx.shape[1])
    return idx[:n].copy(), vals[:n].copy()


def csf_from_coo(idx: np.ndarray, vals: np.ndarray, mode_order):
    """Restated ``CsfTensor::from_coo`` (csf.rs:137-264). Returns
    (fptr list, fids list, vals) with the reference's nnz-offset fptr."""
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    vals = np.ascontiguousarray(vals, dtype=np.float32)
    nnz, ndim = idx.shape
    mo = np.asarray(mode_order, dtype=np.int64)
    if mo.shape[0] != ndim:
        raise ValueError("Invalid mode order: length mismatch")
    fptr = np.zeros((ndim, nnz + 1), dtype=np.int64)
    fids = np.zeros((ndim, max(nnz, 1)), dtype=np.int64)
    vout = np.zeros(max(nnz, 1), dtype=np.float32)
    lens = np.zeros(2 * ndim, dtype=np.int64)
    rc = lib().orc_csf_from_coo_f32(_ptr(idx), _ptr(vals), nnz, ndim, _ptr(mo), _ptr(fptr),
                                    _ptr(fids), _ptr(vout), _ptr(lens))
    if rc:
        raise ValueError("Invalid mode order: not a permutation")
    fp = [fptr[l, :lens[2 * l]].copy() for l in range(ndim)]
    fi = [fids[l, :lens[2 * l + 1]].copy() for l in range(ndim)]
    nv = len(fi[-1]) if ndim > 1 else 0
    return fp, fi, vout[:nv].copy()


def nmode_product(X: np.ndarray, M: np.ndarray, mode: int) -> np.ndarray:
    """Restated ``nmode_product`` (nmode.rs:72-131) in FP64: unfold along
    `mode`, M . X_(mode), fold back with shape[mode] replaced by M's rows."""
    X = np.asarray(X, dtype=np.float64)
    M = np.asarray(M, dtype=np.float64)
    if not 0 <= mode < X.ndim:
        raise ValueError(f"Mode {mode} out of bounds for tensor with rank {X.ndim}")
    if M.shape[1] != X.shape[mode]:
        raise ValueError(f"Matrix columns ({M.shape[1]}) must match tensor mode-{mode} size "
                         f"({X.shape[mode]})")
    return np.moveaxis(np.tensordot(M, X, axes=(1, mode)), 0, mode)


def hicoo_from_coo(idx, vals, block_shape):
    """Restated ``HiCooTensor::from_coo`` (hicoo.rs:118-203): block
    coordinates i // b and local coordinates i % b, a stable sort by block
    coordinate (lexicographic, mode 0 first), cumulative block pointers.
    Returns (block_coords, block_ptrs, local_coords, values)."""
    idx = np.ascontiguousarray(idx, dtype=np.int64).reshape(len(vals), -1)
    vals = np.ascontiguousarray(vals, dtype=np.float32)
    bs = np.asarray(block_shape, dtype=np.int64)
    if len(vals) == 0:
        return (np.zeros((0, len(bs)), np.int64), np.zeros(1, np.int64),
                np.zeros((0, len(bs)), np.int64), vals.copy())
    blk = idx // bs
    loc = idx % bs
    # np.lexsort is stable; its last key is the primary one
    order = np.lexsort(tuple(blk[:, m] for m in range(blk.shape[1] - 1, -1, -1)))
    blk, loc, v = blk[order], loc[order], vals[order]
    new = np.ones(len(v), bool)
    new[1:] = np.any(blk[1:] != blk[:-1], axis=1)
    starts = np.flatnonzero(new)
    ptrs = np.append(starts, len(v)).astype(np.int64)
    return blk[starts], ptrs, loc, v


def csf_mttkrp(fptr, fids, vals, mode_order, shape, factors, threads: int = 1):
    """Restated 3-way CSF MTTKRP (fp32, rooted at mode_order[0]) over the
    reference CSF arrays of csf_from_coo; threads > 1 runs the roots in
    parallel (OpenMP), 1 serially. Returns the root mode's I x R result."""
    fs = [np.ascontiguousarray(f, dtype=np.float32) for f in factors]
    R = fs[0].shape[1]
    mo = list(mode_order)
    a = [np.ascontiguousarray(x, dtype=np.int64) for x in (fptr[0], fids[0], fptr[1], fids[1],
                                                           fids[2])]
    v = np.ascontiguousarray(vals, dtype=np.float32)
    out = np.zeros((shape[mo[0]], R), np.float32)
    lib().orc_csf_mttkrp_f32(len(a[1]), _ptr(a[0]), _ptr(a[1]), len(a[3]), _ptr(a[2]),
                             _ptr(a[3]), _ptr(a[4]), _ptr(v), _ptr(fs[mo[1]]), _ptr(fs[mo[2]]), R,
                             shape[mo[0]], _ptr(out), int(threads))
    return out


def coo_mttkrp(idx, vals, shape, factors, mode):
    """Sparse MTTKRP definition (no reference implementation), FP64."""
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    fs = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
    shp = np.asarray(shape, dtype=np.int64)
    R = fs[0].shape[1]
    out = np.zeros((shape[mode], R))
    lib().orc_coo_mttkrp_f64(_ptr(idx), _ptr(vals), idx.shape[0], idx.shape[1], _ptr(shp),
                             _ptr_array(fs), R, mode, _ptr(out))
    return out


def compute_fit(X: np.ndarray, factors, xnorm_sq: float) -> float:
    """Restated ``compute_fit`` (cp/helpers.rs:513-530) in FP64:
    ||Xhat||^2 from the Hadamard of the factor Grams (helpers.rs:533-556),
    <X, Xhat> from the mode-0 MTTKRP of the factors (helpers.rs:558-579)."""
    R = factors[0].shape[1]
    H = np.ones((R, R))
    for f in factors:
        H *= gram(f)
    inner = float(np.sum(mttkrp(X, factors, 0) * factors[0]))
    err = np.sqrt(max(xnorm_sq + float(H.sum()) - 2.0 * inner, 0.0))
    return min(max(1.0 - err / np.sqrt(xnorm_sq), 0.0), 1.0)


INIT_STRATEGIES = ("random", "random_normal", "svd", "nnsvd", "leverage_score")


def initialize_factors(X: np.ndarray, rank: int, strategy: str, seed: int):
    """Restated ``initialize_factors`` (cp/helpers.rs:192-377) in FP64 with
    the library's seeded streams in place of thread_rng: U(0,1) on stream
    200 + n (:215-222), N(0,1) on 400 + n (:223-231), the N(0, 0.01) padding
    of the SVD-based strategies on 500 + n. The SVD is numpy's (LAPACK gesdd)
    thin SVD of the mode-n unfolding; each u_r is oriented so that its
    largest-magnitude entry is positive (first such entry on ties) and v_r
    with it. Svd :232-263, Nnsvd :264-317, LeverageScore :318-373."""
    from tenrso_b200 import synth
    X = np.asarray(X, dtype=np.float64)
    out = []
    for n, I in enumerate(X.shape):
        if strategy == "random":
            out.append(synth.uniform(seed, 200 + n, (I, rank)))
            continue
        if strategy == "random_normal":
            out.append(synth.normal(seed, 400 + n, (I, rank)))
            continue
        Xn = np.moveaxis(X, n, 0).reshape(I, -1)
        u, s, vt = np.linalg.svd(Xn, full_matrices=False)
        k = min(rank, u.shape[1], vt.shape[0])
        for r in range(k):
            i = int(np.argmax(np.abs(u[:, r])))
            if u[i, r] < 0:
                u[:, r] *= -1.0
                vt[r] *= -1.0
        F = np.zeros((I, rank))
        pad = synth.normal(seed, 500 + n, (I, rank - k)) * 0.01 if rank > k else None
        if strategy == "svd":
            F[:, :k] = u[:, :k]
            if pad is not None:
                F[:, k:] = pad
        elif strategy == "nnsvd":
            for r in range(k):
                up, un = np.maximum(u[:, r], 0), np.maximum(-u[:, r], 0)
                vp, vn = np.maximum(vt[r], 0), np.maximum(-vt[r], 0)
                pp = np.linalg.norm(up) * np.linalg.norm(vp)
                nn = np.linalg.norm(un) * np.linalg.norm(vn)
                F[:, r] = up * np.sqrt(s[r] * pp) if pp >= nn else un * np.sqrt(s[r] * nn)
            if pad is not None:
                F[:, k:] = np.abs(pad)
        elif strategy == "leverage_score":
            lev = np.sum(u[:, :k] ** 2, axis=1) / k
            total = lev.sum()
            if total > np.finfo(np.float32).eps:
                lev = lev / total
            F[:, :k] = u[:, :k] * np.sqrt(s[:k]) * np.sqrt(lev * I)[:, None]
            if pad is not None:
                F[:, k:] = pad * lev[:, None]
        else:
            raise ValueError(f"unknown strategy {strategy!r}")
        out.append(F)
    return out


def cp_als_accelerated(X: np.ndarray, rank: int, max_iters: int, tol: float, init_factors,
                       trace=None):
    """Restated ``cp_als_accelerated`` (cp/advanced.rs:51-213) in FP64 from
    injected factors: per mode the MTTKRP, Gram-Hadamard and solve of
    cp_als, then ``line_search_cp`` (helpers.rs:130-189: the fit of
    prev + a (new - prev) for a in 0.25, 0.5, 0.75, 1, 1.25, the first best
    kept), then from the second iteration on the extrapolation
    new += a_ls * alpha * (new - prev), prev being the factor before the
    previous update. After each sweep: the fit, the adaptive alpha (x1.05 up
    to 0.9 when the fit rose, else x0.7 down to 0.1 and one more oscillation;
    stop at > 5 oscillations after iteration 10), and the relative-change
    tolerance |fit - prev| / (|prev| + 1e-10) < tol. Returns (factors, info).
    With `trace` a list, each line search appends (iteration, mode, chosen a,
    the five trial fits)."""
    if rank == 0:
        raise ValueError(f"Invalid rank: {rank}")
    if not (0.0 < tol < 1.0):
        raise ValueError(f"Invalid tolerance: {tol}")
    X = np.ascontiguousarray(X, dtype=np.float64)
    U = [np.array(f, dtype=np.float64) for f in init_factors]
    prev = [f.copy() for f in U]
    alpha, alpha_max, alpha_min = 0.5, 0.9, 0.1
    xn = float(np.sum(X * X))
    prev_fit, fit, osc, change, reason = 0.0, 0.0, 0, 0.0, "MaxIterations"
    hist, iters = [], 0
    alphas = (0.25, 0.5, 0.75, 1.0, 1.25)
    for it in range(max_iters):
        iters = it + 1
        for n in range(X.ndim):
            M = mttkrp(X, U, n)
            G = np.ones((rank, rank))
            for m in range(X.ndim):
                if m != n:
                    G *= gram(U[m])
            new = solve(M, G)
            best_a, best_fit, fits = 1.0, -np.inf, []
            for a in alphas:
                test = list(U)
                test[n] = prev[n] + a * (new - prev[n])
                f = compute_fit(X, test, xn)
                fits.append(f)
                if f > best_fit:
                    best_fit, best_a = f, a
            if trace is not None:
                trace.append((it, n, best_a, fits))
            if it > 0:
                new = new + best_a * alpha * (new - prev[n])
            prev[n] = U[n].copy()
            U[n] = new
        fit = compute_fit(X, U, xn)
        hist.append(fit)
        if it > 0:
            if fit > prev_fit:
                alpha = min(alpha * 1.05, alpha_max)
            else:
                alpha = max(alpha * 0.7, alpha_min)
                osc += 1
                if osc > 5 and it > 10:
                    reason = "Oscillation"
                    break
        if it > 0:
            change = abs(fit - prev_fit)
            if change / (abs(prev_fit) + 1e-10) < tol:
                reason = "FitTolerance"
                break
        prev_fit = fit
    info = dict(fit=fit, iters=iters, reason=reason, oscillation_count=osc, oscillated=osc > 0,
                final_fit_change=change, fit_history=np.asarray(hist))
    return U, info


def cp_als_coo(idx, vals, shape, rank: int, max_iters: int, tol: float, init_factors):
    """CP-ALS of a sparse tensor given as COO, in FP64: the loop of
    ``cp_als`` (cp/core.rs:59-182; mode order, solve_least_squares restated
    as the oracle's FP64 solve, fit of helpers.rs:513-530, stopping rules)
    with every MTTKRP the FP64 sparse definition (coo_mttkrp) instead of the
    dense unfolding. tenrso has no sparse cp_als: this is its dense loop on
    the nonzeros, for tensors too large to densify. Returns (factors, info)."""
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    U = [np.array(f, dtype=np.float64) for f in init_factors]
    N = len(shape)
    xn = float(vals @ vals)
    prev_fit, fit, osc, change, reason = 0.0, 0.0, 0, 0.0, "MaxIterations"
    hist, iters = [], 0
    for it in range(max_iters):
        iters = it + 1
        M = None
        for n in range(N):
            M = coo_mttkrp(idx, vals, shape, U, n)
            G = np.ones((rank, rank))
            for m in range(N):
                if m != n:
                    G *= gram(U[m])
            U[n] = solve(M, G)
        # <X, Xhat> from the last mode's MTTKRP (equal to compute_inner_product)
        inner = float(np.sum(M * U[N - 1]))
        H = np.ones((rank, rank))
        for f in U:
            H *= gram(f)
        err = np.sqrt(max(xn + float(H.sum()) - 2.0 * inner, 0.0))
        fit = min(max(1.0 - err / np.sqrt(xn), 0.0), 1.0)
        hist.append(fit)
        if it > 0 and fit < prev_fit:
            osc += 1
        change = abs(fit - prev_fit)
        if it > 0 and change < tol:
            reason = "FitTolerance"
            break
        if osc > 5 and it > 10:
            reason = "Oscillation"
            break
        prev_fit = fit
    info = dict(fit=fit, iters=iters, reason=reason, oscillation_count=osc, oscillated=osc > 0,
                final_fit_change=change, fit_history=np.asarray(hist))
    return U, info


def cp_reconstruct(factors, weights=None):
    """Restated ``tenrso_kernels::cp_reconstruct`` (outer.rs:223-274), FP64."""
    fs = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
    shape = np.asarray([f.shape[0] for f in fs], dtype=np.int64)
    R = fs[0].shape[1]
    out = np.zeros(tuple(shape))
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    lib().orc_cp_reconstruct_f64(_ptr_array(fs), len(fs), _ptr(shape), R,
                                 None if w is None else _ptr(w), _ptr(out))
    return out


def cp_reconstruction_grad(factors, grad_output, weights=None):
    """Restated ``CpReconstructionGrad::compute_factor_gradients``
    (tenrso-ad/src/grad.rs:81-120): dL/dU_n = unfold(G, n) . KR_{!=n} . diag(w)."""
    G = np.ascontiguousarray(grad_output, dtype=np.float64)
    out = []
    for n in range(G.ndim):
        g = mttkrp(G, factors, n)
        if weights is not None:
            g = g * np.asarray(weights, dtype=np.float64)[None, :]
        out.append(g)
    return out


def cp_loss_grad_vjp(X, factors, reg: float):
    """CPU VJP of L = ||X - [[U]]||^2 + reg * sum ||U_n||^2 in FP64: restated
    cp_reconstruct, G = 2 (Xhat - X), restated CpReconstructionGrad on G, plus
    2 reg U_n. Returns (loss, [dL/dU_n])."""
    Xd = np.asarray(X, dtype=np.float64)
    fs = [np.asarray(f, dtype=np.float64) for f in factors]
    Xh = cp_reconstruct(fs)
    D = Xh - Xd
    loss = float(np.sum(D * D) + reg * sum(float(np.sum(f * f)) for f in fs))
    grads = cp_reconstruction_grad(fs, 2.0 * D)
    return loss, [g + 2.0 * reg * f for g, f in zip(grads, fs)]


def cp_slice_sqerr(X, factors, mode: int, index: int) -> float:
    """sum over the slice i_mode = index of (X - Xhat)^2, FP64."""
    Xd = np.ascontiguousarray(X, dtype=np.float64)
    fs = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
    shp = np.asarray(Xd.shape, dtype=np.int64)
    return float(lib().orc_cp_slice_sqerr_f64(_ptr(Xd), Xd.ndim, _ptr(shp), _ptr_array(fs), fs[0].shape[1], mode, index))


def fd_grad_entries(X, factors, reg: float, mode: int, entries, h: float = 1e-6):
    """FP64 central differences of L = ||X - [[U]]||^2 + reg sum ||U||^2 in the
    entries (i, r) of U_mode, each from the loss restricted to slice i (the
    only part of ||X - Xhat||^2 the entry changes)."""
    fs = [np.array(f, dtype=np.float64) for f in factors]
    out = []
    for i, r in entries:
        u0 = fs[mode][i, r]
        fs[mode][i, r] = u0 + h
        lp = cp_slice_sqerr(X, fs, mode, i) + reg * (u0 + h) ** 2
        fs[mode][i, r] = u0 - h
        lm = cp_slice_sqerr(X, fs, mode, i) + reg * (u0 - h) ** 2
        fs[mode][i, r] = u0
        out.append((lp - lm) / (2.0 * h))
    return np.array(out)


def csf_to_coo(fptr, fids, vals, mode_order):
    """A correct inverse of the reference CSF layout (every fptr level holds
    nnz offsets into the sorted entry list). The reference's own CsfIterator
    (csf.rs:423-495) mis-reconstructs fibers holding more than one nonzero,
    so it is not used as an oracle."""
    ndim = len(mode_order)
    nnz = len(fids[-1])
    out = np.zeros((nnz, ndim), dtype=np.int64)
    pos = np.arange(nnz)
    for level in range(ndim - 1):
        f = np.searchsorted(np.asarray(fptr[level]), pos, side="right") - 1
        out[:, mode_order[level]] = np.asarray(fids[level])[f]
    out[:, mode_order[-1]] = np.asarray(fids[-1])
    return out, np.asarray(vals)

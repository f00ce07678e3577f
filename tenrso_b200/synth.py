"""Seeded synthetic inputs for the CP-ALS workloads.

Every random number comes from one counter-based generator (SplitMix64 of
``key + counter * golden``), so a (seed, stream, counter) triple names one
value on any machine. tenrso itself draws from an unseeded ``thread_rng``
(``crates/tenrso-decomp/src/cp/helpers.rs:212-222``), so its streams cannot be
reproduced; these generators stand in for it on both sides of every parity
test. Workloads:

* ``dense_lowrank`` — sum of R rank-1 terms plus relative Gaussian noise
  (64^3 R=8 with N(0,1) factors and 1% noise; 256^3 R=64 with U(0,1) factors
  and 0.5% noise).
* ``zipf_coo`` — 3-way sparse COO with per-mode Zipf(s) indices over a seeded
  permutation, trimmed so that deduplication leaves exactly ``nnz`` entries.
* ``batched_instances`` — many small low-rank tensors of uneven shape/rank.
* ``init_factors`` — U(0,1) factor initialisation (tenrso's
  ``InitStrategy::Random``).
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def _key(seed: int, stream: int) -> np.uint64:
    with np.errstate(over="ignore"):
        s = np.array([(seed * 0x100000001B3 + stream * 0x2545F4914F6CDD1D) & (2**64 - 1)],
                     dtype=np.uint64)
        return _mix(s + _GOLDEN)[0]


def raw_u64(seed: int, stream: int, n: int, start: int = 0) -> np.ndarray:
    """n 64-bit words: splitmix64(key + (start+i) * golden)."""
    k = _key(seed, stream)
    with np.errstate(over="ignore"):
        ctr = np.arange(start, start + n, dtype=np.uint64)
        return _mix(k + ctr * _GOLDEN)


def uniform(seed: int, stream: int, shape, start: int = 0) -> np.ndarray:
    """U[0,1) doubles (53-bit)."""
    n = int(np.prod(shape))
    u = (raw_u64(seed, stream, n, start) >> np.uint64(11)).astype(np.float64)
    return (u * (1.0 / 9007199254740992.0)).reshape(shape)


def normal(seed: int, stream: int, shape) -> np.ndarray:
    """N(0,1) doubles by Box-Muller on two independent uniform streams."""
    n = int(np.prod(shape))
    u1 = 1.0 - uniform(seed, stream, (n,))          # (0, 1]
    u2 = uniform(seed, stream + 0x5151, (n,))
    return (np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)).reshape(shape)


def _outer_sum(factors) -> np.ndarray:
    """sum_r outer(U_0[:,r], ..., U_{N-1}[:,r]) in float64 via one GEMM."""
    shape = [f.shape[0] for f in factors]
    R = factors[0].shape[1]
    kr = factors[1]
    for f in factors[2:]:
        kr = (kr[:, None, :] * f[None, :, :]).reshape(-1, R)
    return (factors[0] @ kr.T).reshape(shape)


def dense_lowrank(shape, rank: int, seed: int, dist: str = "normal",
                  noise: float = 0.01, dtype=np.float32):
    """Tensor = sum of `rank` rank-1 terms (factor entries N(0,1) or U(0,1))
    plus i.i.d. Gaussian noise of std ``noise * ||X0|| / sqrt(|X|)``."""
    gen = normal if dist == "normal" else uniform
    fs = [gen(seed, 100 + m, (n, rank)) for m, n in enumerate(shape)]
    X0 = _outer_sum(fs)
    sigma = noise * np.linalg.norm(X0.ravel()) / np.sqrt(X0.size)
    X = X0 + sigma * normal(seed, 999, X0.shape)
    return X.astype(dtype), fs


def init_factors(shape, rank: int, seed: int, dtype=np.float32):
    """U(0,1) initial factors (tenrso InitStrategy::Random, helpers.rs:215-222)."""
    return [uniform(seed, 200 + m, (n, rank)).astype(dtype) for m, n in enumerate(shape)]


def zipf_indices(seed: int, stream: int, size: int, s: float, n: int, start: int = 0):
    """n draws of pi[Zipf(s) over 1..size - 1] for a seeded permutation pi."""
    ranks = np.arange(1, size + 1, dtype=np.float64)
    cdf = np.cumsum(ranks ** (-s))
    cdf /= cdf[-1]
    u = uniform(seed, stream, (n,), start)
    z = np.minimum(np.searchsorted(cdf, u, side="right"), size - 1)
    perm = np.argsort(raw_u64(seed, stream + 0x777, size), kind="stable")
    return perm[z].astype(np.int64)


def zipf_coo(shape, nnz: int, seed: int, s: float = 1.2, batch: int | None = None):
    """Raw COO (with duplicates, in draw order) whose deduplication leaves
    exactly ``nnz`` distinct coordinates. Returns (idx[n,ndim] int64,
    vals[n] float32, n_duplicates)."""
    ndim = len(shape)
    batch = batch or max(nnz // 4, 1024)
    strides = np.ones(ndim, dtype=np.uint64)
    for d in range(ndim - 2, -1, -1):
        strides[d] = strides[d + 1] * np.uint64(shape[d + 1])
    idx_parts, drawn = [], 0
    while True:
        cols = [zipf_indices(seed, 10 + d, shape[d], s, batch, drawn) for d in range(ndim)]
        idx_parts.append(np.stack(cols, axis=1))
        drawn += batch
        idx = np.concatenate(idx_parts) if len(idx_parts) > 1 else idx_parts[0]
        keys = (idx.astype(np.uint64) * strides[None, :]).sum(axis=1)
        uniq, first = np.unique(keys, return_index=True)
        if uniq.shape[0] >= nnz:
            break
    first.sort()
    cut = int(first[nnz - 1]) + 1          # raw prefix holding exactly nnz keys
    idx = np.ascontiguousarray(idx[:cut])
    vals = uniform(seed, 50, (cut,)).astype(np.float32)
    return idx, vals, cut - nnz


def batched_instances(count: int, seed: int, nmin: int = 16, nmax: int = 96,
                      rmin: int = 4, rmax: int = 16, noise: float = 0.01):
    """`count` independent 3-way low-rank N(0,1) tensors plus `noise` relative
    Gaussian noise; mode sizes ~ U{nmin..nmax}, ranks ~ U{rmin..rmax}."""
    sz = nmin + (raw_u64(seed, 1, count * 3) % np.uint64(nmax - nmin + 1)).astype(np.int64)
    rk = rmin + (raw_u64(seed, 2, count) % np.uint64(rmax - rmin + 1)).astype(np.int64)
    out = []
    for b in range(count):
        shape = tuple(int(x) for x in sz[3 * b:3 * b + 3])
        X, _ = dense_lowrank(shape, int(rk[b]), seed * 1000003 + b, "normal", noise)
        init = init_factors(shape, int(rk[b]), seed * 1000003 + b)
        out.append((X, int(rk[b]), init))
    return out

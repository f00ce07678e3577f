"""CP-ALS over several processes by slabs of mode 0 (one process per GPU).

Rank p holds the slab X[rows_p, ...] of mode 0 (rows_p = a contiguous range,
as even as possible), its rows of U_0, and every other factor in full. One
sweep is cp_als's (crates/tenrso-decomp/src/cp/core.rs:59-182) with the
exchanges the partition needs:

  mode 0      M_0 rows from the local slab alone (they are complete), the
              solve of those rows with the shared G_0, and one all-reduce of
              the R x R partial Grams U_0[rows_p]^T U_0[rows_p];
  mode n > 0  the local slab's partial M_n (I_n x R), one all-reduce (sum, in
              FP64) to the full M_n, then the same solve on every rank
              (U_n stays replicated).

||X||^2 is one all-reduce at the start; the fit uses the last mode's full
M_n, and rank 0's fit is broadcast each sweep, so that every rank takes the
same stop decision (the replicated factors agree to rounding). U_0 is
all-gathered once at the end. The collectives go through
torch.distributed (NCCL between GPUs; gloo, on host copies, between processes
that share a GPU or run on CPU).

The compute is a backend: DeviceBackend runs the library's MTTKRP and FP64
solve kernels on this process's GPU. Any object with the same methods (put,
mttkrp, solve, norm_sq, to_host) can stand in for it.

The same partition serves the other sharded paths:
  cp_als_sparse_sharded   a COO tensor, each rank keeping the nonzeros of its
                          mode-0 slab (SparseDeviceBackend: the CSF MTTKRP);
  loss_grad_sharded       the loss and every gradient of ||X - [[U]]||^2 +
                          reg sum ||U_n||^2: partial MTTKRPs of modes >= 1 and
                          the slab scalars summed, dL/dU_0 rows all-gathered;
  batched_cp_als_sharded  independent instances partitioned by work, no
                          collective.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import TenrsoError, check
from .dense import REASONS, ConvergenceInfo, _ctx_handle, _i64, _prec, _ptr


def slab_rows(n_rows: int, world: int, rank: int):
    """[start, stop) of rank's slab: the first n_rows % world ranks take one
    row more."""
    base, extra = divmod(n_rows, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


class DeviceBackend:
    """The library's kernels on this process's GPU (torch CUDA tensors)."""

    def __init__(self, precision: str = "fp32", ctx=None):
        import torch
        self.torch = torch
        self.precision = precision
        self.ctx = ctx

    def put(self, a: np.ndarray):
        return self.torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()

    def to_host(self, t) -> np.ndarray:
        return t.detach().cpu().numpy()

    def mttkrp(self, X, factors, mode: int):
        """M_mode of the local slab X (device tensor) with the given factors."""
        R = factors[0].shape[1]
        out = self.torch.empty(X.shape[mode], R, dtype=self.torch.float32, device=X.device)
        if X.numel() == 0:
            out.zero_()
            return out
        shp = _i64(list(X.shape))
        ptrs = (C.c_void_p * len(factors))(*[f.data_ptr() for f in factors])
        check(_lib.load().tsr_mttkrp_dev_f32(_ctx_handle(self.ctx), C.c_void_p(X.data_ptr()),
                                             X.dim(), _ptr(shp), ptrs, R, mode,
                                             _prec(self.precision), C.c_void_p(out.data_ptr())))
        return out

    def solve(self, M, H: np.ndarray):
        """(U = M H^-1, U^T U in FP64, <M, U>) on the device."""
        torch = self.torch
        rows, R = M.shape
        U = torch.empty(rows, R, dtype=torch.float32, device=M.device)
        dH = torch.from_numpy(np.ascontiguousarray(H, dtype=np.float64)).to(M.device)
        G = torch.empty(R, R, dtype=torch.float64, device=M.device)
        inner = C.c_double(0.0)
        ridge = C.c_int(0)
        check(_lib.load().tsr_als_solve_dev_f32(
            _ctx_handle(self.ctx), C.c_void_p(M.data_ptr() if rows else 0), rows, R,
            C.c_void_p(dH.data_ptr()), C.c_void_p(U.data_ptr() if rows else 0),
            C.c_void_p(G.data_ptr()), C.byref(inner), C.byref(ridge)))
        return U, G.cpu().numpy(), float(inner.value)

    def norm_sq(self, X) -> float:
        return float(X.double().pow(2).sum().item()) if X.numel() else 0.0


def _allreduce_sum(x, dist, group):
    """Sum over ranks of a numpy array or torch tensor (FP64 on the wire)."""
    import torch
    if dist is None:
        return x
    backend = dist.get_backend(group)
    if isinstance(x, np.ndarray):
        t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64))
        if backend == "nccl":
            t = t.cuda()
        dist.all_reduce(t, group=group)
        return t.cpu().numpy()
    t = x.double()
    if backend != "nccl" and t.is_cuda:
        h = t.cpu()
        dist.all_reduce(h, group=group)
        t = h.to(x.device)
    else:
        dist.all_reduce(t, group=group)
    return t.to(x.dtype)


def _broadcast_scalar(v: float, dist, group) -> float:
    """Rank 0's value of v on every rank."""
    import torch
    if dist is None:
        return v
    t = torch.tensor([v], dtype=torch.float64)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.broadcast(t, src=0, group=group)
    return float(t.item())


@dataclass
class ShardedCpDecomp:
    factors: List[np.ndarray]
    fit: float
    iters: int
    convergence: ConvergenceInfo


def cp_als_sharded(X_slab, n_rows_total: int, rank: int, max_iters: int, tol: float,
                   init_factors: Sequence[np.ndarray], backend=None, group=None,
                   dist=None) -> ShardedCpDecomp:
    """CP-ALS of the tensor whose mode-0 slab rows slab_rows(n_rows_total,
    world, me) this process holds in X_slab (host array or device tensor, the
    other modes complete). init_factors are the full initial factors (the same
    on every rank). Returns the full factors on every rank, with cp_als's fit
    history and stop reason (same validation: rank >= 1, 0 <= tol < 1)."""
    if dist is None:
        import torch.distributed as tdist
        dist = tdist if tdist.is_available() and tdist.is_initialized() else None
    world = dist.get_world_size(group) if dist else 1
    me = dist.get_rank(group) if dist else 0
    if rank == 0:
        raise TenrsoError(5, f"Invalid rank: {rank}")
    if not 0.0 <= tol < 1.0:
        raise TenrsoError(6, f"Invalid tolerance: {tol}")
    be = backend if backend is not None else DeviceBackend()
    r0, r1 = slab_rows(n_rows_total, world, me)
    X = X_slab if not isinstance(X_slab, np.ndarray) else be.put(X_slab)
    if X.shape[0] != r1 - r0:
        raise ValueError(f"slab has {X.shape[0]} rows, rank {me} of {world} owns {r1 - r0}")
    ndim = X.dim() if hasattr(X, "dim") else X.ndim
    R = rank
    U = [be.put(np.asarray(init_factors[0])[r0:r1])] + \
        [be.put(np.asarray(f)) for f in init_factors[1:]]
    grams = [np.zeros((R, R)) for _ in range(ndim)]
    g0 = be.to_host(U[0]).astype(np.float64)
    grams[0] = _allreduce_sum(g0.T @ g0, dist, group)
    for n in range(1, ndim):
        h = be.to_host(U[n]).astype(np.float64)
        grams[n] = h.T @ h
    xn = float(_allreduce_sum(np.array([be.norm_sq(X)]), dist, group)[0])
    hist, fit, prev_fit, change, osc = [], 0.0, 0.0, 0.0, 0
    reason, iters = 0, 0
    for it in range(max_iters):
        iters = it + 1
        inner = 0.0
        for n in range(ndim):
            H = np.ones((R, R))
            for m in range(ndim):
                if m != n:
                    H = H * grams[m]
            M = be.mttkrp(X, U, n)
            if n > 0:
                M = _allreduce_sum(M, dist, group)
            U[n], G, inner = be.solve(M, H)
            grams[n] = _allreduce_sum(G, dist, group) if n == 0 else G
        # fit of helpers.rs:513-530 from the last mode's full M and the Grams
        H = np.ones((R, R))
        for m in range(ndim):
            H = H * grams[m]
        err = np.sqrt(max(xn + float(H.sum()) - 2.0 * inner, 0.0))
        fit = min(max(1.0 - err / np.sqrt(xn), 0.0), 1.0) if xn > 0 else 0.0
        # the replicated solves may round differently on each rank (FP64
        # atomics): rank 0's fit drives every rank's stop decision
        fit = _broadcast_scalar(fit, dist, group)
        hist.append(fit)
        # cp_als's stopping rules (core.rs:145-166)
        if it > 0 and fit < prev_fit:
            osc += 1
        change = abs(fit - prev_fit)
        if it > 0 and change < tol:
            reason = 1
            break
        if osc > 5 and it > 10:
            reason = 2
            break
        prev_fit = fit
    # the full U_0 on every rank
    u0 = be.to_host(U[0])
    if dist is not None and world > 1:
        import torch
        counts = [slab_rows(n_rows_total, world, p) for p in range(world)]
        width = max(b - a for a, b in counts)
        buf = np.zeros((width, R), np.float32)
        buf[:u0.shape[0]] = u0
        t = torch.from_numpy(buf)
        if dist.get_backend(group) == "nccl":
            t = t.cuda()
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(parts, t, group=group)
        u0 = np.concatenate([p.cpu().numpy()[:b - a] for p, (a, b) in zip(parts, counts)])
    factors = [u0] + [be.to_host(u) for u in U[1:]]
    conv = ConvergenceInfo(fit_history=np.asarray(hist), reason=REASONS[reason],
                           oscillated=osc > 0, oscillation_count=osc, final_fit_change=change)
    return ShardedCpDecomp(factors=factors, fit=fit, iters=iters, convergence=conv)


# ---------------------------------------------------------------------------
# Sparse slabs: the nonzeros of a mode-0 slab, behind the same backend methods


class SparseSlab:
    """The nonzeros of rows [r0, r1) of mode 0, with mode-0 indices made
    local (i0 - r0); `sp` is the device tensor (None when the slab holds no
    nonzero). shape / ndim describe the local slab."""

    def __init__(self, indices: np.ndarray, values: np.ndarray, shape: Sequence[int], r0: int,
                 r1: int, ctx=None):
        idx = np.asarray(indices, np.int64).reshape(-1, len(shape))
        vals = np.asarray(values, np.float32)
        keep = (idx[:, 0] >= r0) & (idx[:, 0] < r1)
        idx = idx[keep].copy()
        idx[:, 0] -= r0
        vals = vals[keep]
        self.shape = [r1 - r0] + [int(s) for s in shape[1:]]
        self.ndim = len(shape)
        self.nnz = int(vals.size)
        # ||X||^2 of the merged tensor: duplicates summed in fp32 in their
        # order, as the device tensor merges them (coo.rs:320-347)
        merged = vals
        if self.nnz:
            keys = np.ravel_multi_index(tuple(idx.T), self.shape)
            order = np.argsort(keys, kind="stable")
            _, starts = np.unique(keys[order], return_index=True)
            merged = np.add.reduceat(vals[order], starts).astype(np.float32)
        self.norm_sq = float(np.sum(merged.astype(np.float64) ** 2))
        self.sp = None
        if self.nnz and self.shape[0] > 0:
            from .sparse import CooTensor, SparseTensor
            self.sp = SparseTensor(CooTensor(idx, vals, self.shape), ctx=ctx)

    def close(self):
        if self.sp is not None:
            self.sp.close()
            self.sp = None


class SparseDeviceBackend(DeviceBackend):
    """The library's CSF MTTKRP (tsr_mttkrp_csf_dev_f32) on this process's GPU
    for a SparseSlab; the FP64 solve as DeviceBackend."""

    def mttkrp(self, X: SparseSlab, factors, mode: int):
        torch = self.torch
        R = factors[0].shape[1]
        if X.sp is None:
            return torch.zeros(X.shape[mode], R, dtype=torch.float32, device=factors[-1].device)
        # the CSF MTTKRP writes every output row on the library context's own
        # stream and returns without synchronizing: order it against torch's
        # stream on both sides
        out = torch.empty(X.shape[mode], R, dtype=torch.float32, device=factors[-1].device)
        torch.cuda.synchronize()
        X.sp.mttkrp_dev([f.data_ptr() for f in factors], R, mode, out.data_ptr())
        torch.cuda.synchronize()
        return out

    def norm_sq(self, X: SparseSlab) -> float:
        return X.norm_sq


def cp_als_sparse_sharded(indices, values, shape, rank: int, max_iters: int, tol: float,
                          init_factors: Sequence[np.ndarray], backend=None, group=None,
                          dist=None) -> ShardedCpDecomp:
    """CP-ALS of a sparse tensor (COO: indices nnz x ndim, values) sharded by
    mode-0 slabs: each rank keeps the nonzeros of its rows slab_rows(shape[0],
    world, rank) and runs cp_als_sharded with the CSF MTTKRP as its compute.
    Equals cp_als on the tensor with its zeros (core.rs:59-182)."""
    if dist is None:
        import torch.distributed as tdist
        dist = tdist if tdist.is_available() and tdist.is_initialized() else None
    world = dist.get_world_size(group) if dist else 1
    me = dist.get_rank(group) if dist else 0
    r0, r1 = slab_rows(int(shape[0]), world, me)
    be = backend if backend is not None else SparseDeviceBackend()
    slab = SparseSlab(indices, values, shape, r0, r1,
                      ctx=getattr(be, "ctx", None)) if isinstance(be, SparseDeviceBackend) \
        else be.slab(indices, values, shape, r0, r1)
    try:
        return cp_als_sharded(slab, int(shape[0]), rank, max_iters, tol, init_factors, backend=be,
                              group=group, dist=dist)
    finally:
        if isinstance(slab, SparseSlab):
            slab.close()


# ---------------------------------------------------------------------------
# The loss / gradient of ||X - [[U]]||^2 + reg sum ||U_n||^2 by mode-0 slabs


def _all_gather_rows(u: np.ndarray, n_rows_total: int, dist, group) -> np.ndarray:
    """The full row-stacked matrix from every rank's slab rows."""
    import torch
    if dist is None:
        return u
    world = dist.get_world_size(group)
    if world == 1:
        return u
    counts = [slab_rows(n_rows_total, world, p) for p in range(world)]
    width = max(b - a for a, b in counts)
    buf = np.zeros((width, u.shape[1]), u.dtype)
    buf[:u.shape[0]] = u
    t = torch.from_numpy(buf)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    return np.concatenate([p.cpu().numpy()[:b - a] for p, (a, b) in zip(parts, counts)])


def loss_grad_sharded(X_slab, n_rows_total: int, factors: Sequence[np.ndarray], reg: float,
                      backend=None, group=None, dist=None):
    """(loss, [dL/dU_n]) of ||X - [[U]]||^2 + reg sum_n ||U_n||^2 with X held
    by mode-0 slabs (this rank: rows slab_rows(n_rows_total, world, rank)) and
    every factor replicated. Gram form, as tsr_cp_loss_grad_dev_f32:
      dL/dU_n = 2 (U_n H_n - M_n + reg U_n),  H_n = *_{m != n} U_m^T U_m,
      loss = ||X||^2 - 2 <M_0, U_0> + sum prod_n Gram_n + reg sum_n tr(Gram_n).
    Exchanges: the partial MTTKRPs M_n of modes n >= 1, U_0's partial Gram and
    the slab scalars are summed over ranks (FP64), dL/dU_0's rows all-gathered.
    Every rank returns the full loss and gradients (FP64 host arrays)."""
    if dist is None:
        import torch.distributed as tdist
        dist = tdist if tdist.is_available() and tdist.is_initialized() else None
    world = dist.get_world_size(group) if dist else 1
    me = dist.get_rank(group) if dist else 0
    be = backend if backend is not None else DeviceBackend()
    r0, r1 = slab_rows(n_rows_total, world, me)
    X = X_slab if not isinstance(X_slab, np.ndarray) else be.put(X_slab)
    if X.shape[0] != r1 - r0:
        raise ValueError(f"slab has {X.shape[0]} rows, rank {me} of {world} owns {r1 - r0}")
    N = len(factors)
    R = int(np.asarray(factors[0]).shape[1])
    if R == 0:
        raise TenrsoError(5, f"Invalid rank: {R}")
    U = [be.put(np.asarray(factors[0])[r0:r1])] + [be.put(np.asarray(f)) for f in factors[1:]]
    Uh = [np.asarray(be.to_host(u), np.float64) for u in U]
    grams = [u.T @ u for u in Uh]
    grams[0] = _allreduce_sum(grams[0], dist, group)
    M = []
    for n in range(N):
        m = np.asarray(be.to_host(be.mttkrp(X, U, n)), np.float64)
        M.append(m if n == 0 else _allreduce_sum(m, dist, group))
    scal = np.array([be.norm_sq(X), float(np.sum(M[0] * Uh[0]))])
    scal = _allreduce_sum(scal, dist, group)
    grads = []
    for n in range(N):
        H = np.ones((R, R))
        for m in range(N):
            if m != n:
                H = H * grams[m]
        grads.append(2.0 * (Uh[n] @ H - M[n] + reg * Uh[n]))
    H = np.ones((R, R))
    for g in grams:
        H = H * g
    loss = float(scal[0] - 2.0 * scal[1] + H.sum() + reg * sum(np.trace(g) for g in grams))
    grads[0] = _all_gather_rows(grads[0], n_rows_total, dist, group)
    return loss, grads


# ---------------------------------------------------------------------------
# Batched CP-ALS: independent instances partitioned over ranks


def partition_instances(work: Sequence[float], world: int) -> List[List[int]]:
    """Instance ids per rank: largest work first, each to the rank with the
    least work so far (ties to the lower rank); ids ascending within a rank."""
    order = sorted(range(len(work)), key=lambda i: (-float(work[i]), i))
    loads = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        p = min(range(world), key=lambda q: (loads[q], q))
        parts[p].append(i)
        loads[p] += float(work[i])
    return [sorted(p) for p in parts]


def batched_cp_als_sharded(tensors: Sequence[np.ndarray], ranks: Sequence[int], max_iters: int,
                           tol: float, inits: Sequence[Sequence[np.ndarray]], group=None,
                           dist=None, ctx=None):
    """This rank's share of a batch of independent CP-ALS instances (no
    collective): partition_instances by n0 n1 n2 R work, then one
    BatchedCpAls run over the rank's instances. Returns (ids, results) with
    results[k] the CpDecomp of instance ids[k]."""
    if dist is None:
        import torch.distributed as tdist
        dist = tdist if tdist.is_available() and tdist.is_initialized() else None
    world = dist.get_world_size(group) if dist else 1
    me = dist.get_rank(group) if dist else 0
    work = [float(np.prod(np.asarray(t).shape)) * r for t, r in zip(tensors, ranks)]
    ids = partition_instances(work, world)[me]
    if not ids:
        return [], []
    from .batched import BatchedCpAls
    b = BatchedCpAls([np.asarray(tensors[i], np.float32) for i in ids], [ranks[i] for i in ids],
                     ctx=ctx)
    try:
        out = b.cp_als(max_iters, tol, init=[inits[i] for i in ids])
    finally:
        b.close()
    return ids, out

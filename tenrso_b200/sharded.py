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
solve kernels on this process's GPU. Any object with the same four methods
(mttkrp, solve, norm_sq, to_host) can stand in for it.
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

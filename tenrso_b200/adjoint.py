"""Python mirror of tenrso's CP reconstruction and its gradient rule over the C ABI.

  cp_reconstruct          crates/tenrso-kernels/src/outer.rs:223-274
  CpReconstructionGrad    crates/tenrso-ad/src/grad.rs:41-150
                          (compute_factor_gradients, grad.rs:81-120)
  VjpOp.vjp               crates/tenrso-ad/src/vjp.rs:30-44
  AdOperation             crates/tenrso-ad/src/hooks.rs:44-80

The gradient of the reconstruction w.r.t. factor n is the MTTKRP of the
incoming gradient G with the other factors (times diag(weights)); the CUDA
library forms the Khatri-Rao rows on the fly and never stores them.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check
from .dense import Context, _ctx_handle, _f32, _i64, _prec, _ptr


def _host_factors(factors):
    fs = [_f32(f) for f in factors]
    for f in fs:
        if f.ndim != 2:
            raise ValueError("factor matrices must be 2-D")
    rows = _i64([f.shape[0] for f in fs]) if fs else _i64([0])
    cols = _i64([f.shape[1] for f in fs]) if fs else _i64([0])
    ptrs = (C.c_void_p * max(len(fs), 1))(*[f.ctypes.data for f in fs])
    return fs, rows, cols, ptrs


def cp_reconstruct(factors: Sequence, weights=None, ctx: Optional[Context] = None) -> np.ndarray:
    """X = sum_r w_r U_0[:, r] o ... o U_{N-1}[:, r] (shape = factor rows).
    Errors as tenrso's: "Need at least one factor matrix for CP reconstruction",
    "Factor {i} has {c} columns, expected {R}", "Weights length {n} must match rank {R}"."""
    fs, rows, cols, ptrs = _host_factors(factors)
    w = None if weights is None else _f32(weights).ravel()
    valid = len(fs) > 0 and all(f.shape[1] == fs[0].shape[1] for f in fs) and (
        w is None or w.size == fs[0].shape[1])
    out = np.zeros(tuple(f.shape[0] for f in fs) if fs else (0,), dtype=np.float32)
    h = _ctx_handle(ctx) if valid else None
    check(_lib.load().tsr_cp_reconstruct_f32(h, ptrs, len(fs), _ptr(rows), _ptr(cols),
                                             None if w is None else _ptr(w),
                                             0 if w is None else w.size, _ptr(out)))
    return out


def cp_reconstruct_dev(d_factors: Sequence[int], shape, rank: int, d_out: int,
                       d_weights: Optional[int] = None, ctx: Optional[Context] = None):
    """Device-pointer reconstruction into d_out (row-major, stream-ordered)."""
    shp = _i64(shape)
    ptrs = (C.c_void_p * max(len(d_factors), 1))(*d_factors)
    check(_lib.load().tsr_cp_reconstruct_dev_f32(_ctx_handle(ctx), ptrs, len(shape), _ptr(shp),
                                                 rank, C.c_void_p(d_weights) if d_weights
                                                 else None, C.c_void_p(d_out)))


def cp_residual_dev(d_tensor: int, shape, d_factors: Sequence[int], rank: int, d_out: int,
                    alpha: float = 2.0, d_weights: Optional[int] = None, want_sq: bool = True,
                    ctx: Optional[Context] = None) -> Optional[float]:
    """d_out = alpha * (Xhat - X); returns sum (Xhat - X)^2 (FP64) when want_sq."""
    shp = _i64(shape)
    ptrs = (C.c_void_p * max(len(d_factors), 1))(*d_factors)
    sq = C.c_double(0.0)
    check(_lib.load().tsr_cp_residual_dev_f32(_ctx_handle(ctx), C.c_void_p(d_tensor), len(shape),
                                              _ptr(shp), ptrs, rank,
                                              C.c_void_p(d_weights) if d_weights else None,
                                              float(alpha), C.c_void_p(d_out),
                                              C.byref(sq) if want_sq else None))
    return sq.value if want_sq else None


def reconstruction_grad_dev(d_grad: int, shape, d_factors: Sequence[int], rank: int,
                            d_outs: Sequence[int], d_weights: Optional[int] = None,
                            precision="fp32", ctx: Optional[Context] = None):
    """dL/dU_n = unfold(G, n) . KR_{m != n} . diag(w) into d_outs[n] (device)."""
    shp = _i64(shape)
    ptrs = (C.c_void_p * max(len(d_factors), 1))(*d_factors)
    optrs = (C.c_void_p * max(len(d_outs), 1))(*d_outs)
    check(_lib.load().tsr_cp_reconstruction_grad_dev_f32(
        _ctx_handle(ctx), C.c_void_p(d_grad), len(shape), _ptr(shp), ptrs, rank,
        C.c_void_p(d_weights) if d_weights else None, _prec(precision), optrs))


class CpReconstructionGrad:
    """Gradient context of the CP reconstruction (grad.rs:41-150).

    compute_factor_gradients(grad_output) returns [dL/dU_0, ..., dL/dU_{N-1}]
    for grad_output = dL/dX (the reconstructed tensor's gradient)."""

    def __init__(self, factors: Sequence, weights=None, precision="fp32",
                 ctx: Optional[Context] = None):
        self.factors = [_f32(f) for f in factors]
        self.weights = None if weights is None else _f32(weights).ravel()
        self.precision = precision
        self.ctx = ctx

    def compute_factor_gradients(self, grad_output) -> List[np.ndarray]:
        g = _f32(grad_output)
        fs, rows, cols, ptrs = _host_factors(self.factors)
        R = fs[0].shape[1] if fs else 0
        outs = [np.zeros((f.shape[0], R), dtype=np.float32) for f in fs]
        optrs = (C.c_void_p * max(len(outs), 1))(*[o.ctypes.data for o in outs])
        w = self.weights
        valid = (g.ndim == len(fs) and len(fs) >= 2 and
                 all(f.shape[1] == R for f in fs) and
                 all(f.shape[0] == g.shape[i] for i, f in enumerate(fs)) and
                 (w is None or w.size == R))
        h = _ctx_handle(self.ctx) if valid else None
        check(_lib.load().tsr_cp_reconstruction_grad_f32(
            h, _ptr(g), g.ndim, _ptr(_i64(g.shape) if g.ndim else _i64([0])), ptrs, len(fs),
            _ptr(rows), _ptr(cols), None if w is None else _ptr(w), 0 if w is None else w.size,
            _prec(self.precision), optrs))
        return outs

    def vjp(self, output_grad) -> List[np.ndarray]:
        """VjpOp::vjp (vjp.rs:43): the cotangent of each factor matrix."""
        return self.compute_factor_gradients(output_grad)


class CpReconstructionOp:
    """AdOperation (hooks.rs:44-80) of X = [[w; U_0, ..., U_{N-1}]]: forward
    reconstructs on the GPU, backward applies CpReconstructionGrad."""

    def __init__(self, factors: Sequence, weights=None, precision="fp32",
                 ctx: Optional[Context] = None):
        self.factors = [_f32(f) for f in factors]
        self.weights = weights
        self._grad = CpReconstructionGrad(self.factors, weights, precision, ctx)
        self.ctx = ctx

    def forward(self) -> List[np.ndarray]:
        return [cp_reconstruct(self.factors, self.weights, self.ctx)]

    def backward(self, output_grads: Sequence) -> List[np.ndarray]:
        if len(output_grads) != 1:
            raise ValueError("CpReconstructionOp has one output")
        return self._grad.compute_factor_gradients(output_grads[0])

    def name(self) -> str:
        return "cp_reconstruct"

    def num_inputs(self) -> int:
        return len(self.factors)

    def num_outputs(self) -> int:
        return 1


class DenseTensor:
    """A device tensor prepared for repeated MTTKRPs (per-mode unfoldings
    built once). The device buffer at d_tensor must outlive this object and
    stay unchanged."""

    def __init__(self, d_tensor: int, shape, precision="fp32", ctx: Optional[Context] = None):
        self.shape = tuple(int(s) for s in shape)
        self.ctx = ctx
        self._lib = _lib.load()
        h = C.c_void_p()
        check(self._lib.tsr_dense_create_dev_f32(_ctx_handle(ctx), C.c_void_p(d_tensor),
                                                 len(self.shape), _ptr(_i64(self.shape)),
                                                 _prec(precision), C.byref(h)))
        self.handle = h

    def loss_grad_dev(self, d_factors: Sequence[int], rank: int, reg: float,
                      d_grads: Sequence[int], want_loss: bool = True) -> Optional[float]:
        """||X - [[U]]||^2 + reg sum ||U_n||^2 and dL/dU_n into d_grads (device)."""
        ptrs = (C.c_void_p * len(d_factors))(*d_factors)
        gptrs = (C.c_void_p * len(d_grads))(*d_grads)
        loss = C.c_double(0.0)
        check(self._lib.tsr_cp_loss_grad_dev_f32(_ctx_handle(self.ctx), self.handle, ptrs, rank,
                                                 float(reg), gptrs,
                                                 C.byref(loss) if want_loss else None))
        return loss.value if want_loss else None

    def close(self):
        if getattr(self, "handle", None):
            self._lib.tsr_dense_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cp_loss_grad(tensor, factors: Sequence, reg: float, precision="fp32",
                 ctx: Optional[Context] = None):
    """Host convenience: (loss, [dL/dU_n]) of ||X - [[U]]||^2 + reg sum ||U_n||^2,
    staged through device buffers held by torch (device memory only)."""
    import torch
    X = torch.from_numpy(_f32(tensor)).cuda()
    fs = [torch.from_numpy(_f32(f)).cuda() for f in factors]
    gs = [torch.empty_like(f) for f in fs]
    R = fs[0].shape[1]
    torch.cuda.synchronize()
    d = DenseTensor(X.data_ptr(), X.shape, precision, ctx)
    try:
        loss = d.loss_grad_dev([f.data_ptr() for f in fs], R, reg, [g.data_ptr() for g in gs])
    finally:
        d.close()
    return loss, [g.cpu().numpy() for g in gs]

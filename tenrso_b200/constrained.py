"""cp_als_constrained over the C ABI: the dense CP-ALS sweep with a ridge (or
a Tikhonov finite-difference penalty) on the Gram, soft-thresholding,
non-negativity and orthonormalization applied on the GPU.

  RegularizationType (validate, l1/l2 components)  crates/tenrso-decomp/src/cp/types.rs:65-192
  CpConstraints (+ constructors, effective_l1/l2)   crates/tenrso-decomp/src/cp/types.rs:199-309
  cp_als_constrained                                crates/tenrso-decomp/src/cp/core.rs:225-400

The checks run in tenrso's order and raise its messages (as `TenrsoError`
with the C status of the matching `CpError`) before anything reaches the GPU.
Orthogonality (a QR after every update, taken with a positive diagonal in R)
and Tikhonov regularization of any order run inside the GPU sweep.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from ._lib import CpConstraintsC, CpInfo, TenrsoError, check
from .dense import CpDecomp, _ctx_handle, _f32, _i64, _info_to, _init_ptr, _prec, _ptr

E_INVALID_RANK = 5
E_INVALID_TOL = 6
E_INVALID_REGULARIZATION = 19


def _invalid_reg(msg: str) -> TenrsoError:
    return TenrsoError(E_INVALID_REGULARIZATION, f"Invalid regularization parameter: {msg}")


@dataclass(frozen=True)
class RegularizationType:
    """None / L2{lambda} / L1{lambda} / ElasticNet{lambda, alpha} / Tikhonov{lambda, order}."""
    kind: str = "none"
    lam: float = 0.0
    alpha: float = 0.0
    order: int = 0

    @classmethod
    def none(cls):
        return cls("none")

    @classmethod
    def l2(cls, lam: float):
        return cls("l2", float(lam))

    @classmethod
    def l1(cls, lam: float):
        return cls("l1", float(lam))

    @classmethod
    def elastic_net(cls, lam: float, alpha: float):
        return cls("elastic_net", float(lam), float(alpha))

    @classmethod
    def tikhonov(cls, lam: float, order: int):
        return cls("tikhonov", float(lam), 0.0, int(order))

    def validate(self) -> None:
        """types.rs:105-165, same messages."""
        if self.kind == "none":
            return
        name = {"l2": "L2", "l1": "L1", "elastic_net": "ElasticNet", "tikhonov": "Tikhonov"}
        if self.kind not in name:
            raise ValueError(f"unknown regularization {self.kind!r}")
        if self.lam < 0.0:
            raise _invalid_reg(f"{name[self.kind]} lambda must be >= 0, got {_disp(self.lam)}")
        if self.kind == "elastic_net" and not 0.0 <= self.alpha <= 1.0:
            raise _invalid_reg(f"ElasticNet alpha must be in [0, 1], got {_disp(self.alpha)}")

    def l2_component(self) -> float:
        """types.rs:167-182."""
        if self.kind == "l2":
            return self.lam
        if self.kind == "elastic_net":
            return (1.0 - self.alpha) * self.lam
        if self.kind == "tikhonov" and self.order == 0:
            return self.lam
        return 0.0

    def l1_component(self) -> float:
        """types.rs:184-192."""
        if self.kind == "l1":
            return self.lam
        if self.kind == "elastic_net":
            return self.alpha * self.lam
        return 0.0


def _disp(x: float) -> str:
    # Rust's Display for f64: integral values print without a fraction
    return str(int(x)) if float(x).is_integer() else repr(float(x))


@dataclass
class CpConstraints:
    """types.rs:199-225 with its defaults."""
    nonnegative: bool = False
    l2_reg: float = 0.0
    orthogonal: bool = False
    regularization: RegularizationType = field(default_factory=RegularizationType.none)
    validate_nonneg_input: bool = True

    @classmethod
    def nonnegative_only(cls):
        """CpConstraints::nonnegative() (types.rs:241-246)."""
        return cls(nonnegative=True)

    @classmethod
    def l2_regularized(cls, lam: float):
        return cls(l2_reg=float(lam), regularization=RegularizationType.l2(lam))

    @classmethod
    def l1_regularized(cls, lam: float):
        return cls(regularization=RegularizationType.l1(lam))

    @classmethod
    def elastic_net(cls, lam: float, alpha: float):
        return cls(regularization=RegularizationType.elastic_net(lam, alpha))

    @classmethod
    def tikhonov(cls, lam: float, order: int):
        return cls(regularization=RegularizationType.tikhonov(lam, order))

    @classmethod
    def orthogonal_only(cls):
        """CpConstraints::orthogonal() (types.rs:287-292)."""
        return cls(orthogonal=True)

    def effective_l2(self) -> float:
        """types.rs:298-303: regularization, when set, overrides l2_reg."""
        if self.regularization.kind == "none":
            return self.l2_reg
        return self.regularization.l2_component()

    def effective_l1(self) -> float:
        return self.regularization.l1_component()


def _validate(shape, rank: int, tol: float, c: CpConstraints) -> CpConstraintsC:
    """core.rs:248-267 in order; the tensor's sign check runs on the GPU."""
    if rank == 0 or any(rank > n for n in shape):
        raise TenrsoError(E_INVALID_RANK, f"Invalid rank: {rank}")
    if not 0.0 <= tol < 1.0:
        raise TenrsoError(E_INVALID_TOL, f"Invalid tolerance: {_disp(tol)}")
    c.regularization.validate()
    if c.regularization.kind == "none" and c.l2_reg < 0.0:
        raise TenrsoError(E_INVALID_TOL, f"Invalid tolerance: {_disp(c.l2_reg)}")
    reg = c.regularization
    tik = reg.kind == "tikhonov" and reg.order > 0
    return CpConstraintsC(float(c.effective_l2()), float(c.effective_l1()),
                          1 if c.nonnegative else 0, 1 if c.validate_nonneg_input else 0,
                          1 if c.orthogonal else 0, int(reg.order) if tik else 0,
                          float(reg.lam) if tik else 0.0)


def cp_als_constrained(tensor, rank: int, max_iters: int, tol: float, init="random",
                       constraints: Optional[CpConstraints] = None,
                       time_limit: Optional[float] = None, precision="fp32", seed: int = 0,
                       ctx=None) -> CpDecomp:
    """core.rs:225-400. init: "random" (U(0,1) from the seeded stream `seed`)
    or a list of initial factor matrices."""
    c = constraints if constraints is not None else CpConstraints()
    t = _f32(tensor)
    cc = _validate(t.shape, rank, tol, c)
    shape = _i64(t.shape)
    total = int(sum(n * rank for n in t.shape))
    out = np.zeros(max(total, 1), dtype=np.float32)
    init_ptr, _keep = _init_ptr(t, rank, init, seed, ctx)
    hist = np.zeros(max(max_iters, 1), dtype=np.float64)
    info = CpInfo()
    info.fit_history = hist.ctypes.data_as(C.POINTER(C.c_double))
    check(_lib.load().tsr_cp_als_constrained_f32(
        _ctx_handle(ctx), _ptr(t), t.ndim, _ptr(shape), rank, max_iters, float(tol), init_ptr,
        seed, C.byref(cc), _prec(precision), -1.0 if time_limit is None else float(time_limit),
        _ptr(out), C.byref(info)))
    factors, off = [], 0
    for n in t.shape:
        factors.append(out[off:off + n * rank].reshape(n, rank).copy())
        off += n * rank
    return CpDecomp(factors=factors, weights=None, fit=float(info.fit), iters=int(info.iters),
                    convergence=_info_to(info, hist), ridge_used=bool(info.ridge_used))


def cp_als_constrained_dev(d_tensor: int, shape, rank: int, max_iters: int, tol: float,
                           d_init: int, d_out: int, constraints: Optional[CpConstraints] = None,
                           precision="fp32", time_limit: Optional[float] = None, ctx=None):
    """Device-resident form on raw device pointers; returns (fit, iters, info)."""
    c = constraints if constraints is not None else CpConstraints()
    cc = _validate(list(shape), rank, tol, c)
    sh = _i64(shape)
    hist = np.zeros(max(max_iters, 1), dtype=np.float64)
    info = CpInfo()
    info.fit_history = hist.ctypes.data_as(C.POINTER(C.c_double))
    check(_lib.load().tsr_cp_als_constrained_dev_f32(
        _ctx_handle(ctx), C.c_void_p(d_tensor), len(shape), _ptr(sh), rank, max_iters,
        float(tol), C.c_void_p(d_init), C.byref(cc), _prec(precision),
        -1.0 if time_limit is None else float(time_limit), C.c_void_p(d_out), C.byref(info)))
    return float(info.fit), int(info.iters), _info_to(info, hist)

"""Python mirror of tenrso's dense CP-ALS API over the C ABI.

Names, argument meaning and error behaviour follow the Rust functions:
  khatri_rao                  crates/tenrso-kernels/src/khatri_rao.rs:56-89 (panics -> raises)
  mttkrp / mttkrp_blocked ... crates/tenrso-kernels/src/mttkrp.rs:74-146, 395-992
  mttkrp_all_modes            crates/tenrso-kernels/src/utils.rs:282-307
  cp_als / CpDecomp / ConvergenceInfo  crates/tenrso-decomp/src/cp/core.rs:59-182, types.rs:311-368
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import CpInfo, TenrsoError, check

PRECISIONS = {"fp32": 0, "bf16x3": 1}
REASONS = ("MaxIterations", "FitTolerance", "Oscillation", "TimeLimit")


class Context:
    """One tsr_ctx: a device, a stream and the device workspace."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        self._lib = _lib.load()
        h = C.c_void_p()
        check(self._lib.tsr_ctx_create(device, C.c_void_p(stream) if stream else None,
                                       C.byref(h)))
        self.handle = h
        self.device = device

    def synchronize(self):
        check(self._lib.tsr_ctx_synchronize(self.handle))

    @property
    def launches(self) -> int:
        return int(self._lib.tsr_ctx_launch_count(self.handle))

    def set_trace(self, capacity: int = 4096):
        """Turn kernel timeline tracing of dense cp_als calls on (capacity
        slots) or off (0)."""
        check(self._lib.tsr_ctx_set_trace(self.handle, int(capacity)))
        self._trace_cap = int(capacity)

    def read_trace(self):
        """Records of the last traced cp_als call: a list of
        (kind, mode, start_ns, end_ns), kind one of "mttkrp", "inverse",
        "solve", in launch order."""
        cap = getattr(self, "_trace_cap", 0)
        if cap <= 0:
            return []
        st = np.zeros(cap, np.int64)
        en = np.zeros(cap, np.int64)
        kd = np.zeros(cap, np.int32)
        md = np.zeros(cap, np.int32)
        n = C.c_int(0)
        check(self._lib.tsr_ctx_read_trace(self.handle, cap, _ptr(st), _ptr(en), _ptr(kd),
                                           _ptr(md), C.byref(n)))
        names = ("mttkrp", "inverse", "solve")
        return [(names[kd[i]], int(md[i]), int(st[i]), int(en[i])) for i in range(n.value)]

    def set_wait_budget(self, cycles: int = 0):
        """Budget (clock cycles) of each bounded wait in the tensor-core MTTKRP;
        0 restores the default (about one second)."""
        check(self._lib.tsr_ctx_set_wait_budget(self.handle, int(cycles)))

    def close(self):
        if self.handle:
            self._lib.tsr_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = {}


def default_context(device: int = 0) -> Context:
    if device not in _default:
        _default[device] = Context(device)
    return _default[device]


def _prec(p) -> int:
    if isinstance(p, int):
        return p
    try:
        return PRECISIONS[p]
    except KeyError:
        raise ValueError(f"unknown precision {p!r}; use 'fp32' or 'bf16x3'") from None


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _i64(seq) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(seq, dtype=np.int64))


def _ctx_handle(ctx):
    """The context's handle; NULL when no device context can be created, so
    that the C ABI still reports argument errors first and then fails loudly
    ("null context") for valid arguments."""
    if ctx is not None:
        return ctx.handle
    try:
        return default_context().handle
    except TenrsoError:
        return None


# ---------------------------------------------------------------------------
def khatri_rao(a, b, ctx: Optional[Context] = None) -> np.ndarray:
    """(I*J x K) with row a*J + b = A[a] * B[b]. Raises TenrsoError
    ("Number of columns must match ...") where tenrso panics."""
    a = _f32(a)
    b = _f32(b)
    if a.ndim != 2 or b.ndim != 2:
        raise ValueError("khatri_rao takes two matrices")
    out = np.empty((a.shape[0] * b.shape[0], a.shape[1]), dtype=np.float32)
    h = ctx.handle if ctx else (None if a.shape[1] != b.shape[1] else default_context().handle)
    check(_lib.load().tsr_khatri_rao_f32(h, _ptr(a), a.shape[0], a.shape[1], _ptr(b),
                                         b.shape[0], b.shape[1], _ptr(out)))
    return out


def _mttkrp_args(tensor, factors):
    t = np.asarray(tensor, dtype=np.float32)
    shape = _i64(t.shape)
    strides = _i64([s // 4 for s in t.strides])  # element strides of the view
    fs = [_f32(f) for f in factors]
    for f in fs:
        if f.ndim != 2:
            raise ValueError("factor matrices must be 2-D")
    rows = _i64([f.shape[0] for f in fs]) if fs else _i64([0])
    cols = _i64([f.shape[1] for f in fs]) if fs else _i64([0])
    ptrs = (C.c_void_p * max(len(fs), 1))(*[f.ctypes.data for f in fs])
    return t, shape, strides, fs, rows, cols, ptrs


def _needs_ctx(t, fs, mode):
    # validation happens before any device work; a context is only needed
    # when the arguments are valid
    return not (mode < 0 or mode >= t.ndim or len(fs) != t.ndim or t.ndim < 2 or
                any(f.shape[1] != fs[0].shape[1] for f in fs) or
                any(f.shape[0] != t.shape[i] for i, f in enumerate(fs)))


def mttkrp(tensor, factors: Sequence, mode: int, precision="fp32",
           ctx: Optional[Context] = None) -> np.ndarray:
    """V = X_(mode) . KR(all factors except mode), shape (I_mode, R).
    Accepts any-strided float32 views (packed like as_standard_layout)."""
    t, shape, strides, fs, rows, cols, ptrs = _mttkrp_args(tensor, factors)
    R = fs[0].shape[1] if fs else 0
    out = np.zeros((t.shape[mode] if 0 <= mode < t.ndim else 0, R), dtype=np.float32)
    h = _ctx_handle(ctx) if _needs_ctx(t, fs, mode) else None
    base = t.__array_interface__["data"][0]
    check(_lib.load().tsr_mttkrp_f32(h, C.c_void_p(base), t.ndim, _ptr(shape), _ptr(strides),
                                     ptrs, len(fs), _ptr(rows), _ptr(cols), mode,
                                     _prec(precision), _ptr(out)))
    return out


def mttkrp_blocked(tensor, factors, mode: int, tile_size: int, precision="fp32",
                   ctx: Optional[Context] = None) -> np.ndarray:
    """mttkrp_blocked / mttkrp_blocked_parallel: tile_size must be > 0
    ("Tile size must be greater than 0"); the result is the same MTTKRP."""
    t, shape, strides, fs, rows, cols, ptrs = _mttkrp_args(tensor, factors)
    R = fs[0].shape[1] if fs else 0
    out = np.zeros((t.shape[mode] if 0 <= mode < t.ndim else 0, R), dtype=np.float32)
    h = _ctx_handle(ctx) if (tile_size > 0 and _needs_ctx(t, fs, mode)) else None
    base = t.__array_interface__["data"][0]
    check(_lib.load().tsr_mttkrp_blocked_f32(h, C.c_void_p(base), t.ndim, _ptr(shape),
                                             _ptr(strides), ptrs, len(fs), _ptr(rows),
                                             _ptr(cols), mode, int(tile_size), _prec(precision),
                                             _ptr(out)))
    return out


mttkrp_blocked_parallel = mttkrp_blocked


def mttkrp_fused(tensor, factors, mode: int, precision="fp32", ctx=None) -> np.ndarray:
    """mttkrp_fused / mttkrp_fused_parallel (KR rows on the fly): same kernel."""
    return mttkrp(tensor, factors, mode, precision, ctx)


mttkrp_fused_parallel = mttkrp_fused


def mttkrp_all_modes(tensor, factors, precision="fp32", ctx=None) -> List[np.ndarray]:
    t = _f32(tensor)
    fs = [_f32(f) for f in factors]
    R = fs[0].shape[1]
    outs = [np.zeros((n, R), dtype=np.float32) for n in t.shape]
    ptrs = (C.c_void_p * len(fs))(*[f.ctypes.data for f in fs])
    optrs = (C.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
    check(_lib.load().tsr_mttkrp_all_modes_f32(_ctx_handle(ctx), _ptr(t), t.ndim,
                                               _ptr(_i64(t.shape)), ptrs, R, _prec(precision),
                                               optrs))
    return outs


def mttkrp_dev(d_tensor: int, shape, d_factors: Sequence[int], rank: int, mode: int,
               d_out: int, precision="fp32", ctx: Optional[Context] = None):
    """Device-resident MTTKRP on raw device pointers (stream-ordered)."""
    shp = _i64(shape)
    ptrs = (C.c_void_p * len(d_factors))(*d_factors)
    check(_lib.load().tsr_mttkrp_dev_f32(_ctx_handle(ctx), C.c_void_p(d_tensor), len(shape),
                                         _ptr(shp), ptrs, rank, mode, _prec(precision),
                                         C.c_void_p(d_out)))


# ---------------------------------------------------------------------------
@dataclass
class ConvergenceInfo:
    fit_history: np.ndarray
    reason: str
    oscillated: bool
    oscillation_count: int
    final_fit_change: float


@dataclass
class CpDecomp:
    factors: List[np.ndarray]
    weights: Optional[np.ndarray]
    fit: float
    iters: int
    convergence: Optional[ConvergenceInfo] = None
    ridge_used: bool = False


def _info_to(info: CpInfo, hist: np.ndarray):
    return ConvergenceInfo(fit_history=hist[:info.iters].copy(), reason=REASONS[info.reason],
                           oscillated=bool(info.oscillated),
                           oscillation_count=int(info.oscillation_count),
                           final_fit_change=float(info.final_fit_change))


INIT_STRATEGIES = {"random": 0, "random_normal": 1, "randomnormal": 1, "svd": 2, "nnsvd": 3,
                   "leverage_score": 4, "leveragescore": 4}


def initialize_factors(tensor, rank: int, init="random", seed: int = 0,
                       ctx: Optional[Context] = None) -> List[np.ndarray]:
    """initialize_factors (cp/helpers.rs:192-377) on the device for an
    InitStrategy name: random, random_normal, svd, nnsvd, leverage_score."""
    key = str(init).lower()
    if key not in INIT_STRATEGIES:
        raise ValueError(f"unknown InitStrategy {init!r}")
    t = _f32(tensor)
    total = int(sum(n * rank for n in t.shape))
    out = np.zeros(max(total, 1), dtype=np.float32)
    check(_lib.load().tsr_cp_init_f32(_ctx_handle(ctx), _ptr(t), t.ndim, _ptr(_i64(t.shape)),
                                      rank, INIT_STRATEGIES[key], seed, _ptr(out)))
    factors, off = [], 0
    for n in t.shape:
        factors.append(out[off:off + n * rank].reshape(n, rank).copy())
        off += n * rank
    return factors


def _init_ptr(t: np.ndarray, rank: int, init, seed: int, ctx):
    """(pointer, keep-alive array) of the initial factors: None for Random
    (drawn inside the C call), else the injected or device-initialised ones."""
    if isinstance(init, str):
        if init.lower() == "random":
            return None, None
        init = initialize_factors(t, rank, init, seed, ctx)
    total = int(sum(n * rank for n in t.shape))
    flat = np.concatenate([_f32(f).ravel() for f in init])
    if flat.size != total:
        raise ValueError("initial factors do not match shape x rank")
    return _ptr(flat), flat


def cp_als(tensor, rank: int, max_iters: int, tol: float, init="random",
           time_limit: Optional[float] = None, precision="fp32", seed: int = 0,
           ctx: Optional[Context] = None) -> CpDecomp:
    """CP-ALS with tenrso's loop, validation and convergence rules.
    init: an InitStrategy name ("random": U(0,1) from the seeded SplitMix64
    stream `seed`; "random_normal", "svd", "nnsvd", "leverage_score") or a
    list of initial factor matrices (the injected initialisation)."""
    t = _f32(tensor)
    shape = _i64(t.shape)
    total = int(sum(n * rank for n in t.shape))
    out = np.zeros(max(total, 1), dtype=np.float32)
    init_ptr, _keep = _init_ptr(t, rank, init, seed, ctx)
    hist = np.zeros(max(max_iters, 1), dtype=np.float64)
    info = CpInfo()
    info.fit_history = hist.ctypes.data_as(C.POINTER(C.c_double))
    check(_lib.load().tsr_cp_als_f32(_ctx_handle(ctx), _ptr(t), t.ndim, _ptr(shape), rank,
                                     max_iters, float(tol), init_ptr, seed, _prec(precision),
                                     -1.0 if time_limit is None else float(time_limit),
                                     _ptr(out), C.byref(info)))
    factors, off = [], 0
    for n in t.shape:
        factors.append(out[off:off + n * rank].reshape(n, rank).copy())
        off += n * rank
    return CpDecomp(factors=factors, weights=None, fit=float(info.fit), iters=int(info.iters),
                    convergence=_info_to(info, hist), ridge_used=bool(info.ridge_used))


def cp_als_dev(d_tensor: int, shape, rank: int, max_iters: int, tol: float, d_init: int,
               d_out: int, precision="fp32", time_limit: Optional[float] = None,
               ctx: Optional[Context] = None):
    """Device-resident CP-ALS on raw device pointers; returns (fit, iters,
    ConvergenceInfo). Factors are written to d_out (concatenated)."""
    shp = _i64(shape)
    hist = np.zeros(max(max_iters, 1), dtype=np.float64)
    info = CpInfo()
    info.fit_history = hist.ctypes.data_as(C.POINTER(C.c_double))
    check(_lib.load().tsr_cp_als_dev_f32(_ctx_handle(ctx), C.c_void_p(d_tensor), len(shape),
                                         _ptr(shp), rank, max_iters, float(tol),
                                         C.c_void_p(d_init), _prec(precision),
                                         -1.0 if time_limit is None else float(time_limit),
                                         C.c_void_p(d_out), C.byref(info)))
    return float(info.fit), int(info.iters), _info_to(info, hist)


def cp_als_accelerated(tensor, rank: int, max_iters: int, tol: float, init="random",
                       time_limit: Optional[float] = None, precision="fp32", seed: int = 0,
                       ctx: Optional[Context] = None) -> CpDecomp:
    """cp_als_accelerated (cp/advanced.rs:51-213): the CP-ALS sweep with the
    five-step line search of line_search_cp (cp/helpers.rs:130-189) and the
    adaptive extrapolation U_n = U_new + a_ls * alpha * (U_new - U_prev) from
    the second iteration on. tol must lie in (0, 1). init as in cp_als."""
    if rank == 0:
        raise TenrsoError(5, f"Invalid rank: {rank}")
    if not 0.0 < tol < 1.0:
        raise TenrsoError(6, f"Invalid tolerance: {tol}")
    t = _f32(tensor)
    shape = _i64(t.shape)
    total = int(sum(n * rank for n in t.shape))
    out = np.zeros(max(total, 1), dtype=np.float32)
    init_ptr, _keep = _init_ptr(t, rank, init, seed, ctx)
    hist = np.zeros(max(max_iters, 1), dtype=np.float64)
    info = CpInfo()
    info.fit_history = hist.ctypes.data_as(C.POINTER(C.c_double))
    check(_lib.load().tsr_cp_als_accelerated_f32(
        _ctx_handle(ctx), _ptr(t), t.ndim, _ptr(shape), rank, max_iters, float(tol), init_ptr,
        seed, _prec(precision), -1.0 if time_limit is None else float(time_limit), _ptr(out),
        C.byref(info)))
    factors, off = [], 0
    for n in t.shape:
        factors.append(out[off:off + n * rank].reshape(n, rank).copy())
        off += n * rank
    return CpDecomp(factors=factors, weights=None, fit=float(info.fit), iters=int(info.iters),
                    convergence=_info_to(info, hist), ridge_used=bool(info.ridge_used))


def cp_als_accelerated_dev(d_tensor: int, shape, rank: int, max_iters: int, tol: float,
                           d_init: int, d_out: int, precision="fp32",
                           time_limit: Optional[float] = None, ctx: Optional[Context] = None):
    """Device-resident cp_als_accelerated on raw device pointers; returns
    (fit, iters, ConvergenceInfo). Factors are written to d_out (concatenated)."""
    shp = _i64(shape)
    hist = np.zeros(max(max_iters, 1), dtype=np.float64)
    info = CpInfo()
    info.fit_history = hist.ctypes.data_as(C.POINTER(C.c_double))
    check(_lib.load().tsr_cp_als_accelerated_dev_f32(
        _ctx_handle(ctx), C.c_void_p(d_tensor), len(shape), _ptr(shp), rank, max_iters,
        float(tol), C.c_void_p(d_init), _prec(precision),
        -1.0 if time_limit is None else float(time_limit), C.c_void_p(d_out), C.byref(info)))
    return float(info.fit), int(info.iters), _info_to(info, hist)


def mttkrp_f64(tensor, factors: Sequence[np.ndarray], mode: int,
               ctx: Optional[Context] = None) -> np.ndarray:
    """mttkrp<f64> (mttkrp.rs:74-146): FP64 tensor, factors and result."""
    t = np.ascontiguousarray(np.asarray(tensor, dtype=np.float64))
    fs = [np.ascontiguousarray(np.asarray(f, dtype=np.float64)) for f in factors]
    rows = _i64([f.shape[0] for f in fs] or [0])
    cols = _i64([f.shape[1] if f.ndim == 2 else 0 for f in fs] or [0])
    ptrs = (C.c_void_p * max(len(fs), 1))(*[f.ctypes.data for f in fs])
    R = int(cols[0]) if len(fs) else 0
    n_out = t.shape[mode] if 0 <= mode < t.ndim else 0
    out = np.zeros((max(n_out, 1), max(R, 1)), np.float64)
    check(_lib.load().tsr_mttkrp_f64(_ctx_handle(ctx), _ptr(t), t.ndim, _ptr(_i64(t.shape)), ptrs,
                                     len(fs), _ptr(rows), _ptr(cols), mode, _ptr(out)))
    return out[:n_out, :R]


def cp_als_f64(tensor, rank: int, max_iters: int, tol: float, init="random",
               time_limit: Optional[float] = None, seed: int = 0,
               ctx: Optional[Context] = None) -> CpDecomp:
    """cp_als<f64> (cp/core.rs:59-182): every value in FP64. init: "random"
    (U(0,1) doubles from the seeded stream `seed`) or the initial factors."""
    t = np.ascontiguousarray(np.asarray(tensor, dtype=np.float64))
    total = int(sum(n * rank for n in t.shape))
    out = np.zeros(max(total, 1), dtype=np.float64)
    keep = None
    if isinstance(init, str):
        if init.lower() != "random":
            keep = np.concatenate([np.asarray(f, np.float64).ravel() for f in
                                   initialize_factors(t, rank, init, seed, ctx)])
    else:
        keep = np.concatenate([np.asarray(f, np.float64).ravel() for f in init])
        if keep.size != total:
            raise ValueError("initial factors do not match shape x rank")
    hist = np.zeros(max(max_iters, 1), dtype=np.float64)
    info = CpInfo()
    info.fit_history = hist.ctypes.data_as(C.POINTER(C.c_double))
    check(_lib.load().tsr_cp_als_f64(_ctx_handle(ctx), _ptr(t), t.ndim, _ptr(_i64(t.shape)), rank,
                                     max_iters, float(tol),
                                     _ptr(keep) if keep is not None else None, seed,
                                     -1.0 if time_limit is None else float(time_limit),
                                     _ptr(out), C.byref(info)))
    factors, off = [], 0
    for n in t.shape:
        factors.append(out[off:off + n * rank].reshape(n, rank).copy())
        off += n * rank
    return CpDecomp(factors=factors, weights=None, fit=float(info.fit), iters=int(info.iters),
                    convergence=_info_to(info, hist), ridge_used=bool(info.ridge_used))


def profile_mttkrp_dev(d_tensor: int, shape, d_factors: Sequence[int], rank: int, mode: int,
                       precision="bf16x3", iters: int = 10, flush_l2: bool = True,
                       ctx: Optional[Context] = None):
    """Mean milliseconds of one MTTKRP kernel launch (operands prepared once),
    and the split-K count used. Measurement aid for the roofline figure."""
    shp = _i64(shape)
    ptrs = (C.c_void_p * len(d_factors))(*d_factors)
    ms = C.c_double(0)
    splits = C.c_int64(0)
    check(_lib.load().tsr_profile_mttkrp_dev_f32(_ctx_handle(ctx), C.c_void_p(d_tensor),
                                                 len(shape), _ptr(shp), ptrs, rank, mode,
                                                 _prec(precision), iters, int(flush_l2),
                                                 C.byref(ms), C.byref(splits)))
    return ms.value, splits.value


def gram_inverse(G: np.ndarray, iters: int = 1, ctx: Optional[Context] = None):
    """The CP-ALS solve's FP64 inverse of a symmetric positive definite R x R
    matrix (the stand-in for solve_least_squares' lstsq, cp/helpers.rs:455-495,
    ridge retry included), run `iters` times on the device. Returns
    (G^-1, ridge_used, mean ms per launch)."""
    G = np.ascontiguousarray(G, dtype=np.float64)
    R = G.shape[0]
    if G.shape != (R, R):
        raise ValueError("gram_inverse needs a square matrix")
    out = np.zeros_like(G)
    ridge = C.c_int(0)
    ms = C.c_double(0)
    check(_lib.load().tsr_gram_inverse_f64(_ctx_handle(ctx), _ptr(G), R, int(iters), _ptr(out),
                                           C.byref(ridge), C.byref(ms)))
    return out, int(ridge.value), ms.value

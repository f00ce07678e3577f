"""ctypes binding of libtenrso_b200.so (the C ABI in include/tenrso_b200.h).

The library is the product: there is no CPU fallback. Loading fails loudly
when the shared object is missing, and every call that reaches a kernel needs
a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtenrso_b200.so")

P = C.c_void_p
I64 = C.c_int64
PI64 = C.POINTER(C.c_int64)


class CpConstraintsC(C.Structure):
    """tsr_cp_constraints: the reduced form of CpConstraints the sweep applies."""
    _fields_ = [
        ("l2", C.c_double),
        ("l1", C.c_double),
        ("nonnegative", C.c_int),
        ("validate_nonneg_input", C.c_int),
        ("orthogonal", C.c_int),
        ("tikhonov_order", C.c_int),
        ("tikhonov_lambda", C.c_double),
    ]


class CpInfo(C.Structure):
    _fields_ = [
        ("fit", C.c_double),
        ("iters", C.c_int32),
        ("reason", C.c_int32),
        ("oscillated", C.c_int32),
        ("oscillation_count", C.c_int32),
        ("final_fit_change", C.c_double),
        ("fit_history", C.POINTER(C.c_double)),
        ("ridge_used", C.c_int32),
        ("reserved", C.c_int32),
    ]


# name -> (restype, argtypes)
SIGNATURES = {
    "tsr_last_error": (C.c_char_p, []),
    "tsr_status_string": (C.c_char_p, [C.c_int]),
    "tsr_version": (C.c_char_p, []),
    "tsr_ctx_create": (C.c_int, [C.c_int, P, C.POINTER(P)]),
    "tsr_ctx_destroy": (C.c_int, [P]),
    "tsr_ctx_synchronize": (C.c_int, [P]),
    "tsr_ctx_launch_count": (I64, [P]),
    "tsr_ctx_set_wait_budget": (C.c_int, [P, I64]),
    "tsr_ctx_set_trace": (C.c_int, [P, C.c_int]),
    "tsr_ctx_read_trace": (C.c_int, [P, C.c_int, P, P, P, P, C.POINTER(C.c_int)]),
    "tsr_khatri_rao_f32": (C.c_int, [P, P, I64, I64, P, I64, I64, P]),
    "tsr_mttkrp_f32": (C.c_int, [P, P, C.c_int, P, P, P, C.c_int, P, P, C.c_int, C.c_int, P]),
    "tsr_mttkrp_blocked_f32": (C.c_int, [P, P, C.c_int, P, P, P, C.c_int, P, P, C.c_int, I64,
                                         C.c_int, P]),
    "tsr_mttkrp_all_modes_f32": (C.c_int, [P, P, C.c_int, P, P, I64, C.c_int, P]),
    "tsr_mttkrp_dev_f32": (C.c_int, [P, P, C.c_int, P, P, I64, C.c_int, C.c_int, P]),
    "tsr_gram_inverse_f64": (C.c_int, [P, P, I64, C.c_int, P, C.POINTER(C.c_int),
                                       C.POINTER(C.c_double)]),
    "tsr_profile_mttkrp_dev_f32": (C.c_int, [P, P, C.c_int, P, P, I64, C.c_int, C.c_int, C.c_int,
                                             C.c_int, C.POINTER(C.c_double), PI64]),
    "tsr_mttkrp_mode0_noalloc_f32": (C.c_int, [P, P, C.c_int, P, P, I64, P]),
    "tsr_cp_als_f32": (C.c_int, [P, P, C.c_int, P, I64, C.c_int, C.c_double, P, C.c_uint64,
                                 C.c_int, C.c_double, P, C.POINTER(CpInfo)]),
    "tsr_cp_als_dev_f32": (C.c_int, [P, P, C.c_int, P, I64, C.c_int, C.c_double, P, C.c_int,
                                     C.c_double, P, C.POINTER(CpInfo)]),
    "tsr_cp_als_constrained_f32": (C.c_int, [P, P, C.c_int, P, I64, C.c_int, C.c_double, P,
                                             C.c_uint64, C.POINTER(CpConstraintsC), C.c_int,
                                             C.c_double, P, C.POINTER(CpInfo)]),
    "tsr_cp_als_constrained_dev_f32": (C.c_int, [P, P, C.c_int, P, I64, C.c_int, C.c_double, P,
                                                 C.POINTER(CpConstraintsC), C.c_int, C.c_double,
                                                 P, C.POINTER(CpInfo)]),
    "tsr_cp_als_accelerated_f32": (C.c_int, [P, P, C.c_int, P, I64, C.c_int, C.c_double, P,
                                             C.c_uint64, C.c_int, C.c_double, P,
                                             C.POINTER(CpInfo)]),
    "tsr_cp_als_accelerated_dev_f32": (C.c_int, [P, P, C.c_int, P, I64, C.c_int, C.c_double, P,
                                                 C.c_int, C.c_double, P, C.POINTER(CpInfo)]),
    "tsr_hicoo_create_f32": (C.c_int, [P, P, P, I64, C.c_int, P, P, C.c_int, C.POINTER(P)]),
    "tsr_hicoo_destroy": (C.c_int, [P]),
    "tsr_hicoo_info": (C.c_int, [P, PI64, PI64]),
    "tsr_hicoo_export": (C.c_int, [P, P, P, P, P, P]),
    "tsr_mttkrp_hicoo_f32": (C.c_int, [P, P, P, I64, C.c_int, P]),
    "tsr_mttkrp_hicoo_dev_f32": (C.c_int, [P, P, P, I64, C.c_int, P]),
    "tsr_als_solve_dev_f32": (C.c_int, [P, P, I64, I64, P, P, P, C.POINTER(C.c_double),
                                        C.POINTER(C.c_int)]),
    "tsr_nmode_product_f32": (C.c_int, [P, P, C.c_int, P, P, I64, I64, C.c_int, P]),
    "tsr_nmode_product_dev_f32": (C.c_int, [P, P, C.c_int, P, P, I64, I64, C.c_int, P]),
    "tsr_nmode_products_seq_f32": (C.c_int, [P, P, C.c_int, P, C.c_int, P, P, P, P, P, P]),
    "tsr_tucker_operator_f32": (C.c_int, [P, P, C.c_int, P, C.c_int, P, P, P, P, P, P]),
    "tsr_tucker_reconstruct_f32": (C.c_int, [P, P, C.c_int, P, C.c_int, P, P, P, P, P]),
    "tsr_mttkrp_f64": (C.c_int, [P, P, C.c_int, P, P, C.c_int, P, P, C.c_int, P]),
    "tsr_cp_als_f64": (C.c_int, [P, P, C.c_int, P, I64, C.c_int, C.c_double, P, C.c_uint64,
                                 C.c_double, P, C.POINTER(CpInfo)]),
    "tsr_cp_init_f32": (C.c_int, [P, P, C.c_int, P, I64, C.c_int, C.c_uint64, P]),
    "tsr_cp_init_dev_f32": (C.c_int, [P, P, C.c_int, P, I64, C.c_int, C.c_uint64, P]),
    "tsr_coo_sort_f32": (C.c_int, [P, P, P, I64, C.c_int, P]),
    "tsr_coo_deduplicate_f32": (C.c_int, [P, P, P, I64, C.c_int, P, PI64]),
    "tsr_csf_from_coo_f32": (C.c_int, [P, P, P, I64, C.c_int, P, P, C.c_int, P, P, P, P]),
    "tsr_sparse_create_f32": (C.c_int, [P, P, P, I64, C.c_int, P, C.POINTER(P)]),
    "tsr_sparse_destroy": (C.c_int, [P]),
    "tsr_sparse_create_dev_f32": (C.c_int, [P, P, P, I64, C.c_int, P, C.POINTER(P)]),
    "tsr_coo_deduplicate_dev_f32": (C.c_int, [P, P, P, I64, C.c_int, P, PI64]),
    "tsr_synth_zipf_coo_dev": (C.c_int, [P, C.c_int, P, I64, C.c_uint64, C.c_double, I64, P, P,
                                         PI64]),
    "tsr_sparse_info": (C.c_int, [P, C.c_int, PI64, PI64, PI64]),
    "tsr_mttkrp_csf_f32": (C.c_int, [P, P, P, I64, C.c_int, P]),
    "tsr_mttkrp_csf_dev_f32": (C.c_int, [P, P, P, I64, C.c_int, P]),
    "tsr_profile_mttkrp_csf_dev_f32": (C.c_int, [P, P, P, I64, C.c_int, C.c_int, C.c_int,
                                                 C.POINTER(C.c_double)]),
    "tsr_cp_als_sparse_f32": (C.c_int, [P, P, I64, C.c_int, C.c_double, P, C.c_uint64, C.c_double,
                                        P, C.POINTER(CpInfo)]),
    "tsr_cp_als_sparse_dev_f32": (C.c_int, [P, P, I64, C.c_int, C.c_double, P, C.c_double, P,
                                            C.POINTER(CpInfo)]),
    "tsr_cp_reconstruct_f32": (C.c_int, [P, P, C.c_int, P, P, P, I64, P]),
    "tsr_cp_reconstruct_dev_f32": (C.c_int, [P, P, C.c_int, P, I64, P, P]),
    "tsr_cp_residual_dev_f32": (C.c_int, [P, P, C.c_int, P, P, I64, P, C.c_float, P,
                                          C.POINTER(C.c_double)]),
    "tsr_cp_reconstruction_grad_f32": (C.c_int, [P, P, C.c_int, P, P, C.c_int, P, P, P, I64,
                                                 C.c_int, P]),
    "tsr_cp_reconstruction_grad_dev_f32": (C.c_int, [P, P, C.c_int, P, P, I64, P, C.c_int, P]),
    "tsr_dense_create_dev_f32": (C.c_int, [P, P, C.c_int, P, C.c_int, C.POINTER(P)]),
    "tsr_dense_destroy": (C.c_int, [P]),
    "tsr_cp_loss_grad_dev_f32": (C.c_int, [P, P, P, I64, C.c_double, P, C.POINTER(C.c_double)]),
    "tsr_batch_create_f32": (C.c_int, [P, C.c_int, P, P, P, C.POINTER(P)]),
    "tsr_batch_destroy": (C.c_int, [P]),
    "tsr_batch_factor_layout": (C.c_int, [P, PI64, P]),
    "tsr_batch_set_config": (C.c_int, [P, C.c_int, C.c_int, C.c_int]),
    "tsr_batch_get_config": (C.c_int, [P, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                       C.POINTER(C.c_int)]),
    "tsr_batch_autotune": (C.c_int, [P, P, C.c_int, P, C.c_char_p, C.POINTER(C.c_int)]),
    "tsr_cp_als_batched_f32": (C.c_int, [P, P, C.c_int, C.c_double, P, C.c_uint64, P, P]),
    "tsr_cp_als_batched_dev_f32": (C.c_int, [P, P, C.c_int, C.c_double, P, P, P]),
}

_lib = None


def load():
    """Load the in-tree shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m tenrso_b200.build` "
                "(there is no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


STATUS = {
    0: "TSR_OK", 1: "TSR_E_MODE_OOB", 2: "TSR_E_NFACTORS", 3: "TSR_E_RANK_MISMATCH",
    4: "TSR_E_ROWS_MISMATCH", 5: "TSR_E_INVALID_RANK", 6: "TSR_E_INVALID_TOL",
    7: "TSR_E_NOT_SPD", 8: "TSR_E_TIMEOUT", 9: "TSR_E_CUDA", 10: "TSR_E_INVALID_ARG",
    11: "TSR_E_NEED_2_FACTORS", 12: "TSR_E_TILE_SIZE", 13: "TSR_E_MODE_ORDER",
    14: "TSR_E_UNSUPPORTED", 15: "TSR_E_COLS_MISMATCH", 16: "TSR_E_SHAPE",
    17: "TSR_E_INDEX_OOB", 18: "TSR_E_NONNEG_VIOLATION", 19: "TSR_E_INVALID_REGULARIZATION",
    20: "TSR_E_BLOCK_SHAPE",
}


class TenrsoError(RuntimeError):
    """A non-OK tsr_status; .status is the code, str() is tenrso's message."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status
        self.code = STATUS.get(status, str(status))


def check(rc: int):
    if rc != 0:
        msg = load().tsr_last_error().decode()
        raise TenrsoError(rc, msg)

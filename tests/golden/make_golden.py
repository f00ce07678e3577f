"""Writes tests/golden/reference_kats.json: known-answer vectors transcribed
from tenrso's own unit and doc tests (read as text; tenrso is Rust and cannot
be built in this container). Each entry cites the tenrso file:line it comes
from. Where a reference test computes its expectation in-test (the MTTKRP
"manual verification" loop), the expected array is that loop evaluated here
with exact integer-valued float64 arithmetic.

Run: python tests/golden/make_golden.py
"""
import json
import os

import numpy as np


def manual_mttkrp_mode1():
    # crates/tenrso-kernels/src/mttkrp.rs:1000-1043
    X = np.arange(1, 13, dtype=np.float64).reshape(2, 3, 2)
    u1 = np.array([[1.0, 0.0], [2.0, 1.0]])
    u3 = np.array([[1.0, 0.0], [0.0, 1.0]])
    out = np.zeros((3, 2))
    for i1 in range(3):
        for r in range(2):
            s = 0.0
            for i0 in range(2):
                for i2 in range(2):
                    s += X[i0, i1, i2] * u1[i0, r] * u3[i2, r]
            out[i1, r] = s
    return out.tolist()


def cp_grad_definition(factors, shape, weights=None):
    # dL/dU_n[i, r] = w_r * sum over the other indices of G * prod_{m != n} U_m[i_m, r]
    # with G = ones (crates/tenrso-ad/src/grad.rs:81-120 applied to DenseND::ones)
    U = [np.array(f, dtype=np.float64) for f in factors]
    R = U[0].shape[1]
    w = np.ones(R) if weights is None else np.array(weights, dtype=np.float64)
    out = []
    for n in range(len(U)):
        g = np.zeros((shape[n], R))
        for r in range(R):
            p = w[r]
            for m in range(len(U)):
                if m != n:
                    p *= U[m][:, r].sum()
            g[:, r] = p
        out.append(g.tolist())
    return out


def reconstruct_definition(factors, weights=None):
    # crates/tenrso-kernels/src/outer.rs:223-274 for two factors: A diag(w) B^T
    A, B = (np.array(f, dtype=np.float64) for f in factors)
    w = np.ones(A.shape[1]) if weights is None else np.array(weights, dtype=np.float64)
    return ((A * w) @ B.T).tolist()


GRAD_FACTORS_3WAY = [
    np.arange(1, 13, dtype=np.float64).reshape(4, 3).tolist(),
    (np.arange(1, 16, dtype=np.float64) / 10).reshape(5, 3).tolist(),
    [[1, 0, 0], [0, 1, 0], [0, 0, 1], [0.5, 0.5, 0], [0, 0.5, 0.5], [0.5, 0, 0.5]],
]
GRAD_FACTORS_W = [[[1, 2], [3, 4], [5, 6]], [[0.1, 0.2], [0.3, 0.4], [0.5, 0.6], [0.7, 0.8]]]

KATS = {
    "khatri_rao": [
        {"src": "crates/tenrso-kernels/src/khatri_rao.rs:41-55,479-498",
         "a": [[1, 2], [3, 4]], "b": [[5, 6], [7, 8]],
         "c": [[5, 12], [7, 16], [15, 24], [21, 32]]},
        {"src": "crates/tenrso-kernels/src/khatri_rao.rs:501-516",
         "a": [[1, 2], [3, 4], [5, 6]], "b": [[7, 8], [9, 10]],
         "c_col0": [7, 9, 21, 27, 35, 45]},
        {"src": "crates/tenrso-kernels/src/khatri_rao.rs:519-532",
         "a": [[1], [2], [3]], "b": [[4], [5]], "c": [[4], [5], [8], [10], [12], [15]]},
        {"src": "crates/tenrso-kernels/src/khatri_rao.rs:535-554",
         "a": [[1, 0], [0, 1]], "b": [[2, 0], [0, 3]], "c": [[2, 0], [0, 0], [0, 0], [0, 3]]},
    ],
    "khatri_rao_errors": [
        {"src": "crates/tenrso-kernels/src/khatri_rao.rs:575-581",
         "a": [[1, 2, 3]], "b": [[4, 5]], "expect": "Number of columns must match"},
    ],
    "mttkrp": [
        {"src": "crates/tenrso-kernels/src/mttkrp.rs:1000-1043",
         "shape": [2, 3, 2], "tensor": list(range(1, 13)),
         "factors": [[[1, 0], [2, 1]], [[1, 0], [0.5, 1], [0, 1]], [[1, 0], [0, 1]]],
         "mode": 1, "expected": manual_mttkrp_mode1(), "tol": 1e-10},
    ],
    "mttkrp_errors": [
        {"src": "crates/tenrso-kernels/src/mttkrp.rs:311-319", "shape": [2, 3],
         "factors": [[[1], [1]], [[1], [1], [1]]], "mode": 5, "expect": "Mode"},
        {"src": "crates/tenrso-kernels/src/mttkrp.rs:321-330", "shape": [2, 3, 4],
         "factors": [[[1], [1]], [[1], [1], [1]]], "mode": 0,
         "expect": "Number of factor matrices"},
        {"src": "crates/tenrso-kernels/src/mttkrp.rs:332-340", "shape": [2, 3],
         "factors": [[[1, 2], [1, 2]], [[1], [1], [1]]], "mode": 0, "expect": "columns"},
    ],
    "gram": [
        {"src": "crates/tenrso-decomp/src/cp/tests.rs:26-35",
         "factor": [[1, 2], [3, 4], [5, 6]], "diag": [35.0, 56.0]},
    ],
    "coo_dedup": [
        {"src": "crates/tenrso-sparse/src/coo.rs:420-436",
         "indices": [[0, 0], [0, 0], [1, 1], [1, 1], [2, 2]], "values": [1, 2, 3, 4, 5],
         "shape": [3, 3], "nnz": 3, "out_values": [3, 7, 5]},
    ],
    "coo_sort": [
        {"src": "crates/tenrso-sparse/src/coo.rs:439-452",
         "indices": [[2, 0], [0, 1], [1, 0]], "values": [1, 2, 3], "shape": [3, 3],
         "sorted": [[0, 1], [1, 0], [2, 0]]},
    ],
    # csf.rs:137-264 as written: every fptr level holds nnz offsets. The doc
    # comment (csf.rs:18-30) shows fptr[0]=[0,1,2]; the code yields [0,2,3].
    "csf": [
        {"src": "crates/tenrso-sparse/src/csf.rs:18-30 (example), 137-264 (code)",
         "shape": [3, 4, 5], "indices": [[0, 1, 2], [0, 1, 3], [1, 2, 3]],
         "values": [5, 6, 7], "mode_order": [0, 1, 2],
         "fptr": [[0, 2, 3], [0, 2, 3], [0, 2, 3]],
         "fids": [[0, 1], [1, 2], [2, 3, 3]], "vals": [5, 6, 7]},
        {"src": "crates/tenrso-sparse/src/csf.rs:533-540", "shape": [3, 3, 3],
         "indices": [], "values": [], "mode_order": [0, 1, 2],
         "fptr": [[0], [0], [0]], "fids": [[], [], []], "vals": []},
        {"src": "crates/tenrso-sparse/src/csf.rs:542-558", "shape": [2, 3, 4],
         "indices": [[0, 1, 2], [1, 2, 3]], "values": [1, 2], "mode_order": [2, 1, 0],
         "fptr": [[0, 1, 2], [0, 1, 2], [0, 1, 2]],
         "fids": [[2, 3], [1, 2], [0, 1]], "vals": [1, 2]},
        {"src": "crates/tenrso-sparse/src/csf.rs:637-648", "shape": [5, 5, 5],
         "indices": [[2, 3, 4]], "values": [42], "mode_order": [0, 1, 2],
         "fptr": [[0, 1], [0, 1], [0, 1]], "fids": [[2], [3], [4]], "vals": [42]},
    ],
    "cp_reconstruct": [
        {"src": "crates/tenrso-kernels/src/outer.rs:440-455", "factors": [[[2], [3]], [[4], [5], [6]]],
         "weights": None, "shape": [2, 3], "expected": [[8, 10, 12], [12, 15, 18]]},
        {"src": "crates/tenrso-kernels/src/outer.rs:457-470",
         "factors": [[[1, 0], [0, 1]], [[1, 0], [0, 1]]], "weights": None, "shape": [2, 2],
         "expected": [[1, 0], [0, 1]]},
        {"src": "crates/tenrso-kernels/src/outer.rs:473-483 (pins [0,0] = 46; the rest is "
                "the definition)", "factors": [[[1, 2], [3, 4]], [[5, 6], [7, 8]]],
         "weights": [2, 3], "shape": [2, 2],
         "expected": reconstruct_definition([[[1, 2], [3, 4]], [[5, 6], [7, 8]]], [2, 3])},
        {"src": "crates/tenrso-kernels/src/outer.rs:213-222 (doc example, shape only; values "
                "are the definition)",
         "factors": [[[1, 0], [0, 1]], [[1, 0], [0, 1], [1, 1]]], "weights": None,
         "shape": [2, 3],
         "expected": reconstruct_definition([[[1, 0], [0, 1]], [[1, 0], [0, 1], [1, 1]]])},
    ],
    "cp_reconstruct_errors": [
        {"src": "crates/tenrso-kernels/src/outer.rs:512-520",
         "factors": [[[1, 2], [3, 4]], [[5], [6]]], "expect": "columns"},
    ],
    "cp_grad": [
        {"src": "crates/tenrso-ad/tests/integration_tests.rs:56-99 (ones gradient)",
         "factors": GRAD_FACTORS_3WAY, "weights": None, "shape": [4, 5, 6],
         "expected": cp_grad_definition(GRAD_FACTORS_3WAY, [4, 5, 6])},
        {"src": "crates/tenrso-ad/tests/integration_tests.rs:335-367 (weights)",
         "factors": GRAD_FACTORS_W, "weights": [2, 3], "shape": [3, 4],
         "expected": cp_grad_definition(GRAD_FACTORS_W, [3, 4], [2, 3])},
    ],
    "csf_errors": [
        {"src": "crates/tenrso-sparse/src/csf.rs:516-531", "ndim": 3,
         "bad_orders": [[0, 1], [0, 0, 1], [0, 1, 3]]},
    ],
}


if __name__ == "__main__":
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")
    with open(path, "w") as f:
        json.dump(KATS, f, indent=1)
    print("wrote", path)

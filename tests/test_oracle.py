"""Pins the oracle: tenrso's own known-answer vectors (tests/golden), then
cross-checks against independent numpy/scipy formulations. CPU only."""
import numpy as np
import pytest

from tenrso_b200 import synth


def test_khatri_rao_golden(orc, kats):
    for case in kats["khatri_rao"]:
        c = orc.khatri_rao(np.array(case["a"], float), np.array(case["b"], float))
        if "c" in case:
            assert np.array_equal(c, np.array(case["c"], float)), case["src"]
        else:
            assert np.array_equal(c[:, 0], np.array(case["c_col0"], float)), case["src"]


@pytest.mark.parametrize("faithful", [True, False])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_mttkrp_golden(orc, kats, faithful, dtype):
    case = kats["mttkrp"][0]
    X = np.array(case["tensor"], dtype=dtype).reshape(case["shape"])
    fs = [np.array(f, dtype=dtype) for f in case["factors"]]
    out = orc.mttkrp(X, fs, case["mode"], faithful=faithful)
    assert np.abs(out - np.array(case["expected"])).max() < case["tol"]


def test_gram_golden(orc, kats):
    case = kats["gram"][0]
    G = orc.gram(np.array(case["factor"], float))
    assert np.allclose(np.diag(G), case["diag"], atol=1e-10)


def test_coo_golden(orc, kats):
    case = kats["coo_dedup"][0]
    idx, vals = orc.coo_deduplicate(np.array(case["indices"]), np.array(case["values"]))
    assert idx.shape[0] == case["nnz"]
    assert vals.tolist() == case["out_values"]
    case = kats["coo_sort"][0]
    # sort is the first half of deduplicate; distinct indices keep all entries
    idx, _ = orc.coo_deduplicate(np.array(case["indices"]), np.array(case["values"]))
    assert idx.tolist() == case["sorted"]


def test_csf_golden(orc, kats):
    for case in kats["csf"]:
        idx = np.array(case["indices"], dtype=np.int64).reshape(-1, len(case["shape"]))
        fptr, fids, vals = orc.csf_from_coo(idx, np.array(case["values"], np.float32),
                                            case["mode_order"])
        assert [f.tolist() for f in fptr] == case["fptr"], case["src"]
        assert [f.tolist() for f in fids] == case["fids"], case["src"]
        assert vals.tolist() == case["vals"], case["src"]
    for bad in kats["csf_errors"][0]["bad_orders"]:
        with pytest.raises(ValueError):
            orc.csf_from_coo(np.zeros((0, 3), np.int64), np.zeros(0, np.float32), bad)


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_mttkrp_vs_einsum(orc, mode):
    rng = np.random.default_rng(7)
    shape = (5, 7, 3, 4)
    X = rng.standard_normal(shape)
    fs = [rng.standard_normal((n, 3)) for n in shape]
    letters = "abcd"
    spec = ",".join([letters] + [letters[m] + "r" for m in range(4) if m != mode])
    ref = np.einsum(spec + "->" + letters[mode] + "r", X, *[fs[m] for m in range(4) if m != mode])
    for faithful in (True, False):
        out = orc.mttkrp(X, fs, mode, faithful=faithful)
        assert np.allclose(out, ref, rtol=1e-12, atol=1e-12)


def test_solve_vs_scipy(orc):
    import scipy.linalg as sl
    rng = np.random.default_rng(3)
    A = rng.standard_normal((40, 6))
    G = A.T @ A
    M = rng.standard_normal((11, 6))
    x = orc.solve(M, G)
    assert np.allclose(x, sl.solve(G, M.T, assume_a="pos").T, rtol=1e-10, atol=1e-12)


def test_cp_als_oracle_small(orc):
    X, _ = synth.dense_lowrank((12, 10, 8), 3, seed=0xC1, noise=0.01, dtype=np.float64)
    init = synth.init_factors(X.shape, 3, 0xC1, dtype=np.float64)
    fa, ia = orc.cp_als(X, 3, 15, 0.0, init, faithful=True)
    fb, ib = orc.cp_als(X, 3, 15, 0.0, init, faithful=False)
    assert ia["iters"] == 15 and ib["iters"] == 15
    assert abs(ia["fit"] - ib["fit"]) < 1e-10
    assert 0.0 < ia["fit"] <= 1.0
    # fit is consistent with an explicit reconstruction (decomp
    # property_tests.rs:74-104 checks this within 0.05)
    Xh = orc.cp_reconstruct(fa)
    fit_explicit = 1 - np.linalg.norm(X - Xh) / np.linalg.norm(X)
    assert abs(fit_explicit - ia["fit"]) < 1e-8


def test_cp_als_validation(orc):
    X = np.ones((3, 4, 5))
    init = synth.init_factors(X.shape, 2, 1, dtype=np.float64)
    with pytest.raises(ValueError, match="Invalid rank"):
        orc.cp_als(X, 4, 3, 0.0, synth.init_factors(X.shape, 4, 1, np.float64))
    with pytest.raises(ValueError, match="Invalid tolerance"):
        orc.cp_als(X, 2, 3, 1.5, init)


def test_csf_roundtrip_random(orc):
    rng = np.random.default_rng(11)
    shape = (6, 5, 7)
    idx = np.stack([rng.integers(0, n, 300) for n in shape], axis=1)
    vals = rng.random(300).astype(np.float32)
    for mo in ([0, 1, 2], [2, 0, 1], [1, 2, 0]):
        fptr, fids, v = orc.csf_from_coo(idx, vals, mo)
        back, bv = orc.csf_to_coo(fptr, fids, v, mo)
        order = np.lexsort([idx[:, m] for m in reversed(mo)])  # stable, mode_order keys
        assert np.array_equal(back, idx[order])
        assert np.array_equal(bv, vals[order])
        # every level of fptr is an nnz offset array ending at nnz
        for l in range(3):
            assert fptr[l][-1] == len(idx)


def test_coo_dedup_matches_numpy(orc):
    rng = np.random.default_rng(5)
    idx = np.stack([rng.integers(0, 4, 500) for _ in range(3)], axis=1)
    vals = rng.random(500).astype(np.float32)
    oi, ov = orc.coo_deduplicate(idx, vals)
    keys = idx[:, 0] * 16 + idx[:, 1] * 4 + idx[:, 2]
    order = np.argsort(keys, kind="stable")
    uk, start = np.unique(keys[order], return_index=True)
    assert oi.shape[0] == uk.shape[0]
    # sums in insertion order, sequential float32 (coo.rs:330-346)
    exp = []
    for a, b in zip(start, list(start[1:]) + [len(order)]):
        s = np.float32(0)
        for k, p in enumerate(order[a:b]):
            s = vals[p] if k == 0 else np.float32(s + vals[p])
        exp.append(s)
    assert np.array_equal(ov, np.array(exp, np.float32))


def test_coo_mttkrp_matches_dense(orc):
    rng = np.random.default_rng(9)
    shape = (5, 6, 4)
    idx = np.stack([rng.integers(0, n, 60) for n in shape], axis=1)
    idx, vals = orc.coo_deduplicate(idx, rng.random(60).astype(np.float32))
    X = np.zeros(shape)
    X[tuple(idx.T)] = vals
    fs = [rng.standard_normal((n, 3)) for n in shape]
    for mode in range(3):
        assert np.allclose(orc.coo_mttkrp(idx, vals, shape, fs, mode),
                           orc.mttkrp(X, fs, mode), rtol=1e-12, atol=1e-12)


def test_cp_reconstruct_golden(orc, kats):
    for case in kats["cp_reconstruct"]:
        fs = [np.array(f, float) for f in case["factors"]]
        Xh = orc.cp_reconstruct(fs, case["weights"])
        assert list(Xh.shape) == case["shape"], case["src"]
        assert np.array_equal(Xh, np.array(case["expected"], float)), case["src"]


def test_cp_grad_golden(orc, kats):
    for case in kats["cp_grad"]:
        fs = [np.array(f, float) for f in case["factors"]]
        G = np.ones(case["shape"])
        gs = orc.cp_reconstruction_grad(fs, G, case["weights"])
        for g, f, e in zip(gs, fs, case["expected"]):
            assert g.shape == f.shape, case["src"]
            assert np.allclose(g, np.array(e), rtol=1e-12, atol=0), case["src"]
            assert abs(g.sum()) > 1e-6  # the reference's own assertion


@pytest.mark.parametrize("shape,R", [((6, 5, 4, 3), 3), ((7, 4), 2), ((5, 4, 3), 4)])
def test_cp_vjp_vs_central_differences(orc, shape, R):
    """The CPU VJP (restated reconstruction + CpReconstructionGrad on
    G = 2(Xhat - X), plus 2 reg U) equals FP64 central differences (h=1e-6)
    of ||X - [[U]]||^2 + reg sum ||U||^2 in every factor entry."""
    rng = np.random.default_rng(R)
    X = rng.standard_normal(shape)
    fs = [rng.standard_normal((n, R)) for n in shape]
    _, g = orc.cp_loss_grad_vjp(X, fs, 1e-3)
    for m in range(len(shape)):
        ent = [(i, r) for i in range(shape[m]) for r in range(R)]
        fd = orc.fd_grad_entries(X, fs, 1e-3, m, ent)
        an = np.array([g[m][i, r] for i, r in ent])
        assert np.abs(fd - an).max() <= 1e-7 * np.abs(an).max(), m


def test_oracle_reproduces_c2_fit_fixture(orc):
    """tests/golden/c2_fp64_fit.json (the FP64 fit history the GPU tests and
    bench.py compare with) is what the oracle computes on the 256^3 rank-64
    workload. The oracle's fp32 instantiation sits far below it (0.9345 vs
    0.9700): its sequential f32 sum of squares stagnates at this size
    (helpers.rs:498-510), so the fp32 reference's own fit is not a parity
    target there."""
    import json
    import os
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    import make_c2_fit
    with open(os.path.join(here, "golden", "c2_fp64_fit.json")) as f:
        ref = json.load(f)
    got = make_c2_fit.compute()
    assert np.max(np.abs(np.asarray(got["fp64_fit_history"]) -
                         np.asarray(ref["fp64_fit_history"]))) <= 1e-12
    assert abs(got["fp32_fit"] - ref["fp32_fit"]) <= 1e-6


def test_cp_als_coo_matches_dense_oracle(orc):
    """oracle.cp_als_coo (the FP64 checker of the sparse CP-ALS at sizes that
    cannot be densified) reproduces the dense oracle's cp_als on a tensor
    with half its entries structurally zero."""
    from tenrso_b200 import synth
    shape = (30, 20, 10)
    X, _ = synth.dense_lowrank(shape, 4, seed=5, dist="uniform", noise=0.01)
    X[X < np.quantile(X, 0.5)] = 0
    nz = np.argwhere(X != 0)
    init = synth.init_factors(shape, 4, 5)
    _, a = orc.cp_als_coo(nz, X[tuple(nz.T)], shape, 4, 8, 0.0, init)
    _, b = orc.cp_als(X.astype(np.float64), 4, 8, 0.0, [f.astype(np.float64) for f in init])
    assert np.abs(a["fit_history"] - b["fit_history"]).max() <= 1e-12


def test_accelerated_first_sweep_is_cp_als(orc):
    """No extrapolation in the first iteration (advanced.rs:137-147) and the
    line search picks a = 1 (the solve minimises the error along the line), so
    the first fit of cp_als_accelerated is cp_als's."""
    X = synth.uniform(0xC1, 7, (64, 64, 64))
    init = [f.astype(np.float64) for f in synth.init_factors((64, 64, 64), 8, 0xC1)]
    trace = []
    _, acc = orc.cp_als_accelerated(X, 8, 3, 1e-9, init, trace=trace)
    _, std = orc.cp_als(X, 8, 1, 0.0, init)
    assert abs(acc["fit_history"][0] - std["fit_history"][0]) <= 1e-12
    assert all(a == 1.0 for _, _, a, _ in trace)
    with pytest.raises(ValueError):
        orc.cp_als_accelerated(X, 8, 3, 0.0, init)
    with pytest.raises(ValueError):
        orc.cp_als_accelerated(X, 0, 3, 0.5, init)


@pytest.mark.parametrize("shape,R", [((12, 10, 9), 5), ((7, 6, 5, 4), 3)])
def test_line_search_closed_form(orc, shape, R):
    """The device evaluates line_search_cp's trial fits (helpers.rs:130-189)
    from five sums: <M, prev>, <M, d>, <G, prev'prev>, <G, prev'd>, <G, d'd>
    with d = U_new - prev, M the mode's MTTKRP and G the Hadamard of the other
    Grams. They equal compute_fit of the trial factors."""
    rng = np.random.default_rng(3)
    X = rng.random(shape)
    U = [rng.random((n, R)) for n in shape]
    prev = [rng.random((n, R)) for n in shape]
    xn = float(np.sum(X * X))
    for n in range(len(shape)):
        M = orc.mttkrp(X, U, n)
        G = np.ones((R, R))
        for m in range(len(shape)):
            if m != n:
                G *= orc.gram(U[m])
        new = orc.solve(M, G)
        d = new - prev[n]
        s0, s1 = np.sum(M * prev[n]), np.sum(M * d)
        q1 = np.sum(G * (prev[n].T @ prev[n]))
        q2 = np.sum(G * (prev[n].T @ d))
        q3 = np.sum(G * (d.T @ d))
        for a in (0.25, 0.5, 0.75, 1.0, 1.25):
            test = list(U)
            test[n] = prev[n] + a * d
            lit = orc.compute_fit(X, test, xn)
            err = np.sqrt(max(xn + q1 + 2 * a * q2 + a * a * q3 - 2 * (s0 + a * s1), 0.0))
            closed = min(max(1.0 - err / np.sqrt(xn), 0.0), 1.0)
            assert abs(lit - closed) <= 1e-12, (n, a, lit, closed)


def test_oracle_reproduces_c2_accel_fixture(orc):
    """The committed FP64 history of cp_als_accelerated on the 256^3 rank-64
    workload (tests/golden/make_c2_accel.py): the first two sweeps re-derived."""
    import json
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "c2_accel_fp64.json")) as f:
        ref = json.load(f)
    X, _ = synth.dense_lowrank((256, 256, 256), 64, seed=0xC2, dist="uniform", noise=0.005)
    init = [f.astype(np.float64) for f in synth.init_factors((256, 256, 256), 64, 0xC2)]
    _, info = orc.cp_als_accelerated(X.astype(np.float64), 64, 2, 1e-9, init)
    assert np.allclose(info["fit_history"], ref["fp64_fit_history"][:2], rtol=0, atol=1e-12)


@pytest.mark.parametrize("threads", [1, 4])
def test_csf_mttkrp_restatement_matches_coo_definition(orc, threads):
    """The restated CSF MTTKRP (the C3 CPU baseline) against the FP64 COO
    definition on a Zipf tensor, rooted at every mode."""
    shape = (300, 200, 100)
    idx, vals, _ = synth.zipf_coo(shape, 20000, 0xC3)
    idx, vals = orc.coo_deduplicate(idx, vals)
    rng = np.random.default_rng(2)
    fs = [rng.random((n, 16), dtype=np.float32) for n in shape]
    for root in range(3):
        mo = [root] + sorted((m for m in range(3) if m != root), key=lambda m: shape[m])
        fp, fi, v = orc.csf_from_coo(idx, vals, mo)
        got = orc.csf_mttkrp(fp, fi, v, mo, shape, fs, threads)
        ref = orc.coo_mttkrp(idx, vals, shape, fs, root)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-5

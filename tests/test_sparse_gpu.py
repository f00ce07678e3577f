"""Sparse path on the GPU against the oracle: CooTensor sort/deduplicate and
CsfTensor::from_coo bit-exact (every array element equal), CSF MTTKRP within
1e-5 relative Frobenius of the FP64 definition, sparse CP-ALS fit within 1e-4
of the FP64 dense oracle on the densified tensor."""
import numpy as np
import pytest

import tenrso_b200 as tb
from tenrso_b200 import synth

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300)


def random_coo(shape, n, seed, dup_frac=0.3):
    rng = np.random.default_rng(seed)
    idx = np.stack([rng.integers(0, s, n) for s in shape], axis=1)
    nd = int(n * dup_frac)
    if nd:
        idx[-nd:] = idx[rng.integers(0, n - nd, nd)]  # planted duplicates
    vals = rng.random(n).astype(np.float32)
    return idx.astype(np.int64), vals


def test_csf_golden(kats):
    for case in kats["csf"]:
        idx = np.array(case["indices"], dtype=np.int64).reshape(-1, len(case["shape"]))
        coo = tb.CooTensor(idx, np.array(case["values"], np.float32), case["shape"])
        csf = tb.CsfTensor.from_coo(coo, case["mode_order"])
        assert [csf.fptr(l).tolist() for l in range(csf.ndim())] == case["fptr"], case["src"]
        assert [csf.fids(l).tolist() for l in range(csf.ndim())] == case["fids"], case["src"]
        assert csf.vals().tolist() == case["vals"], case["src"]
        assert csf.nnz() == len(case["values"])


def test_coo_golden(kats):
    case = kats["coo_dedup"][0]
    coo = tb.CooTensor(case["indices"], case["values"], case["shape"])
    coo.deduplicate()
    assert coo.nnz() == case["nnz"]
    assert coo.values().tolist() == case["out_values"]
    case = kats["coo_sort"][0]
    coo = tb.CooTensor(case["indices"], case["values"], case["shape"])
    coo.sort()
    assert coo.indices().tolist() == case["sorted"]


@pytest.mark.parametrize("shape,n", [((7, 5, 9), 400), ((30, 20, 10), 5000),
                                     ((4, 5, 6, 7), 800), ((50, 40), 900), ((13,), 50),
                                     ((3, 4, 2, 3, 2), 200)])
def test_csf_bit_exact_random(orc, shape, n):
    idx, vals = random_coo(shape, n, seed=n)
    coo = tb.CooTensor(idx, vals, shape)
    nd = len(shape)
    rng = np.random.default_rng(1)
    for mo in [list(range(nd)), list(reversed(range(nd))), list(rng.permutation(nd))]:
        csf = tb.CsfTensor.from_coo(coo, mo)
        fp, fi, v = orc.csf_from_coo(idx, vals, mo)
        for l in range(nd):
            assert np.array_equal(csf.fptr(l), fp[l]), (mo, l)
            assert np.array_equal(csf.fids(l), fi[l]), (mo, l)
        assert np.array_equal(csf.vals(), v)
        back = csf.to_coo()
        order = np.lexsort([idx[:, m] for m in reversed(mo)])
        if nd > 1:
            assert np.array_equal(back.indices(), idx[order])


@pytest.mark.parametrize("shape,n", [((7, 5, 9), 400), ((30, 20, 10), 20000),
                                     ((4, 5, 6, 7), 800), ((2, 2), 50)])
def test_coo_deduplicate_bit_exact(orc, shape, n):
    idx, vals = random_coo(shape, n, seed=7 + n, dup_frac=0.5)
    coo = tb.CooTensor(idx, vals, shape)
    coo.deduplicate()
    oi, ov = orc.coo_deduplicate(idx, vals)
    assert np.array_equal(coo.indices(), oi)
    assert np.array_equal(coo.values(), ov)  # fp32 sums in insertion order


def test_coo_sort_stable():
    idx, vals = random_coo((6, 6, 6), 500, seed=3, dup_frac=0.5)
    coo = tb.CooTensor(idx, vals, (6, 6, 6))
    coo.sort()
    order = np.lexsort([idx[:, 2], idx[:, 1], idx[:, 0]])  # stable, lexicographic
    assert np.array_equal(coo.indices(), idx[order])
    assert np.array_equal(coo.values(), vals[order])


def test_csf_empty_and_errors():
    coo = tb.CooTensor.zeros([3, 3, 3])
    csf = tb.CsfTensor.from_coo(coo, [0, 1, 2])
    assert csf.nnz() == 0
    assert [csf.fptr(l).tolist() for l in range(3)] == [[0], [0], [0]]
    for bad in ([0, 1], [0, 0, 1], [0, 1, 3]):
        with pytest.raises(tb.CsfError, match="Invalid mode order"):
            tb.CsfTensor.from_coo(coo, bad)


@pytest.mark.parametrize("R", [32, 8, 4, 64, 5, 128, 96])
@pytest.mark.parametrize("shape", [(60, 50, 40), (300, 7, 90)])
def test_csf_mttkrp_parity(orc, shape, R):
    idx, vals = random_coo(shape, 20000, seed=R, dup_frac=0.2)
    coo = tb.CooTensor(idx, vals, shape)
    sp = tb.SparseTensor(coo)
    rng = np.random.default_rng(R)
    fs = [rng.standard_normal((n, R)).astype(np.float32) for n in shape]
    for mode in range(3):
        out = sp.mttkrp(fs, mode)
        ref = orc.coo_mttkrp(idx, vals.astype(np.float64), shape,
                             [f.astype(np.float64) for f in fs], mode)
        assert rel_err(out, ref) <= 1e-5, (shape, R, mode, rel_err(out, ref))
    sp.close()


def test_csf_mttkrp_4way_and_zipf(orc):
    shape = (20, 30, 10, 15)
    idx, vals = random_coo(shape, 5000, seed=11)
    sp = tb.SparseTensor(tb.CooTensor(idx, vals, shape))
    fs = [np.random.default_rng(m).random((n, 8)).astype(np.float32) for m, n in enumerate(shape)]
    for mode in range(4):
        ref = orc.coo_mttkrp(idx, vals.astype(np.float64), shape,
                             [f.astype(np.float64) for f in fs], mode)
        assert rel_err(sp.mttkrp(fs, mode), ref) <= 1e-5
    sp.close()
    # heavy-headed Zipf indices: privatised heavy root rows
    shape = (2000, 1600, 200)
    idx, vals, _ = synth.zipf_coo(shape, 200000, seed=0xC3)
    coo = tb.CooTensor(idx, vals, shape)
    coo.deduplicate()
    assert coo.nnz() == 200000
    sp = tb.SparseTensor(coo)
    fs = [np.random.default_rng(m).random((n, 32)).astype(np.float32) for m, n in enumerate(shape)]
    for mode in range(3):
        ref = orc.coo_mttkrp(coo.indices(), coo.values().astype(np.float64), shape,
                             [f.astype(np.float64) for f in fs], mode)
        assert rel_err(sp.mttkrp(fs, mode), ref) <= 1e-5
    sp.close()


def test_sparse_cp_als_vs_dense_oracle(orc):
    shape = (40, 30, 20)
    X, _ = synth.dense_lowrank(shape, 4, seed=5, dist="uniform", noise=0.01)
    X[X < np.quantile(X, 0.5)] = 0.0  # half the entries are structural zeros
    nz = np.argwhere(X != 0)
    coo = tb.CooTensor(nz, X[tuple(nz.T)], shape)
    sp = tb.SparseTensor(coo)
    init = synth.init_factors(shape, 4, 5)
    res = sp.cp_als(4, 12, 0.0, init=init)
    _, info = orc.cp_als(X.astype(np.float64), 4, 12, 0.0, [f.astype(np.float64) for f in init])
    assert res.iters == 12
    assert abs(res.fit - info["fit"]) <= 1e-4, (res.fit, info["fit"])
    sp.close()


def test_device_zipf_generator_matches_numpy():
    import torch
    shape = (1000, 800, 100)
    idx, vals, dups = synth.zipf_coo(shape, 20000, seed=0xC3)
    cap = 4 * idx.shape[0]
    d_idx = torch.empty(cap * 3, dtype=torch.int64, device="cuda")
    d_val = torch.empty(cap, dtype=torch.float32, device="cuda")
    n = tb.synth_zipf_coo_dev(shape, 20000, 0xC3, d_idx.data_ptr(), d_val.data_ptr(), cap)
    torch.cuda.synchronize()
    assert n == idx.shape[0]
    assert np.array_equal(d_idx[:n * 3].cpu().numpy().reshape(n, 3), idx)
    assert np.array_equal(d_val[:n].cpu().numpy(), vals)
    m = tb.coo_deduplicate_dev(d_idx.data_ptr(), d_val.data_ptr(), n, shape)
    torch.cuda.synchronize()
    assert m == 20000
    coo = tb.CooTensor(idx, vals, shape)
    coo.deduplicate()
    assert np.array_equal(d_idx[:m * 3].cpu().numpy().reshape(m, 3), coo.indices())
    assert np.array_equal(d_val[:m].cpu().numpy(), coo.values())


def _zipf_device_coo(shape, nnz, seed):
    """Device-drawn Zipf(1.2) COO, merged; returns (SparseTensor, host idx, host vals)."""
    import torch
    cap = 12 * nnz
    d_idx = torch.empty(cap * 3, dtype=torch.int64, device="cuda")
    d_val = torch.empty(cap, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    n_raw = tb.synth_zipf_coo_dev(shape, nnz, seed, d_idx.data_ptr(), d_val.data_ptr(), cap)
    n = tb.coo_deduplicate_dev(d_idx.data_ptr(), d_val.data_ptr(), n_raw, shape)
    sp = tb.SparseTensor(d_indices=d_idx.data_ptr(), d_values=d_val.data_ptr(), nnz=n,
                         shape=shape)
    torch.cuda.synchronize()
    idx = d_idx[:3 * n].view(n, 3).cpu().numpy()
    vals = d_val[:n].cpu().numpy()
    return sp, idx, vals


def test_csf_mttkrp_at_scale(orc):
    """8e6 merged Zipf entries: every warp of the CSF kernel walks several
    tasks and heavy roots span many tasks."""
    shape = (40000, 32000, 4000)
    sp, idx, vals = _zipf_device_coo(shape, 8_000_000, 0xC3)
    rng = np.random.default_rng(3)
    for R in (32, 64):
        fs = [rng.random((n, R)).astype(np.float32) for n in shape]
        for mode in range(3):
            out = sp.mttkrp(fs, mode)
            ref = orc.coo_mttkrp(idx, vals.astype(np.float64), shape,
                                 [f.astype(np.float64) for f in fs], mode)
            assert rel_err(out, ref) <= 1e-5, (R, mode, rel_err(out, ref))
    sp.close()


def test_sparse_cp_als_fit_at_scale():
    """Sparse CP-ALS fit at 2e6 entries against an independent FP64 fit of the
    returned factors: ||X - Xhat||^2 = ||X||^2 - 2 sum_nz v Xhat + sum prod Grams."""
    shape = (20000, 16000, 2000)
    sp, idx, vals = _zipf_device_coo(shape, 2_000_000, 0xC4)
    R = 16
    init = synth.init_factors(shape, R, 0xC4)
    res = sp.cp_als(R, 6, 0.0, init=init)
    U = [f.astype(np.float64) for f in res.factors]
    v = vals.astype(np.float64)
    inner = 0.0
    for a in range(0, len(v), 500_000):
        sl = slice(a, a + 500_000)
        p = U[0][idx[sl, 0]] * U[1][idx[sl, 1]] * U[2][idx[sl, 2]]
        inner += float(v[sl] @ p.sum(axis=1))
    G = np.ones((R, R))
    for f in U:
        G *= f.T @ f
    xn = float(v @ v)
    fit = 1.0 - np.sqrt(max(xn - 2 * inner + G.sum(), 0.0)) / np.sqrt(xn)
    assert res.iters == 6
    assert abs(res.fit - fit) <= 1e-4, (res.fit, fit)
    assert res.fit < 1.0
    sp.close()


def test_dedup_and_csf_bit_exact_at_scale(orc):
    """Device-drawn Zipf(1.2) COO at 1.5e6 distinct entries (several million
    raw draws, heavy duplicates in the Zipf head): the device merge equals the
    restated CooTensor::deduplicate element for element, and the CSF of every
    mode order the sparse CP-ALS builds ([n, other modes by ascending size])
    plus the identity order equals the restated from_coo bit for bit."""
    import torch
    shape = (20000, 16000, 2000)
    nnz = 1_500_000
    cap = 12 * nnz
    d_idx = torch.empty(cap * 3, dtype=torch.int64, device="cuda")
    d_val = torch.empty(cap, dtype=torch.float32, device="cuda")
    n_raw = tb.synth_zipf_coo_dev(shape, nnz, 0xC3, d_idx.data_ptr(), d_val.data_ptr(), cap)
    torch.cuda.synchronize()
    raw_idx = d_idx[:3 * n_raw].view(n_raw, 3).cpu().numpy().copy()
    raw_val = d_val[:n_raw].cpu().numpy().copy()
    assert n_raw >= 2 * nnz  # the duplicates are heavy
    n = tb.coo_deduplicate_dev(d_idx.data_ptr(), d_val.data_ptr(), n_raw, shape)
    torch.cuda.synchronize()
    assert n == nnz
    oi, ov = orc.coo_deduplicate(raw_idx, raw_val)
    idx = d_idx[:3 * n].view(n, 3).cpu().numpy()
    vals = d_val[:n].cpu().numpy()
    assert np.array_equal(idx, oi)
    assert np.array_equal(vals.view(np.uint32), ov.view(np.uint32))
    coo = tb.CooTensor(idx, vals, shape)
    by_size = sorted(range(3), key=lambda m: shape[m])
    orders = [[m] + [o for o in by_size if o != m] for m in range(3)] + [[0, 1, 2]]
    for mo in orders:
        csf = tb.CsfTensor.from_coo(coo, mo)
        fp, fi, v = orc.csf_from_coo(idx, vals, mo)
        for l in range(3):
            assert np.array_equal(csf.fptr(l), fp[l]), (mo, l)
            assert np.array_equal(csf.fids(l), fi[l]), (mo, l)
        assert np.array_equal(csf.vals().view(np.uint32), v.view(np.uint32)), mo


def test_sparse_cp_als_trajectory_vs_fp64_coo_oracle(orc):
    """A C3-shaped run at 2e6 entries, rank 32, 6 iterations: the fit after
    every iteration within 1e-4 of the FP64 oracle running the same loop on
    the nonzeros (oracle.cp_als_coo) from the same init."""
    shape = (20000, 16000, 2000)
    sp, idx, vals = _zipf_device_coo(shape, 2_000_000, 0xC3)
    R = 32
    init = synth.init_factors(shape, R, 0xC3)
    res = sp.cp_als(R, 6, 0.0, init=init)
    _, info = orc.cp_als_coo(idx, vals, shape, R, 6, 0.0, init)
    assert res.iters == info["iters"] == 6
    err = np.abs(np.asarray(res.convergence.fit_history) - info["fit_history"])
    assert err.max() <= 1e-4, err
    sp.close()

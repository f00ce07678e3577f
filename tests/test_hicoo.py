"""HiCOO (crates/tenrso-sparse/src/hicoo.rs) against the oracle restatement
and the reference's own tests (hicoo.rs:369-575, the module example at
hicoo.rs:17-22): the device build bit-exact against oracle.hicoo_from_coo
(stable block sort, nothing merged), the accessors, iteration, to_coo and
to_dense, and the HiCOO MTTKRP (no reference implementation; hicoo.rs:30-34
names it) within 1e-5 relative of the FP64 COO MTTKRP definition."""
import ctypes as C

import numpy as np
import pytest

import tenrso_b200 as tb
from tenrso_b200 import _lib, synth


def coo(shape, entries):
    idx = np.array([e[0] for e in entries], np.int64).reshape(len(entries), len(shape))
    val = np.array([e[1] for e in entries], np.float32)
    return tb.CooTensor(idx, val, shape)


# ---- oracle pinned to the reference's cases (CPU) -----------------------

def test_oracle_module_example(orc):
    """hicoo.rs:17-22: block_shape [2,2,2]; (0,1,2), (1,0,3), (2,3,4) have
    block indices (0,0,1), (0,0,1), (1,1,2) and local coords (0,1,0), (1,0,1),
    (0,1,0)."""
    idx = np.array([[0, 1, 2], [1, 0, 3], [2, 3, 4]])
    bc, bp, lc, v = orc.hicoo_from_coo(idx, np.array([1, 2, 3], np.float32), [2, 2, 2])
    assert bc.tolist() == [[0, 0, 1], [1, 1, 2]]
    assert bp.tolist() == [0, 2, 3]
    assert lc.tolist() == [[0, 1, 0], [1, 0, 1], [0, 1, 0]]


@pytest.mark.parametrize("case", [
    # (shape, entries, block_shape, nnz, num_blocks) from hicoo.rs's tests
    ((8, 8, 8), [([0, 1, 2], 5.0), ([1, 0, 3], 6.0), ([4, 5, 6], 7.0)], [4, 4, 4], 3, 2),  # :370
    ((8, 8, 8), [([2, 3, 4], 42.0)], [4, 4, 4], 1, 1),                                    # :520
    ((4, 4, 4), [([0, 0, 0], 1.0), ([0, 1, 1], 2.0), ([1, 0, 1], 3.0)], [2, 2, 2], 3, 1),  # :533
    ((4, 4, 4), [([0, 0, 0], 1.0), ([2, 2, 2], 2.0)], [2, 2, 2], 2, 2),                    # :545
    ((4,) * 5, [([0, 0, 0, 0, 1], 1.0), ([2, 2, 2, 2, 2], 2.0)], [2] * 5, 2, 2),           # :556
])
def test_oracle_reference_counts(orc, case):
    shape, entries, bs, nnz, nb = case
    t = coo(shape, entries)
    bc, bp, lc, v = orc.hicoo_from_coo(t.indices(), t.values(), bs)
    assert len(v) == nnz and len(bc) == nb and bp[-1] == nnz


def test_oracle_stable_order_and_duplicates(orc):
    """Entries of one block keep their input order; duplicates stay."""
    idx = np.array([[3, 3], [0, 1], [1, 0], [0, 1], [2, 2]])
    v = np.array([1, 2, 3, 4, 5], np.float32)
    bc, bp, lc, vv = orc.hicoo_from_coo(idx, v, [2, 2])
    assert bc.tolist() == [[0, 0], [1, 1]]
    assert vv.tolist() == [2, 3, 4, 1, 5]
    assert lc.tolist() == [[0, 1], [1, 0], [0, 1], [1, 1], [0, 0]]


def test_block_shape_validation_without_device():
    """hicoo.rs:121-133 messages, from the Python mirror and from the C ABI
    (whose checks run before the context is used)."""
    t = coo((8, 8, 8), [([0, 1, 2], 1.0)])
    with pytest.raises(tb.TenrsoError, match=r"Invalid block shape: block_shape length 2 != ndim 3"):
        tb.HiCooTensor.from_coo(t, [4, 4])
    with pytest.raises(tb.TenrsoError, match="Invalid block shape: block_shape cannot contain zeros"):
        tb.HiCooTensor.from_coo(t, [4, 0, 4])
    lib = _lib.load()
    h = C.c_void_p()
    shape = np.array([8, 8, 8], np.int64)
    for bs, msg in (([4, 4], b"length 2 != ndim 3"), ([4, 0, 4], b"cannot contain zeros")):
        b = np.array(bs, np.int64)
        rc = lib.tsr_hicoo_create_f32(None, t.indices().ctypes.data, t.values().ctypes.data, 1, 3,
                                      shape.ctypes.data, b.ctypes.data, len(bs), C.byref(h))
        assert rc == 20 and msg in lib.tsr_last_error()
    b = np.array([512, 4, 4], np.int64)
    rc = lib.tsr_hicoo_create_f32(None, t.indices().ctypes.data, t.values().ctypes.data, 1, 3,
                                  shape.ctypes.data, b.ctypes.data, 3, C.byref(h))
    assert rc == 14  # sides above 256 do not fit the u8 local coordinates


# ---- the device (GPU) ---------------------------------------------------

def random_coo(shape, nnz, seed, dup_frac=0.1):
    rng = np.random.default_rng(seed)
    idx = np.stack([rng.integers(0, n, nnz) for n in shape], axis=1)
    nd = int(nnz * dup_frac)
    if nd:
        idx[-nd:] = idx[rng.integers(0, nnz - nd, nd)]
    return idx.astype(np.int64), rng.random(nnz, dtype=np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,bs,nnz", [
    ((8, 8, 8), (4, 4, 4), 40),
    ((37, 41, 29), (8, 16, 4), 3000),
    ((100, 90, 80), (128, 128, 128), 5000),
    ((300, 200, 100), (2, 3, 5), 20000),
    ((20, 19, 18, 17), (4, 4, 4, 4), 8000),
    ((6, 7, 5, 4, 3), (2, 2, 2, 2, 2), 500),
    ((2000, 1500), (64, 32), 50000),
])
def test_device_build_bit_exact(orc, shape, bs, nnz):
    idx, val = random_coo(shape, nnz, sum(shape))
    h = tb.HiCooTensor.from_coo(tb.CooTensor(idx, val, shape), bs)
    bc, bp, lc, v = orc.hicoo_from_coo(idx, val, bs)
    assert np.array_equal(h.block_coords(), bc)
    assert np.array_equal(h.block_ptrs(), bp)
    assert np.array_equal(h.local_coords(), lc)
    assert np.array_equal(h.values(), v)
    assert h.nnz() == nnz and h.num_blocks() == len(bc)
    # to_coo is the entries in block-major order; the multiset is preserved
    back = h.to_coo()
    a = sorted(zip(map(tuple, idx.tolist()), val.tolist()))
    b = sorted(zip(map(tuple, back.indices().tolist()), back.values().tolist()))
    assert a == b
    h.close()


@pytest.mark.gpu
def test_reference_cases_on_device():
    """hicoo.rs:369-575 through the device build."""
    h = tb.HiCooTensor.from_coo(coo((8, 8, 8), [([0, 1, 2], 5.0), ([1, 0, 3], 6.0),
                                                 ([4, 5, 6], 7.0)]), [4, 4, 4])
    assert h.shape() == [8, 8, 8] and h.nnz() == 3 and h.num_blocks() == 2
    e = tb.HiCooTensor.from_coo(tb.CooTensor.zeros([8, 8, 8]), [4, 4, 4])
    assert e.nnz() == 0 and e.num_blocks() == 0 and e.block_ptrs().tolist() == [0]
    it = tb.HiCooTensor.from_coo(coo((4, 4, 4), [([0, 0, 1], 1.0), ([2, 2, 2], 2.0)]), [2, 2, 2])
    nz = list(it.iter())
    assert ([0, 0, 1], 1.0) in nz and ([2, 2, 2], 2.0) in nz and len(nz) == 2
    d = tb.HiCooTensor.from_coo(coo((4, 4, 4), [([0, 0, 0], 1.0), ([2, 2, 2], 2.0)]), [2, 2, 2])
    dense = d.to_dense()
    assert dense[0, 0, 0] == 1.0 and dense[2, 2, 2] == 2.0 and dense[0, 1, 0] == 0.0
    dn = tb.HiCooTensor.from_coo(coo((10, 10, 10), [([0, 0, 0], 1.0), ([5, 5, 5], 2.0)]),
                                 [5, 5, 5])
    assert abs(dn.density() - 0.002) < 1e-6
    s1 = tb.HiCooTensor.from_coo(coo((8, 8, 8), [([2, 3, 4], 42.0)]), [4, 4, 4])
    assert list(s1.iter()) == [([2, 3, 4], 42.0)]
    g = tb.HiCooTensor.from_coo(coo((4, 4, 4), [([0, 0, 0], 1.0), ([0, 1, 1], 2.0),
                                                 ([1, 0, 1], 3.0)]), [2, 2, 2])
    assert g.num_blocks() == 1
    hd = tb.HiCooTensor.from_coo(coo((4,) * 5, [([0, 0, 0, 0, 1], 1.0),
                                                ([2, 2, 2, 2, 2], 2.0)]), [2] * 5)
    dd = hd.to_dense()
    assert hd.ndim() == 5 and dd[0, 0, 0, 0, 1] == 1.0 and dd[2, 2, 2, 2, 2] == 2.0
    # duplicates: to_dense assigns in block-major order, the later one wins
    dup = tb.HiCooTensor.from_coo(coo((4, 4), [([1, 1], 1.0), ([1, 1], 5.0)]), [2, 2])
    assert dup.nnz() == 2 and dup.to_dense()[1, 1] == 5.0


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.gpu
@pytest.mark.parametrize("shape,bs,nnz,R", [
    ((37, 41, 29), (8, 16, 4), 3000, 8),
    ((300, 200, 100), (128, 128, 128), 200000, 32),
    ((300, 200, 100), (16, 16, 16), 200000, 64),
    ((300, 200, 100), (128, 128, 128), 50000, 130),  # tile above 48 KB: direct atomics
    ((20, 19, 18, 17), (4, 4, 4, 4), 8000, 16),
    ((2000, 1500), (64, 32), 50000, 1),
])
def test_hicoo_mttkrp_vs_fp64_definition(orc, shape, bs, nnz, R):
    idx, val = random_coo(shape, nnz, R + len(shape))
    h = tb.HiCooTensor.from_coo(tb.CooTensor(idx, val, shape), bs)
    rng = np.random.default_rng(R)
    fs = [rng.random((n, R), dtype=np.float32) for n in shape]
    for mode in range(len(shape)):
        got = h.mttkrp(fs, mode)
        ref = orc.coo_mttkrp(idx, val, shape, [f.astype(np.float64) for f in fs], mode)
        assert _rel(got, ref) <= 1e-5, (mode, _rel(got, ref))
    h.close()


@pytest.mark.gpu
def test_hicoo_mttkrp_zipf_and_one_dense_block(orc):
    """Zipf(1.2) indices (heavy head blocks; 300k distinct coordinates, the
    raw draws with their duplicates), and a tensor whose entries all sit in
    one block."""
    shape = (5000, 4000, 3000)
    idx, val, _ = synth.zipf_coo(shape, 300_000, 0xB1)
    h = tb.HiCooTensor.from_coo(tb.CooTensor(idx, val, shape), (128, 128, 128))
    bc, bp, lc, v = orc.hicoo_from_coo(idx, val, (128, 128, 128))
    assert np.array_equal(h.block_ptrs(), bp) and np.array_equal(h.values(), v)
    R = 32
    rng = np.random.default_rng(5)
    fs = [rng.random((n, R), dtype=np.float32) for n in shape]
    for mode in range(3):
        ref = orc.coo_mttkrp(idx, val, shape, [f.astype(np.float64) for f in fs], mode)
        assert _rel(h.mttkrp(fs, mode), ref) <= 1e-5
    h.close()
    rng = np.random.default_rng(6)
    idx = rng.integers(0, 64, (20000, 3)).astype(np.int64)
    val = rng.random(20000, dtype=np.float32)
    h = tb.HiCooTensor.from_coo(tb.CooTensor(idx, val, (64, 64, 64)), (64, 64, 64))
    assert h.num_blocks() == 1
    fs = [rng.random((64, 16), dtype=np.float32) for _ in range(3)]
    for mode in range(3):
        ref = orc.coo_mttkrp(idx, val, (64, 64, 64), [f.astype(np.float64) for f in fs], mode)
        assert _rel(h.mttkrp(fs, mode), ref) <= 1e-5
    h.close()


@pytest.mark.gpu
def test_hicoo_mttkrp_errors():
    h = tb.HiCooTensor.from_coo(coo((8, 8, 8), [([0, 1, 2], 1.0)]), [4, 4, 4])
    fs = [np.ones((8, 4), np.float32)] * 3
    with pytest.raises(tb.TenrsoError) as e:
        h.mttkrp(fs, 3)
    assert e.value.status == 1
    h.close()

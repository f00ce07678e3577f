"""COO ingestion from text, after tenrso-sparse's io tests
(crates/tenrso-sparse/src/io.rs:374-493), plus FROSTT .tns round trips into
the CSF build. CPU only: these exercise host parsing and the CPU CSF layout."""
import io

import numpy as np
import pytest

import tenrso_b200 as tb


def test_header_parse_and_string():
    h = tb.MatrixMarketHeader.parse("%%MatrixMarket matrix coordinate real general")
    assert (h.format, h.data_type, h.symmetry) == ("coordinate", "real", "general")
    h = tb.MatrixMarketHeader("coordinate", "real", "symmetric")
    assert h.header_string() == "%%MatrixMarket matrix coordinate real symmetric"
    for bad, msg in (("Invalid header", "Invalid Matrix Market header format"),
                     ("%%MatrixMarket matrix dense real general", "Unknown format: dense"),
                     ("%%MatrixMarket matrix coordinate quaternion general",
                      "Unknown data type: quaternion"),
                     ("%%MatrixMarket matrix coordinate real odd", "Unknown symmetry: odd")):
        with pytest.raises(tb.SparseIoError, match=msg):
            tb.MatrixMarketHeader.parse(bad)


def test_read_simple_and_comments():
    coo = tb.read_matrix_market(b"%%MatrixMarket matrix coordinate real general\n"
                                b"3 3 3\n1 1 1.0\n2 2 2.0\n3 1 3.0\n")
    assert coo.nnz() == 3 and coo.shape() == [3, 3]
    assert coo.indices().tolist() == [[0, 0], [1, 1], [2, 0]]
    assert coo.values().tolist() == [1.0, 2.0, 3.0]
    coo = tb.read_matrix_market(io.StringIO("%%MatrixMarket matrix coordinate real general\n"
                                            "% This is a comment\n% Another comment\n"
                                            "3 3 2\n1 1 1.5\n2 2 2.5\n"))
    assert coo.nnz() == 2


def test_read_symmetric_skew_pattern():
    coo = tb.read_matrix_market(b"%%MatrixMarket matrix coordinate real symmetric\n"
                                b"3 3 2\n1 1 1.0\n2 1 2.0\n")
    assert coo.nnz() == 3
    assert coo.indices().tolist() == [[0, 0], [1, 0], [0, 1]]
    coo = tb.read_matrix_market(b"%%MatrixMarket matrix coordinate real skew-symmetric\n"
                                b"3 3 1\n3 1 4.0\n")
    assert coo.values().tolist() == [4.0, -4.0]
    coo = tb.read_matrix_market(b"%%MatrixMarket matrix coordinate pattern general\n"
                                b"3 3 2\n1 1\n2 2\n")
    assert coo.nnz() == 2 and coo.values()[0] == 1.0


@pytest.mark.parametrize("text,msg", [
    (b"Invalid header\n3 3 2\n1 1 1.0\n", "Invalid Matrix Market header format"),
    (b"%%MatrixMarket matrix array real general\n3 3\n", "Only coordinate format"),
    (b"%%MatrixMarket matrix coordinate real general\n3 3\n", "Invalid size line format"),
    (b"%%MatrixMarket matrix coordinate real general\n3 x 1\n1 1 1\n", "Invalid ncols"),
    (b"%%MatrixMarket matrix coordinate real general\n3 3 1\n1\n", "Invalid data line format"),
    (b"%%MatrixMarket matrix coordinate real general\n3 3 1\n0 1 1\n", "Invalid row index"),
    (b"%%MatrixMarket matrix coordinate real general\n3 3 1\n1 1\n", "Missing value"),
    (b"%%MatrixMarket matrix coordinate real general\n3 3 1\n1 1 z\n", "Invalid value"),
])
def test_read_errors(text, msg):
    with pytest.raises(tb.SparseIoError, match=msg):
        tb.read_matrix_market(text)


def test_out_of_bounds_entry_is_a_coo_error():
    with pytest.raises(tb.CooError, match="Index out of bounds"):
        tb.read_matrix_market(b"%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n")


def test_write_and_roundtrip(tmp_path):
    coo = tb.CooTensor([[0, 0], [1, 1], [2, 0]], [1.0, 2.0, 3.0], [3, 3])
    out = io.StringIO()
    tb.write_matrix_market(coo, out)
    s = out.getvalue()
    assert "%%MatrixMarket matrix coordinate real general" in s
    for frag in ("3 3 3", "1 1 1", "2 2 2", "3 1 3"):
        assert frag in s
    coo = tb.CooTensor([[0, 0], [1, 1], [0, 2]], [1.5, 2.5, 3.5], [2, 3])
    path = tmp_path / "m.mtx"
    tb.write_matrix_market(coo, str(path))
    back = tb.read_matrix_market(str(path))
    assert back.nnz() == coo.nnz() and back.shape() == coo.shape()
    assert np.array_equal(back.indices(), coo.indices())
    assert np.array_equal(back.values(), coo.values())
    with pytest.raises(tb.SparseIoError, match="Only 2D matrices supported, got 3D"):
        tb.write_matrix_market(tb.CooTensor([[0, 0, 0], [1, 1, 1]], [1.0, 2.0], [2, 2, 2]),
                               io.StringIO())


def test_tns_roundtrip_into_csf(tmp_path, orc):
    rng = np.random.default_rng(7)
    shape = (9, 7, 5)
    idx = np.stack([rng.integers(0, n, 300) for n in shape], axis=1)
    vals = rng.random(300).astype(np.float32)
    coo = tb.CooTensor(idx, vals, shape)
    path = tmp_path / "x.tns"
    tb.write_tns(coo, str(path))
    back = tb.read_tns(str(path), shape=shape)
    assert np.array_equal(back.indices(), idx)
    assert np.array_equal(back.values(), vals)  # shortest round-trip text of fp32
    # duplicates survive the reader; the merge and CSF build see the same COO
    ai, av = orc.coo_deduplicate(coo.indices(), coo.values())
    bi, bv = orc.coo_deduplicate(back.indices(), back.values())
    assert len(ai) < 300
    a = orc.csf_from_coo(ai, av, [0, 1, 2])
    b = orc.csf_from_coo(bi, bv, [0, 1, 2])
    for lvl in range(3):
        assert np.array_equal(a[0][lvl], b[0][lvl]) and np.array_equal(a[1][lvl], b[1][lvl])
    assert np.array_equal(a[2], b[2])


@pytest.mark.gpu
def test_tns_file_to_sparse_mttkrp(tmp_path, orc):
    """A .tns file read from disk feeds the device merge, CSF build and MTTKRP."""
    rng = np.random.default_rng(3)
    shape = (40, 30, 20)
    idx = np.stack([rng.integers(0, n, 5000) for n in shape], axis=1)
    vals = rng.random(5000).astype(np.float32)
    path = tmp_path / "x.tns"
    tb.write_tns(tb.CooTensor(idx, vals, shape), str(path))
    coo = tb.read_tns(str(path), shape=shape)
    coo.deduplicate()  # on the device, bit-exact with the restated merge
    oi, ov = orc.coo_deduplicate(idx, vals)
    assert np.array_equal(coo.indices(), oi) and np.array_equal(coo.values(), ov)
    sp = tb.SparseTensor(coo)
    fs = [rng.standard_normal((n, 16)).astype(np.float32) for n in shape]
    for mode in range(3):
        ref = orc.coo_mttkrp(oi, ov.astype(np.float64), shape,
                             [f.astype(np.float64) for f in fs], mode)
        out = sp.mttkrp(fs, mode)
        assert np.linalg.norm(out - ref) / np.linalg.norm(ref) <= 1e-5
    sp.close()


def test_tns_shape_inference_comments_and_errors():
    coo = tb.read_tns(io.StringIO("# FROSTT\n1 1 1 2.0\n\n3 2 4 -1.5\n% c\n"))
    assert coo.shape() == [3, 2, 4] and coo.nnz() == 2
    assert coo.indices().tolist() == [[0, 0, 0], [2, 1, 3]]
    with pytest.raises(tb.SparseIoError, match="expected 3 indices"):
        tb.read_tns(io.StringIO("1 1 1 2.0\n1 1 2.0\n"))
    with pytest.raises(tb.SparseIoError, match="Invalid index"):
        tb.read_tns(io.StringIO("0 1 1 2.0\n"))
    with pytest.raises(tb.SparseIoError, match="Shape has 2 modes"):
        tb.read_tns(io.StringIO("1 1 1 2.0\n"), shape=(2, 2))
    assert tb.read_tns(io.StringIO(""), shape=(2, 3)).nnz() == 0


def test_tns_fast_and_line_readers_agree(tmp_path, monkeypatch):
    rng = np.random.default_rng(9)
    shape = (50, 40, 30, 20)
    idx = np.stack([rng.integers(0, n, 20000) for n in shape], axis=1)
    vals = (rng.standard_normal(20000) * 10).astype(np.float32)
    path = tmp_path / "x.tns"
    tb.write_tns(tb.CooTensor(idx, vals, shape), str(path))
    fast = tb.read_tns(str(path))
    from tenrso_b200 import sparse_io
    monkeypatch.setattr(sparse_io, "_tns_columns", lambda src: None)
    slow = tb.read_tns(str(path))
    assert fast.shape() == slow.shape() == [int(i) + 1 for i in idx.max(axis=0)]
    assert np.array_equal(fast.indices(), slow.indices())
    assert np.array_equal(fast.values(), slow.values())
    assert np.array_equal(fast.values(), vals)


def test_tns_irregular_text_takes_the_line_reader():
    # '%' comments and integer-looking values parse the same either way
    coo = tb.read_tns(io.StringIO("% header\n1 2 3\n2 1 4\n"))
    assert coo.shape() == [2, 2] and coo.values().tolist() == [3.0, 4.0]
    with pytest.raises(tb.SparseIoError, match="Invalid value"):
        tb.read_tns(b"1 1 x\n")


def test_tns_trailing_comment_and_exponents_same_with_and_without_pandas(monkeypatch):
    """A '#' after the numbers of a data line is an error for both readers, and
    exponent-form values parse to the same fp32 bits either way."""
    from tenrso_b200 import sparse_io
    text = ("1 1 1 1.5e-3\n2 3 1 -7.25E+2\n1 2 2 3.4028234e38\n2 1 2 1e-45\n"
            "1 3 1 0.1\n2 2 2 123456789.123456789\n")
    bad = "1 1 1 2.0 # trailing note\n2 2 2 1.0\n"
    fast = tb.read_tns(io.StringIO(text))
    with pytest.raises(tb.SparseIoError) as e_fast:
        tb.read_tns(io.StringIO(bad))
    monkeypatch.setattr(sparse_io, "_tns_columns", lambda src: None)
    slow = tb.read_tns(io.StringIO(text))
    with pytest.raises(tb.SparseIoError) as e_slow:
        tb.read_tns(io.StringIO(bad))
    assert str(e_fast.value) == str(e_slow.value)
    assert fast.shape() == slow.shape()
    assert np.array_equal(fast.indices(), slow.indices())
    assert np.array_equal(fast.values().view(np.uint32), slow.values().view(np.uint32))

"""COO ingestion from text: Matrix Market (tenrso's reader and writer) and
FROSTT `.tns` (N-way; an extension, tenrso's io module reads matrices only).

  MatrixMarketHeader.parse / header_string   crates/tenrso-sparse/src/io.rs:87-169
  read_matrix_market                         crates/tenrso-sparse/src/io.rs:192-295
  write_matrix_market                        crates/tenrso-sparse/src/io.rs:317-357

The reader keeps tenrso's behaviour: coordinate format only, 1-based indices,
`pattern` entries read as 1.0, a symmetric off-diagonal entry also stored
mirrored (negated for skew-symmetric), entries in file order (the COO is not
sorted or merged; `CooTensor.deduplicate` does that). Errors carry tenrso's
messages, `SparseError::Conversion` wording included.

The result is a host `CooTensor`, which `SparseTensor` uploads and merges on
the GPU.
"""
from __future__ import annotations

import io
import os
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from .sparse import CooTensor

FORMATS = ("coordinate", "array")
DATA_TYPES = ("real", "complex", "integer", "pattern")
SYMMETRIES = ("general", "symmetric", "skew-symmetric", "hermitian")


class SparseIoError(ValueError):
    """tenrso's SparseError for the io module (Conversion or Other)."""


def _conversion(reason: str) -> SparseIoError:
    # error.rs:43-44 and :145 (SparseError::Conversion(ConversionError::Failed))
    return SparseIoError(f"Conversion error: Conversion failed: {reason}")


@dataclass
class MatrixMarketHeader:
    format: str = "coordinate"
    data_type: str = "real"
    symmetry: str = "general"

    @classmethod
    def parse(cls, line: str) -> "MatrixMarketHeader":
        """io.rs:89-140: five fields, `%%MatrixMarket matrix <format> <type> <symmetry>`."""
        parts = line.split()
        if len(parts) != 5 or parts[0] != "%%MatrixMarket" or parts[1] != "matrix":
            raise _conversion("Invalid Matrix Market header format")
        if parts[2] not in FORMATS:
            raise _conversion(f"Unknown format: {parts[2]}")
        if parts[3] not in DATA_TYPES:
            raise _conversion(f"Unknown data type: {parts[3]}")
        if parts[4] not in SYMMETRIES:
            raise _conversion(f"Unknown symmetry: {parts[4]}")
        return cls(parts[2], parts[3], parts[4])

    def header_string(self) -> str:
        return f"%%MatrixMarket matrix {self.format} {self.data_type} {self.symmetry}"


def _open_text(src) -> io.TextIOBase:
    if isinstance(src, (str, os.PathLike)):
        return open(src, "r")
    if isinstance(src, (bytes, bytearray)):
        return io.StringIO(bytes(src).decode())
    if isinstance(src, (io.BufferedIOBase, io.RawIOBase)):
        return io.TextIOWrapper(src)
    return src


def _parse_index(tok: str, what: str) -> int:
    try:
        v = int(tok)
    except ValueError:
        raise _conversion(f"Invalid {what}") from None
    if v < 1:  # 1-based; usize parse rejects negatives and 0 - 1 underflows
        raise _conversion(f"Invalid {what}")
    return v - 1


def read_matrix_market(src) -> CooTensor:
    """Read a coordinate Matrix Market matrix into a 2-way CooTensor (io.rs:192-295).

    `src` is a path, the file's bytes, or an open text or binary stream."""
    f = _open_text(src)
    close = isinstance(src, (str, os.PathLike))
    try:
        line = f.readline()
        header = MatrixMarketHeader.parse(line.strip())
        if header.format != "coordinate":
            raise _conversion("Only coordinate format is supported")
        while True:
            line = f.readline()
            if not line.strip().startswith("%"):
                break
        size = line.split()
        if len(size) != 3:
            raise _conversion("Invalid size line format")
        dims = []
        for tok, what in zip(size, ("nrows", "ncols", "nnz")):
            try:
                v = int(tok)
            except ValueError:
                raise _conversion(f"Invalid {what}") from None
            if v < 0:
                raise _conversion(f"Invalid {what}")
            dims.append(v)
        nrows, ncols, nnz = dims
        rows, cols, vals = [], [], []
        pattern = header.data_type == "pattern"
        for _ in range(nnz):
            parts = f.readline().split()
            if len(parts) < 2:
                raise _conversion("Invalid data line format")
            r = _parse_index(parts[0], "row index")
            c = _parse_index(parts[1], "column index")
            if pattern:
                v = 1.0
            elif len(parts) < 3:
                raise _conversion("Missing value in data line")
            else:
                try:
                    v = float(parts[2])
                except ValueError:
                    raise _conversion("Invalid value") from None
            rows.append(r)
            cols.append(c)
            vals.append(v)
            if r != c and header.symmetry == "symmetric":
                rows.append(c)
                cols.append(r)
                vals.append(v)
            elif r != c and header.symmetry == "skew-symmetric":
                rows.append(c)
                cols.append(r)
                vals.append(-v)
    finally:
        if close:
            f.close()
    idx = np.stack([np.asarray(rows, np.int64), np.asarray(cols, np.int64)], axis=1) \
        if rows else np.zeros((0, 2), np.int64)
    return CooTensor(idx, np.asarray(vals, np.float32), [nrows, ncols])


def write_matrix_market(coo: CooTensor, dst) -> None:
    """Write a 2-way CooTensor as `coordinate real general` (io.rs:317-357).

    `dst` is a path or a writable text stream. Entries go out in storage
    order with 1-based indices."""
    if coo.rank() != 2:
        raise SparseIoError(f"Only 2D matrices supported, got {coo.rank()}D")
    lines = [MatrixMarketHeader().header_string(),
             f"{coo.shape()[0]} {coo.shape()[1]} {coo.nnz()}"]
    idx, vals = coo.indices(), coo.values()
    lines += [f"{int(i) + 1} {int(j) + 1} {_fmt(v)}" for (i, j), v in zip(idx, vals)]
    _write_lines(dst, lines)


def _fmt(v) -> str:
    # shortest round-trip text of the fp32 value (Rust's Display prints
    # integral floats without a fraction: 1.0 -> "1")
    return np.format_float_positional(np.float32(v), trim="-")


def _write_lines(dst, lines) -> None:
    text = "\n".join(lines) + "\n"
    if isinstance(dst, (str, os.PathLike)):
        with open(dst, "w") as f:
            f.write(text)
    else:
        dst.write(text)


def _tns_columns(src):
    """Fast path: pandas' C tokenizer over whitespace-separated columns, or
    None when the text is anything but well-formed integer indices and a
    numeric value (the line-by-line reader then gives the exact error)."""
    try:
        import pandas as pd
    except ImportError:
        return None
    try:
        # no comment handling here: a '#' or '%' anywhere leaves non-numeric
        # tokens, and the file goes to the line-by-line reader; values parse
        # with correct rounding, as Python's float() does there
        df = pd.read_csv(src, sep=r"\s+", header=None, engine="c", skip_blank_lines=True,
                         float_precision="round_trip")
    except Exception:
        return None
    if df.shape[1] < 2 or df.isna().to_numpy().any():
        return None
    from pandas.api.types import is_integer_dtype, is_numeric_dtype
    idx = df.iloc[:, :-1]
    if not all(is_integer_dtype(t) for t in idx.dtypes):
        return None
    if not is_numeric_dtype(df.dtypes.iloc[-1]):
        return None
    idx = idx.to_numpy(np.int64)
    if idx.size and idx.min() < 1:
        return None
    return idx - 1, df.iloc[:, -1].to_numpy(np.float64)


def read_tns(src, shape: Optional[Sequence[int]] = None) -> CooTensor:
    """Read a FROSTT `.tns` tensor: one entry per line, N 1-based indices then
    the value; blank lines and lines starting with `#` or `%` are skipped.

    The order N is taken from the first entry and must be the same on every
    line. `shape` defaults to the largest index seen in each mode. Entries
    stay in file order (duplicates are kept for `CooTensor.deduplicate`).
    Large files are tokenised by pandas' C parser when it is installed; any
    irregular text goes through the line-by-line reader below."""
    if isinstance(src, (bytes, bytearray)):
        src = io.StringIO(bytes(src).decode())
    elif not isinstance(src, (str, os.PathLike)):
        src = io.StringIO(_open_text(src).read())  # replayable for the fallback
    cols = _tns_columns(src)
    if cols is not None:
        idx, vals = cols
        ndim = idx.shape[1]
        if shape is None:
            shape = (idx.max(axis=0) + 1).tolist() if len(idx) else None
        if shape is not None and len(shape) != ndim:
            raise _conversion(f"Shape has {len(shape)} modes but the entries have {ndim} indices")
        if shape is not None:
            return CooTensor(idx, vals.astype(np.float32), list(shape))
    if isinstance(src, io.StringIO):
        src.seek(0)
    f = _open_text(src)
    close = isinstance(src, (str, os.PathLike))
    ndim = None
    idx_rows, vals = [], []
    try:
        for lineno, line in enumerate(f, 1):
            s = line.strip()
            if not s or s[0] in "#%":
                continue
            parts = s.split()
            if ndim is None:
                ndim = len(parts) - 1
                if ndim < 1:
                    raise _conversion(f"Invalid data line format (line {lineno})")
            if len(parts) != ndim + 1:
                raise _conversion(f"Invalid data line format (line {lineno}): expected "
                                  f"{ndim} indices and a value")
            idx_rows.append([_parse_index(t, f"index (line {lineno})") for t in parts[:ndim]])
            try:
                vals.append(float(parts[ndim]))
            except ValueError:
                raise _conversion(f"Invalid value (line {lineno})") from None
    finally:
        if close:
            f.close()
    if ndim is None:
        if shape is None:
            raise _conversion("Empty tensor file and no shape given")
        ndim = len(shape)
    idx = np.asarray(idx_rows, np.int64).reshape(-1, ndim)
    if shape is None:
        shape = (idx.max(axis=0) + 1).tolist()
    elif len(shape) != ndim:
        raise _conversion(f"Shape has {len(shape)} modes but the entries have {ndim} indices")
    return CooTensor(idx, np.asarray(vals, np.float32), list(shape))


def write_tns(coo: CooTensor, dst) -> None:
    """Write a CooTensor in FROSTT `.tns` form (1-based indices, storage order)."""
    idx, vals = coo.indices(), coo.values()
    lines = [" ".join(str(int(i) + 1) for i in row) + " " + _fmt(v) for row, v in zip(idx, vals)]
    text = "\n".join(lines) + ("\n" if lines else "")
    if isinstance(dst, (str, os.PathLike)):
        with open(dst, "w") as f:
            f.write(text)
    else:
        dst.write(text)


"""Binary case format of the reference crate, read and written with numpy.

Mirrors ``io/loaders.rs`` and ``io/bin_format.rs`` of wgpu_solver_backend and
the writers of ``wgpu_solver_backend_convert_cli/src/main.rs:407-494`` and
``wgpu_solver_backend_cli/src/main.rs:445-464``:

* ``matrix.csr.bin``: u32 magic 0x43535231 ("CSR1"), u32 version 1, u32 n_rows,
  u32 n_cols, u32 nnz, 3 reserved u32, then row_ptr u32[n_rows+1],
  col_idx u32[nnz], values f32[nnz]; all little-endian.
* ``rhs.bin`` / ``x0.bin`` / ``x.bin`` / ``x_ref.bin``: u32 n, f32[n].
* ``block_starts.bin``: u32 len, u32[len].

Validation follows loaders.rs:44-212 and raises ``ValueError`` with the same
messages where the reference returns ``Err(String)``.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass

import numpy as np

MATRIX_MAGIC_CSR1 = 0x43535231


@dataclass
class CsrMatrixBin:
    n_rows: int
    n_cols: int
    nnz: int
    row_ptr: np.ndarray
    col_idx: np.ndarray
    values: np.ndarray


@dataclass
class CaseInputBin:
    a: CsrMatrixBin
    b: np.ndarray
    x0: np.ndarray
    block_starts: np.ndarray


def _read_u32(buf: bytes, pos: int, label: str):
    if pos + 4 > len(buf):
        raise ValueError(f"Unexpected EOF while reading {label}: need 4 bytes, have {len(buf) - pos}")
    return int.from_bytes(buf[pos:pos + 4], "little"), pos + 4


def _read_arr(buf: bytes, pos: int, count: int, dtype, label: str):
    nbytes = 4 * count
    if pos + nbytes > len(buf):
        have = (len(buf) - pos) // 4
        raise ValueError(f"Unexpected EOF while reading {label}[{have}]: need 4 bytes, have {(len(buf) - pos) % 4}")
    return np.frombuffer(buf, dtype=dtype, count=count, offset=pos).copy(), pos + nbytes


def load_csr_matrix_bin(path: str) -> CsrMatrixBin:
    """loaders.rs:44-124."""
    with open(path, "rb") as f:
        buf = f.read()
    pos = 0
    magic, pos = _read_u32(buf, pos, "magic")
    if magic != MATRIX_MAGIC_CSR1:
        raise ValueError(f"Bad matrix magic in {path}: expected 0x{MATRIX_MAGIC_CSR1:08x}, got 0x{magic:08x}")
    version, pos = _read_u32(buf, pos, "version")
    if version != 1:
        raise ValueError(f"Unsupported matrix version in {path}: expected 1, got {version}")
    n_rows, pos = _read_u32(buf, pos, "n_rows")
    n_cols, pos = _read_u32(buf, pos, "n_cols")
    nnz, pos = _read_u32(buf, pos, "nnz")
    for lab in ("reserved0", "reserved1", "reserved2"):
        _, pos = _read_u32(buf, pos, lab)
    row_ptr, pos = _read_arr(buf, pos, n_rows + 1, "<u4", "row_ptr")
    col_idx, pos = _read_arr(buf, pos, nnz, "<u4", "col_idx")
    values, pos = _read_arr(buf, pos, nnz, "<f4", "values")
    if row_ptr[0] != 0:
        raise ValueError("CSR row_ptr must start with 0")
    if row_ptr[-1] != nnz:
        raise ValueError(f"CSR row_ptr must end with nnz ({nnz}), got Some({row_ptr[-1]})")
    if n_rows > 0 and np.any(row_ptr[1:] < row_ptr[:-1]):
        raise ValueError("CSR row_ptr must be non-decreasing")
    max_col = int(col_idx.max()) if nnz else 0
    if n_cols > 0 and max_col >= n_cols:
        raise ValueError(f"CSR col_idx contains out-of-range column {max_col} for n_cols={n_cols}")
    if pos != len(buf):
        raise ValueError(f"matrix.csr.bin has {len(buf) - pos} trailing bytes after expected payload")
    return CsrMatrixBin(n_rows, n_cols, nnz, row_ptr.astype(np.uint32), col_idx.astype(np.uint32),
                        values.astype(np.float32))


def load_vector_bin(path: str) -> np.ndarray:
    """loaders.rs:126-144 (u32 n + f32[n])."""
    with open(path, "rb") as f:
        buf = f.read()
    n, pos = _read_u32(buf, 0, "n")
    vals, pos = _read_arr(buf, pos, n, "<f4", "values")
    if pos != len(buf):
        raise ValueError(f"{path} has {len(buf) - pos} trailing bytes after expected payload")
    return vals.astype(np.float32)


def load_block_starts_bin(path: str) -> np.ndarray:
    """loaders.rs:146-162 (u32 len + u32[len])."""
    with open(path, "rb") as f:
        buf = f.read()
    n, pos = _read_u32(buf, 0, "len")
    vals, pos = _read_arr(buf, pos, n, "<u4", "block_starts")
    if pos != len(buf):
        raise ValueError(f"{path} has {len(buf) - pos} trailing bytes after expected payload")
    return vals.astype(np.uint32)


def validate_block_starts(starts: np.ndarray, n: int) -> None:
    """loaders.rs:164-184."""
    if len(starts) == 0:
        raise ValueError("block_starts must not be empty")
    if starts[0] != 0:
        raise ValueError(f"block_starts must start with 0, got {starts[0]}")
    if starts[-1] != n:
        raise ValueError(f"block_starts must end with n ({n}), got {starts[-1]}")
    if np.any(starts[1:] <= starts[:-1]):
        raise ValueError("block_starts must be strictly increasing")


def load_case_dir(case_dir: str) -> CaseInputBin:
    """loaders.rs:8-42."""
    a = load_csr_matrix_bin(os.path.join(case_dir, "matrix.csr.bin"))
    b = load_vector_bin(os.path.join(case_dir, "rhs.bin"))
    x0 = load_vector_bin(os.path.join(case_dir, "x0.bin"))
    bs = load_block_starts_bin(os.path.join(case_dir, "block_starts.bin"))
    if a.n_rows != a.n_cols:
        raise ValueError(f"matrix must be square for PCG: got {a.n_rows}x{a.n_cols}")
    if len(b) != a.n_rows:
        raise ValueError(f"rhs length mismatch: b.n={len(b)} but matrix n_rows={a.n_rows}")
    if len(x0) != a.n_rows:
        raise ValueError(f"x0 length mismatch: x0.n={len(x0)} but matrix n_rows={a.n_rows}")
    validate_block_starts(bs, a.n_rows)
    return CaseInputBin(a, b, x0, bs)


def write_vector_bin(path: str, v) -> None:
    v = np.ascontiguousarray(v, dtype="<f4")
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "wb") as f:
        f.write(np.uint32(len(v)).astype("<u4").tobytes())
        f.write(v.tobytes())


def write_case_dir(out_dir: str, row_ptr, col_idx, values, b, x0, block_starts, x_ref=None) -> None:
    """Same files as convert_cli main.rs:407-494 (meta.json included)."""
    os.makedirs(out_dir, exist_ok=True)
    row_ptr = np.ascontiguousarray(row_ptr, "<u4")
    col_idx = np.ascontiguousarray(col_idx, "<u4")
    values = np.ascontiguousarray(values, "<f4")
    n = len(row_ptr) - 1
    hdr = np.array([MATRIX_MAGIC_CSR1, 1, n, n, len(col_idx), 0, 0, 0], "<u4")
    with open(os.path.join(out_dir, "matrix.csr.bin"), "wb") as f:
        f.write(hdr.tobytes())
        f.write(row_ptr.tobytes())
        f.write(col_idx.tobytes())
        f.write(values.tobytes())
    write_vector_bin(os.path.join(out_dir, "rhs.bin"), b)
    write_vector_bin(os.path.join(out_dir, "x0.bin"), x0)
    bs = np.ascontiguousarray(block_starts, "<u4")
    with open(os.path.join(out_dir, "block_starts.bin"), "wb") as f:
        f.write(np.uint32(len(bs)).astype("<u4").tobytes())
        f.write(bs.tobytes())
    if x_ref is not None:
        write_vector_bin(os.path.join(out_dir, "x_ref.bin"), x_ref)
    meta = dict(format="wgpu-solver-backend-text-v0", n=n, nnz=len(col_idx), row_ptr_len=len(row_ptr),
                col_idx_len=len(col_idx), values_len=len(values), rhs_len=len(b), x0_len=len(x0),
                block_starts_len=len(bs), x_ref_present=x_ref is not None)
    with open(os.path.join(out_dir, "meta.json"), "w") as f:
        f.write(json.dumps(meta, indent=2))

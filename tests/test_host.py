"""Host-side checks that need no GPU: the C ABI library loads and exports
every entry point of include/wsb.h; the host LU builder matches the oracle bit
for bit; input validation returns the reference's messages; the lattice
generator and the binary case format behave."""
import os
import re
import tempfile

import numpy as np
import pytest

import oracle
import wgpu_solver_backend_b200 as wsb
from wgpu_solver_backend_b200 import _lib
from wgpu_solver_backend_b200 import io as wio
from conftest import ROOT, load_case


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "wsb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(wsb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 50
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # The Python mirror declares a signature for each of them.
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


@pytest.mark.parametrize("k", [1, 2, 3])
def test_host_lu_builder_bit_exact_with_oracle(k):
    case, _, fx = load_case(k)
    a = case.a
    lu = wsb.build_lu_blocks_from_csr_block_starts_6(a.n_rows, a.row_ptr, a.col_idx, a.values, case.block_starts)
    assert np.array_equal(lu.view(np.uint32), fx["lu"].view(np.uint32))


def test_host_lu_builder_on_lattice_and_odd_blocks():
    s = wsb.lattice_generate(5, seed=3)
    lu = wsb.build_lu_blocks_from_csr_block_starts_6(s["n"], s["row_ptr"], s["col_idx"], s["values"],
                                                     s["block_starts"])
    st, lu2, _, _ = oracle.build_lu_blocks_6(s["n"], s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
    assert st == 0 and np.array_equal(lu.view(np.uint32), lu2.view(np.uint32))
    # Irregular partition: blocks of 1..9 rows (rows 6.. of long blocks unused).
    n = s["n"]
    rng = np.random.default_rng(1)
    cuts = [0]
    while cuts[-1] < n:
        cuts.append(min(n, cuts[-1] + int(rng.integers(1, 10))))
    bs = np.array(cuts, np.uint32)
    lu = wsb.build_lu_blocks_from_csr_block_starts_6(n, s["row_ptr"], s["col_idx"], s["values"], bs)
    st, lu2, _, _ = oracle.build_lu_blocks_6(n, s["row_ptr"], s["col_idx"], s["values"], bs)
    assert st == 0 and np.array_equal(lu.view(np.uint32), lu2.view(np.uint32))


def test_lu_errors_follow_reference_messages():
    mat = np.eye(6, dtype=np.float32).ravel().copy()
    mat[7] = 0.0  # (1,1)
    with pytest.raises(wsb.WsbError) as e:
        wsb.lu_factor_inplace_6(mat, 4)
    assert e.value.status == _lib.ZERO_PIVOT and "LU zero pivot at k = 1" in str(e.value)
    with pytest.raises(wsb.WsbError) as e:
        wsb.lu_factor_inplace_6(np.zeros(36, np.float32), 7)
    assert "n must be <= 6" in str(e.value)
    rp, ci, v = [0, 1, 2], [0, 1], [1.0, 1.0]
    with pytest.raises(wsb.WsbError) as e:
        wsb.build_lu_blocks_from_csr_block_starts_6(2, rp, ci, v, [0, 2, 2])
    assert "strictly increasing" in str(e.value)
    with pytest.raises(wsb.WsbError) as e:
        wsb.build_lu_blocks_from_csr_block_starts_6(2, rp, ci, v, [1, 2])
    assert "must start at 0" in str(e.value)
    with pytest.raises(wsb.WsbError) as e:
        wsb.build_lu_blocks_from_csr_block_starts_6(2, rp, ci, v, [0, 1])
    assert "last must equal n" in str(e.value)
    # Fewer than two starts: Ok(empty), compute.rs:111-113.
    assert wsb.build_lu_blocks_from_csr_block_starts_6(2, rp, ci, v, [0]).size == 0


def test_lattice_generator_sizes_symmetry_and_determinism():
    for side, n, nnz in [(10, 6000, 230400), (80, 3072000, 127641600), (4, 384, 36 * (64 + 2 * 144))]:
        sz = wsb.lattice_sizes(side)
        assert sz["n"] == n and sz["nnz"] == nnz
    s1 = wsb.lattice_generate(6, seed=11, aniso_log10=2.0)
    s2 = wsb.lattice_generate(6, seed=11, aniso_log10=2.0)
    for key in ("row_ptr", "col_idx", "values", "block_starts", "b"):
        assert np.array_equal(s1[key], s2[key])
    import scipy.sparse as sp

    A = sp.csr_matrix((s1["values"], s1["col_idx"], s1["row_ptr"]), shape=(s1["n"], s1["n"]))
    assert (A - A.T).count_nonzero() == 0
    assert np.all(np.diff(s1["block_starts"]) == 6)
    assert np.all(s1["b"] >= -1) and np.all(s1["b"] <= 1)
    # Sorted columns in every row.
    rp, ci = s1["row_ptr"], s1["col_idx"]
    for i in range(0, s1["n"], 37):
        assert np.all(np.diff(ci[rp[i]:rp[i + 1]].astype(np.int64)) > 0)


def test_case_dir_round_trip_and_validation():
    case, x_ref, _ = load_case(1)
    with tempfile.TemporaryDirectory() as d:
        wio.write_case_dir(d, case.a.row_ptr, case.a.col_idx, case.a.values, case.b, case.x0, case.block_starts,
                           x_ref)
        c2 = wio.load_case_dir(d)
        assert np.array_equal(c2.a.values, case.a.values) and np.array_equal(c2.b, case.b)
        # Trailing garbage is an error (loaders.rs:107-114).
        with open(os.path.join(d, "rhs.bin"), "ab") as f:
            f.write(b"\0")
        with pytest.raises(ValueError, match="trailing bytes"):
            wio.load_case_dir(d)


def _random_csr(rng, n, density):
    """Random square CSR with unsorted columns, duplicate entries in a row
    (the LU extraction keeps the later one) and some exact zeros."""
    rows, cols, vals = [], [], []
    for i in range(n):
        k = int(rng.binomial(n, density))
        cs = list(rng.integers(0, n, k)) + [i]
        if rng.random() < 0.3 and cs:
            cs.append(cs[0])  # a duplicate
        rng.shuffle(cs)
        for c in cs:
            rows.append(i)
            cols.append(int(c))
            v = float(rng.normal()) if rng.random() > 0.05 else 0.0
            vals.append(v + (4.0 if c == i and rng.random() > 0.1 else 0.0))
    rp = np.zeros(n + 1, np.uint32)
    np.add.at(rp, np.array(rows) + 1, 1)
    return np.cumsum(rp).astype(np.uint32), np.array(cols, np.uint32), np.array(vals, np.float32)


@pytest.mark.parametrize("seed", range(40))
def test_host_lu_builder_matches_oracle_on_random_systems(seed):
    """build_lu_blocks_from_csr_block_starts_6 (compute.rs:84-181) against
    the oracle's restatement on random systems: blocks of 1..9 rows, unsorted
    and duplicate columns, exact zeros. Same status, same first zero pivot
    (block order), and the same factor bits when it succeeds."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 60))
    rp, ci, v = _random_csr(rng, n, float(rng.uniform(0.02, 0.3)))
    cuts = [0]
    while cuts[-1] < n:
        cuts.append(min(n, cuts[-1] + int(rng.integers(1, 10))))
    bs = np.array(cuts, np.uint32)
    st, lu_o, bad, pk = oracle.build_lu_blocks_6(n, rp, ci, v, bs)
    if st == oracle.OK:
        lu = wsb.build_lu_blocks_from_csr_block_starts_6(n, rp, ci, v, bs)
        assert np.array_equal(lu.view(np.uint32), lu_o.view(np.uint32))
    else:
        assert st == oracle.ZERO_PIVOT
        with pytest.raises(wsb.WsbError) as e:
            wsb.build_lu_blocks_from_csr_block_starts_6(n, rp, ci, v, bs)
        assert e.value.status == _lib.ZERO_PIVOT and f"LU zero pivot at k = {pk}" in str(e.value)

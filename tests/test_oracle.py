"""Pins the CPU oracle against the reference's own golden data (CPU only).

* The three fea_app datasets with their x_ref sections, solved at the
  settings of commands.txt:26-54 and judged by the compare-x rule of
  wgpu_solver_backend_cli/src/main.rs:603-719 at commands.txt:56-78.
* The known answers of the five sanity subcommands, main.rs:171-443.
"""
import numpy as np
import pytest

import oracle
from conftest import COMPARE_X_GATES, DATASET_SOLVE, load_case


@pytest.mark.parametrize("k", [1, 2, 3])
def test_oracle_passes_reference_compare_x_on_datasets(k):
    case, x_ref, fx = load_case(k)
    a = case.a
    st, lu, _, _ = oracle.build_lu_blocks_6(a.n_rows, a.row_ptr, a.col_idx, a.values, case.block_starts)
    assert st == oracle.OK
    res = oracle.pcg_ref_f32(a.row_ptr, a.col_idx, a.values, lu, case.block_starts, case.b, case.x0,
                             DATASET_SOLVE["max_iter"], DATASET_SOLVE["rel_tol"], DATASET_SOLVE["abs_tol"])
    assert res["status"] == oracle.OK
    cmp = oracle.compare_x(x_ref, res["x"])
    rel_tol, abs_tol = COMPARE_X_GATES[k]
    assert cmp["rel_l2"] <= rel_tol or cmp["rmse"] <= abs_tol, cmp
    # The committed fixture is this oracle's output (regression pin).
    assert res["iterations"] == int(fx["iterations"])
    assert np.array_equal(res["x"].view(np.uint32), fx["x"].view(np.uint32))
    assert np.array_equal(lu.view(np.uint32), fx["lu"].view(np.uint32))


@pytest.mark.parametrize("k", [1, 2, 3])
def test_f64dot_variant_agrees_with_reference_restatement(k):
    case, x_ref, fx = load_case(k)
    a = case.a
    res = oracle.pcg_f64dot(a.row_ptr, a.col_idx, a.values, fx["lu"], case.block_starts, case.b, case.x0,
                            DATASET_SOLVE["max_iter"], DATASET_SOLVE["rel_tol"], DATASET_SOLVE["abs_tol"])
    assert res["status"] == oracle.OK
    it_ref = int(fx["iterations"])
    # FP64 accumulation on these cond 1e10-1e12 systems: 2% or 2 iterations.
    assert abs(res["iterations"] - it_ref) <= max(2, 0.02 * it_ref)
    cmp = oracle.compare_x(x_ref, res["x"])
    rel_tol, abs_tol = COMPARE_X_GATES[k]
    assert cmp["rel_l2"] <= rel_tol or cmp["rmse"] <= abs_tol


def test_known_answers_of_sanity_subcommands():
    # vec-test (main.rs:171-211): y = 1 + 3*2 = 7
    y = oracle.axpy(3.0, np.full(1024, 2.0, np.float32), np.ones(1024, np.float32))
    assert np.all(np.abs(y - 7.0) < 1e-6)
    # dot-test (main.rs:213-248): [1,2,3].[4,5,6] = 32
    assert abs(oracle.dot_tree256([1, 2, 3], [4, 5, 6]) - 32.0) < 1e-5
    # spmv-test (main.rs:250-315)
    y = oracle.spmv([0, 2, 4, 6], [0, 2, 0, 1, 1, 2], [10, 2, 3, 9, 7, 8], [1, 2, 3])
    assert np.array_equal(y, np.array([16, 21, 38], np.float32))
    # block-jacobi-test (main.rs:317-368): identity LU blocks, z == r
    lu = np.zeros(72, np.float32)
    for blk in range(2):
        for i in range(6):
            lu[blk * 36 + i * 6 + i] = 1.0
    r = np.arange(1, 13, dtype=np.float32)
    assert np.array_equal(oracle.block_jacobi_apply(12, lu, [0, 6, 12], r), r)
    # pcg-update-scalars-test (main.rs:370-443): slots PAP 0, RZ_NEW 1, RZ_OLD 2
    s = np.zeros(8, np.float32)
    s[0], s[2], s[1] = 2.0, 10.0, 5.0
    s = oracle.update_scalars(s, 0, 1, 2, 3, 4, 5)
    assert (s[3], s[4], s[5]) == (5.0, -5.0, 0.5)


def test_dot_tree_order_is_the_reference_tree():
    # 256-lane tree over chunks, then re-reduction: differs from a sequential
    # sum for values that cancel, and is exact for this construction.
    rng = np.random.default_rng(0)
    a = rng.standard_normal(70000).astype(np.float32)
    b = rng.standard_normal(70000).astype(np.float32)
    got = oracle.dot_tree256(a, b)
    # Recompute the tree in numpy with explicit float32 pairwise steps.
    prod = (a * b).astype(np.float32)
    pad = np.zeros(((len(prod) + 255) // 256) * 256, np.float32)
    pad[: len(prod)] = prod

    def tree(v):
        v = v.reshape(-1, 256).copy()
        off = 128
        while off >= 1:
            v[:, :off] = (v[:, :off] + v[:, off:2 * off]).astype(np.float32)
            off //= 2
        return v[:, 0]

    parts = tree(pad)
    while len(parts) > 1:
        p2 = np.zeros(((len(parts) + 255) // 256) * 256, np.float32)
        p2[: len(parts)] = parts
        parts = tree(p2)
    assert np.float32(parts[0]) == got
    assert oracle.dot_tree256(np.zeros(0, np.float32), np.zeros(0, np.float32)) == 0.0


def test_lu_zero_pivot_and_identity_padding():
    mat = np.zeros(36, np.float32)
    for i in range(6):
        mat[i * 6 + i] = 1.0
    mat[0] = 0.0
    st, k = oracle.lu_factor_inplace_6(mat, 3)
    assert st == oracle.ZERO_PIVOT and k == 0
    # A block of 3 rows: rows/cols 3..5 stay identity.
    rp = np.array([0, 1, 2, 3], np.uint32)
    ci = np.array([0, 1, 2], np.uint32)
    v = np.array([2.0, 4.0, 8.0], np.float32)
    st, lu, _, _ = oracle.build_lu_blocks_6(3, rp, ci, v, [0, 3])
    assert st == 0
    m = lu.reshape(6, 6)
    assert np.array_equal(np.diag(m), np.array([2, 4, 8, 1, 1, 1], np.float32))


@pytest.mark.parametrize("side,seed,aniso", [(1, 3, 0.0), (4, 7, 2.0), (7, 11, 3.0), (10, 2024, 0.0)])
def test_oracle_lattice_generator_matches_the_product_generator(side, seed, aniso):
    # The benchmark's CPU legs build their inputs with the oracle's generator
    # (so that they never load the product library); both must give the same
    # systems bit for bit.
    import wgpu_solver_backend_b200 as wsb

    a = oracle.lattice_generate(side, seed, aniso)
    b = wsb.lattice_generate(side, seed=seed, aniso_log10=aniso)
    assert a["n"] == b["n"] and a["nnz"] == b["nnz"]
    for k in ("row_ptr", "col_idx", "values", "block_starts", "b"):
        assert np.array_equal(a[k].view(np.uint32), b[k].view(np.uint32)), k


def test_many_reference_solves_equal_single_solves():
    # The batched CPU baseline runs orc_pcg_ref_f32 per system, concurrently
    # for small systems and with inner threads for large ones: same bits as
    # one solve at a time.
    systems = []
    for side, seed in ((3, 1), (5, 2), (4, 3), (6, 4)):
        s = oracle.lattice_generate(side, seed, 1.0)
        st, lu, _, _ = oracle.build_lu_blocks_6(s["n"], s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
        assert st == oracle.OK
        systems.append(dict(s, lu=lu))
    many = oracle.pcg_ref_f32_many(systems, 5000, 1e-6, 0.0, par_min_n=500)
    for s, m in zip(systems, many):
        one = oracle.pcg_ref_f32(s["row_ptr"], s["col_idx"], s["values"], s["lu"], s["block_starts"], s["b"],
                                 np.zeros(s["n"], np.float32), 5000, 1e-6, 0.0)
        assert m["status"] == one["status"] == oracle.OK
        assert m["iterations"] == one["iterations"]
        assert np.array_equal(m["x"].view(np.uint32), one["x"].view(np.uint32))

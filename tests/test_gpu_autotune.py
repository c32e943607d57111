"""Tile-size autotuner (wsb_matrix_autotune): it times candidate tilings of
the SpMV and update kernels, keeps the fastest, and later matrices of the same
shape class start with the recorded tiles. A tiling regroups the FP64 partial
sums of the dot products, so a retuned solve agrees with the untuned one to
FP64 rounding; matrices with the same tiles solve bit-identically."""
import numpy as np
import pytest

import wgpu_solver_backend_b200 as wsb

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("layout", [wsb.LAYOUT_BSR6, wsb.LAYOUT_CSR])
def test_autotune_choice_and_solutions(ctx, layout):
    wsb.autotune_clear()
    s = wsb.lattice_generate(12, seed=4, aniso_log10=1.0)
    args = (s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
    m0 = wsb.Matrix.create(ctx, *args, layout=layout)
    x0, r0 = m0.solve(s["b"], max_iter=5000, rel_tol=1e-6)
    m = wsb.Matrix.create(ctx, *args, layout=layout)
    t = m.autotune(iterations=4)
    assert t["candidates"] >= 2
    assert 0 < t["spmv_ms"] <= t["default_spmv_ms"] * 1.0000001
    assert 0 < t["update_ms"] <= t["default_update_ms"] * 1.0000001
    # Caps within the kernels' stages: SpMV tiles of at most 128 rows, update
    # tiles of at most 6 rows per consumer thread (768 with 128 consumers).
    assert 1 <= t["spmv_rows"] <= 128 and 1 <= t["spmv_cap"] and 6 <= t["update_rows"] <= 768
    assert t["update_blocks"] <= t["update_rows"]
    x1, r1 = m.solve(s["b"], max_iter=5000, rel_tol=1e-6)
    assert abs(int(r1["iterations"]) - int(r0["iterations"])) <= 1
    assert rel(x1, x0.astype(np.float64)) < 1e-6
    # A matrix of the same shape class created now starts with the tuned
    # tiles: its solve is bit-identical to the tuned matrix's.
    m2 = wsb.Matrix.create(ctx, *args, layout=layout)
    x2, r2 = m2.solve(s["b"], max_iter=5000, rel_tol=1e-6)
    assert r2["iterations"] == r1["iterations"]
    assert np.array_equal(x2.view(np.uint32), x1.view(np.uint32))
    wsb.autotune_clear()
    m3 = wsb.Matrix.create(ctx, *args, layout=layout)
    x3, r3 = m3.solve(s["b"], max_iter=5000, rel_tol=1e-6)
    assert r3["iterations"] == r0["iterations"] and np.array_equal(x3.view(np.uint32), x0.view(np.uint32))


def test_autotuned_matrix_in_a_batch_matches_alone(ctx):
    wsb.autotune_clear()
    s = wsb.lattice_generate(10, seed=8)
    o = wsb.lattice_generate(7, seed=9)
    m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
    m.autotune(iterations=4)
    mo = wsb.Matrix.create(ctx, o["row_ptr"], o["col_idx"], o["values"], o["block_starts"])
    xa, ra = m.solve(s["b"], max_iter=5000, rel_tol=1e-7)
    bt = wsb.Batch(ctx)
    bt.add(m, s["b"], max_iter=5000, rel_tol=1e-7)
    bt.add(mo, o["b"], max_iter=5000, rel_tol=1e-7)
    bt.solve()
    xb, rb = bt.result(0, s["n"])
    assert rb["iterations"] == ra["iterations"] and np.array_equal(xb.view(np.uint32), xa.view(np.uint32))
    wsb.autotune_clear()

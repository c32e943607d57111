"""Mixed precision, batched and served solves (GPU).

* MIXED_F64_IR reaches a true FP64 relative residual of 1e-10 and its error
  against the FP64 CPU PCG oracle is stated and bounded.
* A system's result is bit-identical alone, in a batch and in the server mix
  (per-system tiles and a fixed reduction order make the arithmetic
  independent of what else shares the launch).
"""
import numpy as np
import pytest

import oracle
import wgpu_solver_backend_b200 as wsb

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64)) / np.linalg.norm(b))


@pytest.mark.parametrize("side,aniso", [(6, 0.0), (8, 3.0)])
def test_mixed_precision_reaches_1e_10_against_fp64_oracle(ctx, side, aniso):
    s = wsb.lattice_generate(side, seed=17, aniso_log10=aniso)
    m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
    x64 = np.zeros(s["n"], np.float64)
    x, res = m.solve(s["b"], max_iter=20000, rel_tol=0.0, precision=wsb.PREC_MIXED_F64_IR,
                     target_relres=1e-10, x64_out=x64)
    assert res["rc"] == 0 and res["refine_sweeps"] >= 1
    tr = oracle.true_relres_f64(s["row_ptr"], s["col_idx"], s["values"], s["b"], x64)
    assert tr <= 1e-10, tr
    # The device's FP64 residual and the oracle's differ only by the rounding
    # of the residual sums themselves (a few percent at relres 1e-11).
    assert abs(tr - res["final_relres"]) <= 0.05 * tr + 1e-12
    ref = oracle.pcg_f64(s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], s["b"], rel_tol=1e-13,
                         max_iter=200000)
    assert ref["status"] == 0
    err = rel(x64, ref["x"])
    # Error bound: relres 1e-10 times a condition-number factor of the system.
    assert err < 1e-6, err
    assert np.array_equal(x, x64.astype(np.float32))


def _systems():
    out = []
    for i, (side, aniso) in enumerate([(4, 0.0), (7, 1.0), (5, 2.0), (9, 0.0), (3, 0.0), (6, 1.5)]):
        s = wsb.lattice_generate(side, seed=100 + i, aniso_log10=aniso)
        out.append(s)
    return out


def test_batch_results_identical_to_alone(ctx):
    systems = _systems()
    mats = [wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"]) for s in systems]
    precs = [wsb.PREC_F32_F64DOT, wsb.PREC_MIXED_F64_IR] * 3
    alone = []
    for m, s, p in zip(mats, systems, precs):
        alone.append(m.solve(s["b"], max_iter=5000, rel_tol=1e-8, precision=p, raise_on_error=False))
    bt = wsb.Batch(ctx)
    ids = [bt.add(m, s["b"], max_iter=5000, rel_tol=1e-8, precision=p) for m, s, p in zip(mats, systems, precs)]
    bt.solve()
    for i, (m, s) in enumerate(zip(mats, systems)):
        x, r = bt.result(ids[i], s["n"])
        xa, ra = alone[i]
        assert r["rc"] == ra["rc"] and r["iterations"] == ra["iterations"], (i, r, ra)
        assert np.array_equal(x.view(np.uint32), xa.view(np.uint32)), i


def test_server_results_identical_to_alone_and_budget(ctx):
    systems = _systems()
    precs = [wsb.PREC_F32_F64DOT, wsb.PREC_MIXED_F64_IR] * 3
    alone = []
    for s, p in zip(systems, precs):
        m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
        alone.append(m.solve(s["b"], max_iter=5000, rel_tol=1e-8, precision=p, raise_on_error=False))
    srv = wsb.Server(ctx, memory_budget_bytes=64 << 20, iters_per_step=8)
    try:
        rids = [srv.submit(s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], s["b"], max_iter=5000,
                           rel_tol=1e-8, precision=p) for s, p in zip(systems, precs)]
        for i, rid in enumerate(rids):
            x, r = srv.wait(rid, 120.0)
            xa, ra = alone[i]
            assert r["rc"] == ra["rc"] and r["iterations"] == ra["iterations"], (i, r, ra)
            assert np.array_equal(x.view(np.uint32), xa.view(np.uint32)), i
            assert r["total_ms"] > 0
        # A request larger than the whole budget is rejected, not queued forever.
        big = wsb.lattice_generate(40, seed=1)  # ~130 MB of CSR
        rid = srv.submit(big["row_ptr"], big["col_idx"], big["values"], big["block_starts"], big["b"],
                         max_iter=10, rel_tol=1e-8)
        x, r = srv.wait(rid, 60.0)
        assert r["rc"] == wsb._lib.OUT_OF_MEMORY
        st = srv.stats()
        assert st["completed"] == len(systems) and st["rejected"] == 1
        assert st["device_bytes_peak"] <= 64 << 20
    finally:
        srv.close()


def test_server_overlapping_arrivals(ctx):
    """Requests submitted while others iterate are admitted at step
    boundaries and all finish with the same answers as alone."""
    import time

    systems = [wsb.lattice_generate(side, seed=200 + side) for side in (10, 4, 6, 12, 5, 8, 3, 7)]
    srv = wsb.Server(ctx, iters_per_step=4)
    try:
        rids = []
        for s in systems:
            rids.append(srv.submit(s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], s["b"],
                                   max_iter=5000, rel_tol=1e-6))
            time.sleep(0.002)
        res = [srv.wait(r, 120.0) for r in rids]
    finally:
        srv.close()
    for s, (x, r) in zip(systems, res):
        m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
        xa, ra = m.solve(s["b"], max_iter=5000, rel_tol=1e-6)
        assert r["rc"] == 0 and r["iterations"] == ra["iterations"]
        assert np.array_equal(x, xa)


@pytest.mark.parametrize("borrow,device_prep", [(True, False), (False, True), (True, True)])
def test_server_borrowed_inputs_and_device_preparation(ctx, borrow, device_prep):
    """The server's options change where the work happens, not the answers:
    borrowed inputs (read in place, no copy at submit) and GPU-side
    preparation (column check, BSR6 conversion and LU on the device) give
    each request the same iterations and bits as solving it alone, and a
    request whose first block has a zero pivot fails with the LU message."""
    systems = _systems()
    precs = [wsb.PREC_F32_F64DOT, wsb.PREC_MIXED_F64_IR] * 3
    alone = []
    for s, p in zip(systems, precs):
        m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
        alone.append(m.solve(s["b"], max_iter=5000, rel_tol=1e-8, precision=p, raise_on_error=False))
    bad = wsb.lattice_generate(3, seed=5)
    vals = bad["values"].copy()
    vals[: bad["row_ptr"][6]] = 0.0  # rows 0..5: the first 6x6 block is all zero
    srv = wsb.Server(ctx, iters_per_step=8, borrow_inputs=borrow, device_prep=device_prep)
    try:
        rids = [srv.submit(s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], s["b"], max_iter=5000,
                           rel_tol=1e-8, precision=p) for s, p in zip(systems, precs)]
        rbad = srv.submit(bad["row_ptr"], bad["col_idx"], vals, bad["block_starts"], bad["b"], max_iter=100,
                          rel_tol=1e-8)
        for i, rid in enumerate(rids):
            x, r = srv.wait(rid, 120.0)
            xa, ra = alone[i]
            assert r["rc"] == ra["rc"] and r["iterations"] == ra["iterations"], (i, r, ra)
            assert np.array_equal(x.view(np.uint32), xa.view(np.uint32)), i
        _, r = srv.wait(rbad, 60.0)
        assert r["rc"] == wsb._lib.ZERO_PIVOT
        assert "LU zero pivot at k = 0" in ctx.last_error()
        st = srv.stats()
        assert st["completed"] == len(systems) and st["failed"] == 1
        if device_prep:
            assert st["host_prep_ms"] == 0.0
    finally:
        srv.close()


def test_server_slot_reuse_while_a_large_request_runs(ctx):
    """Small requests retire and new ones take their slots while one large
    request keeps iterating: the engine leaves a stopped system's tiles in
    its work lists (skipped) until a quarter of the listed tiles have
    stopped, so a new system in a slot the lists still name must force the
    lists to be laid out again. Every answer is bit-identical to a solve
    alone."""
    import time

    big = wsb.lattice_generate(24, seed=300)
    smalls = [wsb.lattice_generate(side, seed=310 + i) for i, side in enumerate((4, 5, 3, 6, 4, 5, 3, 4))]
    srv = wsb.Server(ctx, iters_per_step=4)
    try:
        rid_big = srv.submit(big["row_ptr"], big["col_idx"], big["values"], big["block_starts"], big["b"],
                             max_iter=20000, rel_tol=1e-8)
        rids, got = [], {}
        for s in smalls:
            rid = srv.submit(s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], s["b"], max_iter=5000,
                             rel_tol=1e-6)
            rids.append(rid)
            if len(rids) % 2 == 0:
                got[rid] = srv.wait(rid, 120.0)  # retired before the next one is submitted
            else:
                time.sleep(0.001)
        res = [got[r] if r in got else srv.wait(r, 120.0) for r in rids]
        xb, rb = srv.wait(rid_big, 300.0)
        st = srv.stats()
    finally:
        srv.close()
    assert st["completed"] == len(smalls) + 1
    for s, (x, r) in zip(smalls, res):
        m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
        xa, ra = m.solve(s["b"], max_iter=5000, rel_tol=1e-6)
        assert r["rc"] == 0 and r["iterations"] == ra["iterations"]
        assert np.array_equal(x.view(np.uint32), xa.view(np.uint32))
    m = wsb.Matrix.create(ctx, big["row_ptr"], big["col_idx"], big["values"], big["block_starts"])
    xa, ra = m.solve(big["b"], max_iter=20000, rel_tol=1e-8)
    assert rb["rc"] == 0 and rb["iterations"] == ra["iterations"]
    assert np.array_equal(xb.view(np.uint32), xa.view(np.uint32))

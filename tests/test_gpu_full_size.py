"""Full-size checks through properties that need no oracle run at that size.

* The plain 80^3 lattice (n = 3,072,000, nnz = 127,641,600, BSR6 tiles):
  the solve converges; it is exactly homogeneous (b -> 2b gives the same
  iterations and x -> 2x bit for bit, since scaling by a power of two is
  exact in every FP32 and FP64 operation of the recurrence); the CSR layout
  gives the same iterations and bits; FP64 refinement reaches a true FP64
  relative residual of 1e-8, checked on the host.
* A batch of 512 systems of lattice side 4..24: every system converges, and
  a sample solves bit-identically alone.
"""
import numpy as np
import pytest

import oracle
import wgpu_solver_backend_b200 as wsb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lattice80():
    s = wsb.lattice_generate(80, seed=2024)
    assert s["n"] == 3_072_000 and len(s["values"]) == 127_641_600
    return s


def test_80cubed_converges_and_is_homogeneous(ctx, lattice80):
    s = lattice80
    m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
    assert m.info["layout"] == wsb.LAYOUT_BSR6
    x, r = m.solve(s["b"], max_iter=20000, rel_tol=1e-6)
    assert r["rc"] == 0 and 0 < r["iterations"] < 20000
    assert r["final_relres"] <= 1e-6 * (1 + 1e-6)
    b2 = (2.0 * s["b"]).astype(np.float32)
    x2, r2 = m.solve(b2, max_iter=20000, rel_tol=1e-6)
    assert r2["iterations"] == r["iterations"]
    assert np.array_equal(x2.view(np.uint32), (2.0 * x).astype(np.float32).view(np.uint32))
    # The CSR layout: same row sums in the same order, same iterations and bits.
    mc = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], layout=wsb.LAYOUT_CSR)
    xc, rc = mc.solve(s["b"], max_iter=20000, rel_tol=1e-6)
    assert rc["iterations"] == r["iterations"]
    assert np.array_equal(xc.view(np.uint32), x.view(np.uint32))


def test_80cubed_refinement_reaches_true_fp64_relres(ctx, lattice80):
    s = lattice80
    m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
    x64 = np.zeros(s["n"], np.float64)
    x, r = m.solve(s["b"], max_iter=60000, rel_tol=0.0, precision=wsb.PREC_MIXED_F64_IR, target_relres=1e-8,
                   x64_out=x64)
    assert r["rc"] == 0 and r["refine_sweeps"] >= 1
    tr = oracle.true_relres_f64(s["row_ptr"], s["col_idx"], s["values"], s["b"], x64)
    assert tr <= 1e-8, tr
    assert abs(tr - r["final_relres"]) <= 0.05 * tr + 1e-12
    assert np.array_equal(x, x64.astype(np.float32))


def test_batch_of_512_systems(ctx):
    rng = np.random.default_rng(512)
    sides = rng.integers(4, 25, 512)
    systems = [wsb.lattice_generate(int(sd), seed=50_000 + i) for i, sd in enumerate(sides)]
    mats = [wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"]) for s in systems]
    bt = wsb.Batch(ctx)
    ids = [bt.add(m, s["b"], max_iter=20000, rel_tol=1e-6) for m, s in zip(mats, systems)]
    bt.solve()
    results = [bt.result(i, s["n"]) for i, s in zip(ids, systems)]
    assert all(r["rc"] == 0 and r["final_relres"] <= 1e-6 * (1 + 1e-6) for _, r in results)
    for i in rng.choice(512, 8, replace=False):
        xa, ra = mats[i].solve(systems[i]["b"], max_iter=20000, rel_tol=1e-6)
        xb, rb = results[i]
        assert rb["iterations"] == ra["iterations"], i
        assert np.array_equal(xb.view(np.uint32), xa.view(np.uint32)), i

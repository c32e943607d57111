"""Device-side preparation of a system (matrix creation): the block-Jacobi LU
factors built on the GPU are bit-identical to the host builder's
(build_lu_blocks_from_csr_block_starts_6, compute.rs:84-181), the BSR6
conversion gives the same SpMV bits as CSR, and the input errors carry the
reference's messages."""
import numpy as np
import pytest

import oracle
import wgpu_solver_backend_b200 as wsb
from conftest import load_case

pytestmark = pytest.mark.gpu


def _irregular(side, seed):
    s = wsb.lattice_generate(side, seed=seed)
    rng = np.random.default_rng(seed)
    cuts = [0]
    while cuts[-1] < s["n"]:
        cuts.append(min(s["n"], cuts[-1] + int(rng.integers(1, 10))))
    s["block_starts"] = np.array(cuts, np.uint32)
    return s


def _host_lu(s):
    return wsb.build_lu_blocks_from_csr_block_starts_6(s["n"], s["row_ptr"], s["col_idx"], s["values"],
                                                        s["block_starts"])


@pytest.mark.parametrize("k", [1, 2, 3])
def test_device_lu_bit_identical_on_datasets(ctx, k):
    case, _, _ = load_case(k)
    rp, ci, v, bs = case.a.row_ptr, case.a.col_idx, case.a.values, case.block_starts
    m = wsb.Matrix.create(ctx, rp, ci, v, bs)
    host = wsb.build_lu_blocks_from_csr_block_starts_6(len(rp) - 1, rp, ci, v, bs)
    assert np.array_equal(m.lu().view(np.uint32), host.view(np.uint32))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_device_lu_bit_identical_on_irregular_blocks(ctx, seed):
    s = _irregular(6, seed)
    m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
    assert m.info["layout"] == wsb.LAYOUT_CSR
    assert np.array_equal(m.lu().view(np.uint32), _host_lu(s).view(np.uint32))


@pytest.mark.parametrize("side,aniso", [(7, 0.0), (16, 2.0)])
def test_device_bsr6_conversion_and_lu(ctx, side, aniso):
    s = wsb.lattice_generate(side, seed=3, aniso_log10=aniso)
    mb = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
    assert mb.info["layout"] == wsb.LAYOUT_BSR6
    assert mb.info["num_blocks"] == s["n"] // 6
    assert np.array_equal(mb.lu().view(np.uint32), _host_lu(s).view(np.uint32))
    mc = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], layout=wsb.LAYOUT_CSR)
    # Same iterations and solution bits from both layouts, and the FP64-dot
    # oracle's iteration count.
    xb, rb = mb.solve(s["b"], max_iter=5000, rel_tol=1e-6)
    xc, rc = mc.solve(s["b"], max_iter=5000, rel_tol=1e-6)
    assert rb["iterations"] == rc["iterations"]
    assert np.array_equal(xb.view(np.uint32), xc.view(np.uint32))
    f64 = oracle.pcg_f64dot(s["row_ptr"], s["col_idx"], s["values"], _host_lu(s), s["block_starts"], s["b"],
                            np.zeros(s["n"], np.float32), 5000, 1e-6, 0.0)
    assert rb["iterations"] == f64["iterations"]


def test_bsr6_refused_for_incomplete_blocks(ctx):
    s = _irregular(4, 5)
    with pytest.raises(wsb.WsbError) as e:
        wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], layout=wsb.LAYOUT_BSR6)
    assert e.value.status == wsb._lib.BAD_INPUT and "BSR6 layout needs" in str(e.value)


def test_out_of_range_column_rejected(ctx):
    rp, ci, v, bs = [0, 1, 2], [0, 5], [1.0, 1.0], [0, 2]
    with pytest.raises(wsb.WsbError) as e:
        wsb.Matrix.create(ctx, rp, ci, v, bs)
    assert e.value.status == wsb._lib.BAD_INPUT
    assert "out-of-range column 5 for n_cols=2" in str(e.value)


def test_first_zero_pivot_block_reported(ctx):
    # Block 0 is fine, blocks 1 and 2 have a zero pivot at k = 1 and k = 0:
    # the first failing block in block order is reported, as the host loop.
    rp = [0, 1, 3, 5, 6, 7]
    ci = [0, 1, 2, 1, 2, 3, 4]
    v = [2.0, 1.0, 1.0, 1.0, 1.0, 0.0, 1.0]
    bs = [0, 1, 3, 4, 5]
    with pytest.raises(wsb.WsbError) as e:
        wsb.Matrix.create(ctx, rp, ci, v, bs)
    assert e.value.status == wsb._lib.ZERO_PIVOT and "LU zero pivot at k = 1" in str(e.value)
    with pytest.raises(wsb.WsbError) as eh:
        wsb.build_lu_blocks_from_csr_block_starts_6(5, np.array(rp, np.uint32), np.array(ci, np.uint32),
                                                     np.array(v, np.float32), np.array(bs, np.uint32))
    assert eh.value.status == wsb._lib.ZERO_PIVOT and "LU zero pivot at k = 1" in str(eh.value)

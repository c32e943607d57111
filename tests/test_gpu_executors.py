"""The five sanity subcommands of the reference CLI (main.rs:171-443) with
their known answers, through the executor entry points; and bit-exactness of
each executor against the oracle's restatement of its WGSL pass."""
import numpy as np
import pytest

import oracle
import wgpu_solver_backend_b200 as wsb

pytestmark = pytest.mark.gpu


def test_vec_test(ctx):
    x = ctx.create_storage_buffer(np.full(1024, 2.0, np.float32))
    y = ctx.create_storage_buffer(np.ones(1024, np.float32))
    wsb.VecOpsExecutor.create(ctx).encode_axpy_inplace(x, y, 1024, 3.0)
    assert np.all(np.abs(ctx.readback(y) - 7.0) < 1e-6)


def test_dot_test(ctx):
    a = ctx.create_storage_buffer(np.array([1, 2, 3], np.float32))
    b = ctx.create_storage_buffer(np.array([4, 5, 6], np.float32))
    ex = wsb.DotScalarExecutor.create(ctx, 3, 4)
    ex.encode_dot_scalar_into(a, b, 3, 0)
    assert abs(ex.readback_scalar_results()[0] - 32.0) < 1e-5
    with pytest.raises(wsb.WsbError, match="out_index out of range"):
        ex.encode_dot_scalar_into(a, b, 3, 4)


def test_spmv_test(ctx):
    ex = wsb.SpmvExecutor.create(ctx, 3, [0, 2, 4, 6], [0, 2, 0, 1, 1, 2], [10, 2, 3, 9, 7, 8])
    x = ctx.create_storage_buffer(np.array([1, 2, 3], np.float32))
    y = ctx.create_storage_buffer_uninit(3)
    ex.spmv(x, y)
    assert np.array_equal(ctx.readback(y), np.array([16, 21, 38], np.float32))


def test_block_jacobi_test(ctx):
    lu = np.zeros(72, np.float32)
    for blk in range(2):
        for i in range(6):
            lu[blk * 36 + i * 6 + i] = 1.0
    r = np.arange(1, 13, dtype=np.float32)
    bj = wsb.BlockJacobiExecutor.create(ctx, 12, lu, [0, 6, 12])
    rb = ctx.create_storage_buffer(r)
    zb = ctx.create_storage_buffer_uninit(12)
    bj.encode_apply(rb, zb)
    assert np.array_equal(ctx.readback(zb), r)


def test_pcg_update_scalars_test(ctx):
    host = np.zeros(8, np.float32)
    host[0], host[2], host[1] = 2.0, 10.0, 5.0  # PAP 0, RZ_OLD 2, RZ_NEW 1
    s = ctx.create_storage_buffer(host)
    wsb.PcgUpdateScalarsExecutor.create(ctx).encode_update_scalars(s, 0, 1, 2, 3, 4, 5)
    out = ctx.readback(s)
    assert (out[3], out[4], out[5]) == (5.0, -5.0, 0.5)
    # Zero denominators give 0 (pcg_update_scalars.wgsl:54-67).
    s2 = ctx.create_storage_buffer(np.zeros(8, np.float32))
    wsb.PcgUpdateScalarsExecutor.create(ctx).encode_update_scalars(s2, 0, 1, 2, 3, 4, 5)
    assert np.all(ctx.readback(s2)[3:6] == 0.0)


@pytest.mark.parametrize("n", [1, 255, 256, 257, 65536, 65537, 300001])
def test_dot_executor_bit_exact_with_tree_oracle(ctx, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n).astype(np.float32)
    b = rng.standard_normal(n).astype(np.float32)
    ex = wsb.DotScalarExecutor.create(ctx, n, 2)
    ex.encode_dot_scalar_into(ctx.create_storage_buffer(a), ctx.create_storage_buffer(b), n, 1)
    got = ex.readback_scalar_results()[1]
    assert np.float32(got).view(np.uint32) == np.float32(oracle.dot_tree256(a, b)).view(np.uint32)


def test_spmv_and_block_jacobi_bit_exact_on_lattice(ctx):
    s = wsb.lattice_generate(8, seed=21, aniso_log10=2.0)
    n = s["n"]
    rng = np.random.default_rng(2)
    x = rng.standard_normal(n).astype(np.float32)
    ex = wsb.SpmvExecutor.create(ctx, n, s["row_ptr"], s["col_idx"], s["values"])
    yb = ctx.create_storage_buffer_uninit(n)
    ex.spmv(ctx.create_storage_buffer(x), yb)
    ref = oracle.spmv(s["row_ptr"], s["col_idx"], s["values"], x)
    assert np.array_equal(ctx.readback(yb).view(np.uint32), ref.view(np.uint32))
    lu = wsb.build_lu_blocks_from_csr_block_starts_6(n, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
    bj = wsb.BlockJacobiExecutor.create(ctx, n, lu, s["block_starts"])
    zb = ctx.create_storage_buffer_uninit(n)
    bj.encode_apply(ctx.create_storage_buffer(x), zb)
    zr = oracle.block_jacobi_apply(n, lu, s["block_starts"], x)
    assert np.array_equal(ctx.readback(zb).view(np.uint32), zr.view(np.uint32))


def test_product_spmv_bit_exact_csr_and_bsr(ctx):
    import torch

    s = wsb.lattice_generate(12, seed=8, aniso_log10=1.0)
    n = s["n"]
    x = np.random.default_rng(4).standard_normal(n).astype(np.float32)
    ref = oracle.spmv(s["row_ptr"], s["col_idx"], s["values"], x)
    dx = torch.from_numpy(x).cuda()
    for layout in (wsb.LAYOUT_CSR, wsb.LAYOUT_BSR6):
        m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], layout=layout)
        dy = torch.full((n,), float("nan"), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        # Two launches in a row on the matrix's own descriptor, then the
        # error check that waits for them.
        for _ in range(2):
            m.spmv_device(dx.data_ptr(), dy.data_ptr())
        m.spmv_check()
        ctx.synchronize()
        assert np.array_equal(dy.cpu().numpy().view(np.uint32), ref.view(np.uint32)), layout


def test_adapter_info_and_describe(ctx):
    info = ctx.adapter_info
    assert info["backend"] == "Cuda" and info["cc"][0] >= 10 and info["sm_count"] > 0
    assert "backend=Cuda" in ctx.describe()

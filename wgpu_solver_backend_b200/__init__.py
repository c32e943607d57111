"""B200-native block-Jacobi PCG: Python host mirror of the C ABI (libwsb.so).

The names follow the Rust crate ``wgpu_solver_backend`` so that code and tests
written against it read the same way:

    GpuContext.create(backend)                  gpu/context.rs:60-109
    SpmvExecutor.create(ctx, n, rp, ci, v)      compute/spmv_exec.rs:38-118
    DotScalarExecutor.create(ctx, n_max, len)   compute/dot_scalar_exec.rs:42-123
    VecOpsExecutor.create(ctx)                  compute/vec_ops_exec.rs:40-79
    BlockJacobiExecutor.create(ctx, n, lu, bs)  compute/block_jacobi_exec.rs:48-91
    PcgUpdateScalarsExecutor.create(ctx)        compute/pcg_update_scalars_exec.rs:34-58
    build_lu_blocks_from_csr_block_starts_6     compute.rs:84-181
    lu_factor_inplace_6                         compute.rs:37-71
    pcg_block_jacobi_csr_wgpu                   compute.rs:189-495

Errors the reference returns as ``Err(String)`` raise :class:`WsbError` with the
same message. Everything numeric runs in libwsb.so on the GPU; this module only
moves arguments across the C ABI.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (ALG_CLASSIC, ALG_SINGLE_REDUCTION, LAYOUT_AUTO, LAYOUT_BSR6, LAYOUT_CSR, PREC_F32_F64DOT,
                   PREC_MIXED_F64_IR, PREC_REFERENCE_F32, MatrixInfo, ServerOpts, ServerStats, SolveOpts, SolveResult)

__all__ = ["WsbError", "GpuBackend", "GpuContext", "GpuBuffer", "SpmvExecutor", "DotScalarExecutor",
           "VecOpsExecutor", "BlockJacobiExecutor", "PcgUpdateScalarsExecutor", "lu_factor_inplace_6",
           "build_lu_blocks_from_csr_block_starts_6", "pcg_block_jacobi_csr_wgpu", "Matrix", "Batch", "Server",
           "lattice_sizes", "lattice_generate", "PREC_F32_F64DOT", "PREC_REFERENCE_F32", "PREC_MIXED_F64_IR",
           "LAYOUT_AUTO", "LAYOUT_CSR", "LAYOUT_BSR6", "ALG_CLASSIC", "ALG_SINGLE_REDUCTION"]


class WsbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status
        self.status_name = _lib.STATUS_NAMES.get(status, str(status))


def _lib_handle():
    return _lib.load()


def _check(rc: int, ctx=None):
    if rc != 0:
        msg = _lib_handle().wsb_last_error(ctx).decode(errors="replace")
        raise WsbError(rc, msg)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _p(a, t):
    return a.ctypes.data_as(t)


class GpuBackend:
    """GpuBackend (gpu/context.rs:22-28). Only CUDA exists here; the reference's
    choices are accepted for compatibility and all select the CUDA device."""
    AUTO, VULKAN, DX12, METAL, CUDA = "auto", "vulkan", "dx12", "metal", "cuda"


class GpuBuffer:
    """GpuBuffer<T> (gpu/buffer.rs:6-17): a device allocation with a length."""

    def __init__(self, ctx: "GpuContext", handle, length: int, dtype):
        self.ctx, self.handle, self.len, self.dtype = ctx, handle, int(length), np.dtype(dtype)

    @property
    def nbytes(self):
        return self.len * self.dtype.itemsize

    @property
    def device_ptr(self) -> int:
        return _lib_handle().wsb_buffer_device_ptr(self.handle)

    def __del__(self):
        if getattr(self, "handle", None):
            _lib_handle().wsb_buffer_destroy(self.handle)
            self.handle = None


class GpuContext:
    """GpuContext (gpu/context.rs:40-178) on one CUDA device."""

    def __init__(self, handle):
        self.handle = handle

    @staticmethod
    def create(backend: str = GpuBackend.AUTO, device: int = 0) -> "GpuContext":
        h = C.c_void_p()
        _check(_lib_handle().wsb_context_create(int(device), C.byref(h)))
        return GpuContext(h)

    def describe(self) -> str:
        buf = C.create_string_buffer(512)
        _check(_lib_handle().wsb_context_describe(self.handle, buf, 512), self.handle)
        return buf.value.decode()

    @property
    def adapter_info(self) -> dict:
        ai = _lib.AdapterInfo()
        _check(_lib_handle().wsb_context_adapter_info(self.handle, C.byref(ai)), self.handle)
        return dict(name=ai.name.decode(), backend=ai.backend.decode(), device_type=ai.device_type.decode(),
                    vendor=ai.vendor, device=ai.device, sm_count=ai.sm_count, cc=(ai.cc_major, ai.cc_minor),
                    total_mem_bytes=ai.total_mem_bytes)

    def last_error(self) -> str:
        return _lib_handle().wsb_last_error(self.handle).decode(errors="replace")

    def set_stream(self, cuda_stream_ptr: int | None):
        _check(_lib_handle().wsb_context_set_stream(self.handle, C.c_void_p(cuda_stream_ptr or 0)), self.handle)

    def set_wait_limit(self, cycles: int = 0):
        """Limit of every pipeline wait in the solver kernels, in SM clock
        cycles (0: the default of about 2 s). A wait that runs out ends the
        solves in flight with status TIMEOUT."""
        _check(_lib_handle().wsb_context_set_wait_limit(self.handle, int(cycles)), self.handle)

    def synchronize(self):
        _check(_lib_handle().wsb_context_synchronize(self.handle), self.handle)

    def create_storage_buffer(self, data) -> GpuBuffer:
        arr = np.ascontiguousarray(data)
        h = C.c_void_p()
        _check(_lib_handle().wsb_buffer_create(self.handle, arr.ctypes.data_as(C.c_void_p), arr.nbytes, C.byref(h)),
               self.handle)
        return GpuBuffer(self, h, arr.size, arr.dtype)

    def create_storage_buffer_uninit(self, length: int, dtype=np.float32) -> GpuBuffer:
        h = C.c_void_p()
        _check(_lib_handle().wsb_buffer_create(self.handle, None, int(length) * np.dtype(dtype).itemsize, C.byref(h)),
               self.handle)
        return GpuBuffer(self, h, length, dtype)

    def readback(self, buf: GpuBuffer) -> np.ndarray:
        out = np.empty(buf.len, buf.dtype)
        _check(_lib_handle().wsb_buffer_read(self.handle, buf.handle, 0, out.ctypes.data_as(C.c_void_p), out.nbytes),
               self.handle)
        return out

    def write(self, buf: GpuBuffer, data, offset_bytes: int = 0):
        arr = np.ascontiguousarray(data)
        _check(_lib_handle().wsb_buffer_write(self.handle, buf.handle, offset_bytes, arr.ctypes.data_as(C.c_void_p),
                                              arr.nbytes), self.handle)

    def __del__(self):
        if getattr(self, "handle", None):
            _lib_handle().wsb_context_destroy(self.handle)
            self.handle = None


class SpmvExecutor:
    """SpmvExecutor (compute/spmv_exec.rs:17-147); CSR resident on the device."""

    def __init__(self, ctx, handle, n_rows):
        self.ctx, self.handle, self.n_rows = ctx, handle, n_rows

    @staticmethod
    def create(ctx: GpuContext, n_rows, row_ptr, col_idx, values) -> "SpmvExecutor":
        rp, ci, v = _u32(row_ptr), _u32(col_idx), _f32(values)
        h = C.c_void_p()
        _check(_lib_handle().wsb_spmv_executor_create(ctx.handle, int(n_rows), _p(rp, _lib.u32p), _p(ci, _lib.u32p),
                                                      _p(v, _lib.f32p), len(v), C.byref(h)), ctx.handle)
        return SpmvExecutor(ctx, h, int(n_rows))

    def spmv(self, x: GpuBuffer, y: GpuBuffer):
        """encode_copy_x_from + encode_spmv (spmv_exec.rs:122-147): y = A x."""
        _check(_lib_handle().wsb_spmv_executor_spmv(self.handle, x.handle, y.handle), self.ctx.handle)

    def __del__(self):
        if getattr(self, "handle", None):
            _lib_handle().wsb_spmv_executor_destroy(self.handle)
            self.handle = None


class DotScalarExecutor:
    """DotScalarExecutor (compute/dot_scalar_exec.rs:16-271) with its scalar mailbox."""

    def __init__(self, ctx, handle, length):
        self.ctx, self.handle, self.scalar_results_len = ctx, handle, length

    @staticmethod
    def create(ctx: GpuContext, n_max: int, scalar_results_len: int) -> "DotScalarExecutor":
        h = C.c_void_p()
        _check(_lib_handle().wsb_dot_scalar_executor_create(ctx.handle, int(n_max), int(scalar_results_len),
                                                            C.byref(h)), ctx.handle)
        return DotScalarExecutor(ctx, h, int(scalar_results_len))

    def encode_dot_scalar_into(self, a: GpuBuffer, b: GpuBuffer, n: int, out_index: int):
        _check(_lib_handle().wsb_dot_scalar_executor_dot_into(self.handle, a.handle, b.handle, int(n), int(out_index)),
               self.ctx.handle)

    def scalar_results_buffer(self) -> GpuBuffer:
        h = _lib_handle().wsb_dot_scalar_executor_scalar_results(self.handle)
        return _BorrowedBuffer(self.ctx, C.c_void_p(h), self.scalar_results_len)

    def readback_scalar_results(self) -> np.ndarray:
        out = np.zeros(self.scalar_results_len, np.float32)
        _check(_lib_handle().wsb_dot_scalar_executor_readback(self.handle, _p(out, _lib.f32p), len(out)),
               self.ctx.handle)
        return out

    def __del__(self):
        if getattr(self, "handle", None):
            _lib_handle().wsb_dot_scalar_executor_destroy(self.handle)
            self.handle = None


class _BorrowedBuffer(GpuBuffer):
    """A buffer owned by an executor (not freed from Python)."""

    def __init__(self, ctx, handle, length):
        super().__init__(ctx, handle, length, np.float32)

    def __del__(self):
        self.handle = None


class VecOpsExecutor:
    """VecOpsExecutor (compute/vec_ops_exec.rs:23-239)."""

    def __init__(self, ctx):
        self.ctx = ctx

    @staticmethod
    def create(ctx: GpuContext) -> "VecOpsExecutor":
        return VecOpsExecutor(ctx)

    def encode_axpy_inplace(self, x: GpuBuffer, y: GpuBuffer, n: int, alpha: float):
        _check(_lib_handle().wsb_vec_axpy_inplace(self.ctx.handle, x.handle, y.handle, int(n), float(alpha)),
               self.ctx.handle)

    def encode_axpy_inplace_from_scalar_results(self, x, y, n, scalar_results, scalar_index):
        _check(_lib_handle().wsb_vec_axpy_inplace_from_scalar_results(self.ctx.handle, x.handle, y.handle, int(n),
                                                                      scalar_results.handle, int(scalar_index)),
               self.ctx.handle)

    def encode_scale_inplace_from_scalar_results(self, x, n, scalar_results, scalar_index):
        _check(_lib_handle().wsb_vec_scale_inplace_from_scalar_results(self.ctx.handle, x.handle, int(n),
                                                                       scalar_results.handle, int(scalar_index)),
               self.ctx.handle)


class BlockJacobiExecutor:
    """BlockJacobiExecutor (compute/block_jacobi_exec.rs:25-133)."""

    def __init__(self, ctx, handle, n):
        self.ctx, self.handle, self.n = ctx, handle, n

    @staticmethod
    def create(ctx: GpuContext, n: int, lu_blocks, block_starts) -> "BlockJacobiExecutor":
        lu, bs = _f32(lu_blocks), _u32(block_starts)
        h = C.c_void_p()
        _check(_lib_handle().wsb_block_jacobi_executor_create(ctx.handle, int(n), _p(lu, _lib.f32p), len(lu),
                                                              _p(bs, _lib.u32p), len(bs), C.byref(h)), ctx.handle)
        return BlockJacobiExecutor(ctx, h, int(n))

    def encode_apply(self, r: GpuBuffer, z: GpuBuffer):
        _check(_lib_handle().wsb_block_jacobi_executor_apply(self.handle, r.handle, z.handle), self.ctx.handle)

    def __del__(self):
        if getattr(self, "handle", None):
            _lib_handle().wsb_block_jacobi_executor_destroy(self.handle)
            self.handle = None


class PcgUpdateScalarsExecutor:
    """PcgUpdateScalarsExecutor (compute/pcg_update_scalars_exec.rs:26-119)."""

    def __init__(self, ctx):
        self.ctx = ctx

    @staticmethod
    def create(ctx: GpuContext) -> "PcgUpdateScalarsExecutor":
        return PcgUpdateScalarsExecutor(ctx)

    def encode_update_scalars(self, scalar_results: GpuBuffer, p_ap, rz_new, rz_old, alpha, minus_alpha, beta):
        _check(_lib_handle().wsb_pcg_update_scalars(self.ctx.handle, scalar_results.handle, p_ap, rz_new, rz_old,
                                                    alpha, minus_alpha, beta), self.ctx.handle)


def lu_factor_inplace_6(mat: np.ndarray, n: int) -> None:
    """compute.rs:37-71 (host). mat: float32 array of >= 36 entries, modified in place."""
    if mat.dtype != np.float32 or not mat.flags.c_contiguous:
        raise TypeError("mat must be a contiguous float32 array")
    _check(_lib_handle().wsb_lu_factor_inplace_6(_p(mat, _lib.f32p), mat.size, int(n)))


def build_lu_blocks_from_csr_block_starts_6(n, row_ptr, col_idx, values, block_starts) -> np.ndarray:
    """compute.rs:84-181 (host): 36 floats per block, row-major packed LU."""
    rp, ci, v, bs = _u32(row_ptr), _u32(col_idx), _f32(values), _u32(block_starts)
    nb = max(len(bs) - 1, 0)
    out = np.zeros(max(nb, 1) * 36, np.float32)
    _check(_lib_handle().wsb_build_lu_blocks_from_csr_block_starts_6(
        int(n), _p(rp, _lib.u32p), len(rp), _p(ci, _lib.u32p), len(ci), _p(v, _lib.f32p), len(v), _p(bs, _lib.u32p),
        len(bs), _p(out, _lib.f32p)))
    return out[: nb * 36]


def _opts(precision, history_capacity, always_write_x, target_relres=None, inner_rel_tol=None, max_refine=None,
          x64_out=None, algorithm=None):
    o = SolveOpts()
    _lib_handle().wsb_solve_opts_default(C.byref(o))
    o.precision = precision
    if algorithm is not None:
        o.algorithm = int(algorithm)
    hist = None
    if history_capacity:
        hist = np.zeros(int(history_capacity), np.float64)
        o.history_capacity = int(history_capacity)
        o.history_out = _p(hist, _lib.f64p)
    o.always_write_x = 1 if always_write_x else 0
    if target_relres is not None:
        o.target_relres = target_relres
    if inner_rel_tol is not None:
        o.inner_rel_tol = inner_rel_tol
    if max_refine is not None:
        o.max_refine = max_refine
    if x64_out is not None:
        if not (x64_out.dtype == np.float64 and x64_out.flags.c_contiguous):
            raise TypeError("x64_out must be a contiguous float64 array")
        o.x64_out = _p(x64_out, _lib.f64p)
    return o, hist


def _result_dict(r: SolveResult, hist=None):
    d = {k: getattr(r, k) for k, _ in SolveResult._fields_ if k != "reserved"}
    if hist is not None:
        d["history"] = hist[: r.history_len].copy()
    return d


def pcg_block_jacobi_csr_wgpu(n, b, x, max_iter, rel_tol, abs_tol, ctx, spmv_exec, vec_ops_exec, dot_scalar_exec,
                              block_jacobi_exec, pcg_update_scalars_exec, precision=PREC_F32_F64DOT,
                              history_capacity=0, always_write_x=False, result=None) -> int:
    """compute.rs:189-495. x (float32 numpy array) holds x0 and receives the
    solution on success. Returns the iteration count; raises WsbError on the
    reference's Err cases. The vec/dot/scalar executors are accepted for
    signature parity; their passes are fused into the solver kernels."""
    b, xa = _f32(b), x
    if not (isinstance(xa, np.ndarray) and xa.dtype == np.float32 and xa.flags.c_contiguous):
        raise TypeError("x must be a contiguous float32 numpy array (it is updated in place)")
    o, hist = _opts(precision, history_capacity, always_write_x)
    it = C.c_uint64(0)
    res = SolveResult()
    rc = _lib_handle().wsb_pcg_block_jacobi_csr(ctx.handle, int(n), _p(b, _lib.f32p), len(b), _p(xa, _lib.f32p),
                                                len(xa), int(max_iter), float(rel_tol), float(abs_tol),
                                                spmv_exec.handle, block_jacobi_exec.handle, C.byref(o), C.byref(it),
                                                C.byref(res))
    if result is not None:
        result.update(_result_dict(res, hist))
    _check(rc, ctx.handle)
    return it.value


class Matrix:
    """A system matrix resident on the device (CSR or BSR6) with its LU factors."""

    def __init__(self, ctx, handle):
        self.ctx, self.handle = ctx, handle
        mi = MatrixInfo()
        _check(_lib_handle().wsb_matrix_info_get(handle, C.byref(mi)), ctx.handle)
        self.info = {k: getattr(mi, k) for k, _ in MatrixInfo._fields_ if k != "reserved"}
        self.n = mi.n

    @staticmethod
    def create(ctx: GpuContext, row_ptr, col_idx, values, block_starts, layout=LAYOUT_AUTO) -> "Matrix":
        rp, ci, v, bs = _u32(row_ptr), _u32(col_idx), _f32(values), _u32(block_starts)
        h = C.c_void_p()
        _check(_lib_handle().wsb_matrix_create(ctx.handle, len(rp) - 1, _p(rp, _lib.u32p), _p(ci, _lib.u32p),
                                               _p(v, _lib.f32p), len(v), _p(bs, _lib.u32p), len(bs), int(layout),
                                               C.byref(h)), ctx.handle)
        return Matrix(ctx, h)

    def autotune(self, iterations: int = 8) -> dict:
        """Times candidate tile sizes of the SpMV and update kernels on this
        matrix, keeps the fastest and records them for matrices of the same
        shape class created later (wsb_matrix_autotune)."""
        r = _lib.TuneResult()
        _check(_lib_handle().wsb_matrix_autotune(self.ctx.handle, self.handle, int(iterations), C.byref(r)),
               self.ctx.handle)
        return {k: getattr(r, k) for k, _ in _lib.TuneResult._fields_ if k != "reserved"}

    def lu(self) -> np.ndarray:
        """The block-Jacobi factors held on the device (num_blocks * 36
        floats, the layout of build_lu_blocks_from_csr_block_starts_6)."""
        out = np.zeros(max(1, int(self.info["num_blocks"]) * 36), np.float32)
        _check(_lib_handle().wsb_matrix_read_lu(self.ctx.handle, self.handle, _p(out, _lib.f32p), out.size),
               self.ctx.handle)
        return out[: int(self.info["num_blocks"]) * 36]

    def solve(self, b, x0=None, max_iter=2000, rel_tol=1e-8, abs_tol=0.0, precision=PREC_F32_F64DOT,
              history_capacity=0, always_write_x=False, raise_on_error=True, **mixed):
        """Returns (x, result dict). x keeps x0 unless the solve succeeded (or
        always_write_x)."""
        b = _f32(b)
        x = np.zeros(self.n, np.float32) if x0 is None else _f32(x0).copy()
        o, hist = _opts(precision, history_capacity, always_write_x, **mixed)
        res = SolveResult()
        rc = _lib_handle().wsb_solve(self.ctx.handle, self.handle, _p(b, _lib.f32p), _p(x, _lib.f32p), int(max_iter),
                                     float(rel_tol), float(abs_tol), C.byref(o), C.byref(res))
        out = _result_dict(res, hist)
        out["rc"] = rc
        if raise_on_error:
            _check(rc, self.ctx.handle)
        return x, out

    def solve_device(self, d_b: int, d_x: int, max_iter=2000, rel_tol=1e-8, abs_tol=0.0,
                     precision=PREC_F32_F64DOT, raise_on_error=True, **mixed):
        o, _ = _opts(precision, 0, False, **mixed)
        res = SolveResult()
        rc = _lib_handle().wsb_solve_device(self.ctx.handle, self.handle, C.c_void_p(d_b), C.c_void_p(d_x),
                                            int(max_iter), float(rel_tol), float(abs_tol), C.byref(o), C.byref(res))
        out = _result_dict(res)
        out["rc"] = rc
        if raise_on_error:
            _check(rc, self.ctx.handle)
        return out

    def kernel_times(self, d_b: int, iterations: int = 20) -> dict:
        """Mean per-launch device time (ms) of the three loop kernels."""
        ms = np.zeros(5, np.float64)
        _check(_lib_handle().wsb_matrix_kernel_times(self.ctx.handle, self.handle, C.c_void_p(d_b), int(iterations),
                                                     _p(ms, _lib.f64p)), self.ctx.handle)
        if int(ms[3]) != int(iterations) or int(ms[4]) != 0:
            raise WsbError(_lib.CUDA, f"kernel timing invalid: system stopped after {int(ms[3])} of {iterations} "
                                      f"iterations (status {int(ms[4])})")
        return dict(spmv_ms=ms[0], update_ms=ms[1], pupdate_ms=ms[2])

    def spmv_device(self, d_x: int, d_y: int):
        """y = A x on the context's stream (not waited for)."""
        _check(_lib_handle().wsb_matrix_spmv_device(self.ctx.handle, self.handle, C.c_void_p(d_x), C.c_void_p(d_y)),
               self.ctx.handle)

    def spmv_check(self):
        """Waits for the last spmv_device launch; raises on a kernel error."""
        _check(_lib_handle().wsb_matrix_spmv_check(self.ctx.handle, self.handle), self.ctx.handle)

    def __del__(self):
        if getattr(self, "handle", None):
            _lib_handle().wsb_matrix_destroy(self.handle)
            self.handle = None


class Batch:
    """Many independent systems solved together (wsb_batch_*)."""

    def __init__(self, ctx: GpuContext):
        self.ctx = ctx
        h = C.c_void_p()
        _check(_lib_handle().wsb_batch_create(ctx.handle, C.byref(h)), ctx.handle)
        self.handle = h
        self._keep = []

    def add(self, matrix: Matrix, b, x0=None, max_iter=2000, rel_tol=1e-8, abs_tol=0.0,
            precision=PREC_F32_F64DOT, history_capacity=0, **mixed) -> int:
        b = _f32(b)
        x0 = np.zeros(matrix.n, np.float32) if x0 is None else _f32(x0)
        o, hist = _opts(precision, history_capacity, False, **mixed)
        bid = C.c_uint32(0)
        _check(_lib_handle().wsb_batch_add(self.handle, matrix.handle, _p(b, _lib.f32p), _p(x0, _lib.f32p),
                                           int(max_iter), float(rel_tol), float(abs_tol), C.byref(o), C.byref(bid)),
               self.ctx.handle)
        self._keep.append((matrix, o, hist))
        return bid.value

    def solve(self):
        _check(_lib_handle().wsb_batch_solve(self.handle), self.ctx.handle)

    def result(self, bid: int, n: int):
        x = np.zeros(n, np.float32)
        res = SolveResult()
        rc = _lib_handle().wsb_batch_result(self.handle, int(bid), _p(x, _lib.f32p), C.byref(res))
        out = _result_dict(res, self._keep[bid][2])
        out["rc"] = rc
        return x, out

    def __del__(self):
        if getattr(self, "handle", None):
            _lib_handle().wsb_batch_destroy(self.handle)
            self.handle = None


class Server:
    """Continuous-batching solve server (wsb_server_*)."""

    def __init__(self, ctx: GpuContext, memory_budget_bytes=0, max_active=0, iters_per_step=0, borrow_inputs=False,
                 device_prep=False):
        """borrow_inputs: requests read the submitted arrays in place (this
        object keeps them alive until the request is done) instead of copying
        them at submit. device_prep: each request's column check, BSR6
        conversion and LU run on the GPU instead of the host."""
        self.ctx = ctx
        so = ServerOpts()
        so.struct_size = C.sizeof(ServerOpts)
        so.memory_budget_bytes = int(memory_budget_bytes)
        so.max_active = int(max_active)
        so.iters_per_step = int(iters_per_step)
        so.flags = (_lib.SERVER_BORROW_INPUTS if borrow_inputs else 0) | (_lib.SERVER_DEVICE_PREP if device_prep else 0)
        h = C.c_void_p()
        _check(_lib_handle().wsb_server_create(ctx.handle, C.byref(so), C.byref(h)), ctx.handle)
        self.handle = h
        self._n = {}
        self._borrowed = {}  # request id -> arrays the server reads in place

    def submit(self, row_ptr, col_idx, values, block_starts, b, x0=None, max_iter=2000, rel_tol=1e-8, abs_tol=0.0,
               precision=PREC_F32_F64DOT, **mixed) -> int:
        rp, ci, v, bs, b = _u32(row_ptr), _u32(col_idx), _f32(values), _u32(block_starts), _f32(b)
        n = len(rp) - 1
        x0 = np.zeros(n, np.float32) if x0 is None else _f32(x0)
        o, _ = _opts(precision, 0, False, **mixed)
        rid = C.c_uint64(0)
        _check(_lib_handle().wsb_server_submit(self.handle, n, _p(rp, _lib.u32p), _p(ci, _lib.u32p), _p(v, _lib.f32p),
                                               len(v), _p(bs, _lib.u32p), len(bs), _p(b, _lib.f32p),
                                               _p(x0, _lib.f32p), int(max_iter), float(rel_tol), float(abs_tol),
                                               C.byref(o), C.byref(rid)), self.ctx.handle)
        self._n[rid.value] = n
        self._borrowed[rid.value] = (rp, ci, v, bs, b, x0)
        return rid.value

    def poll(self, rid: int):
        x = np.zeros(self._n[rid], np.float32)
        res = SolveResult()
        rc = _lib_handle().wsb_server_poll(self.handle, int(rid), _p(x, _lib.f32p), C.byref(res))
        if rc == _lib.PENDING:
            return None
        self._n.pop(rid, None)
        self._borrowed.pop(rid, None)
        out = _result_dict(res)
        out["rc"] = rc
        return x, out

    def wait(self, rid: int, timeout_s: float = 600.0):
        x = np.zeros(self._n[rid], np.float32)
        res = SolveResult()
        rc = _lib_handle().wsb_server_wait(self.handle, int(rid), _p(x, _lib.f32p), C.byref(res), float(timeout_s))
        if rc == _lib.TIMEOUT:
            raise WsbError(rc, _lib_handle().wsb_last_error(self.ctx.handle).decode())
        self._n.pop(rid, None)
        self._borrowed.pop(rid, None)
        out = _result_dict(res)
        out["rc"] = rc
        return x, out

    def stats(self) -> dict:
        st = ServerStats()
        _check(_lib_handle().wsb_server_stats_get(self.handle, C.byref(st)), self.ctx.handle)
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "handle", None):
            _lib_handle().wsb_server_destroy(self.handle)
            self.handle = None
        self._borrowed = {}

    def __del__(self):
        self.close()


def lattice_sizes(side: int) -> dict:
    s = _lib.LatticeSizes()
    _check(_lib_handle().wsb_lattice_sizes_get(int(side), C.byref(s)))
    return {k: getattr(s, k) for k, _ in _lib.LatticeSizes._fields_}


def autotune_clear() -> None:
    """Forgets the tile sizes the autotuner recorded per shape class."""
    _lib_handle().wsb_autotune_clear()


def lattice_generate(side: int, seed: int = 0, aniso_log10: float = 0.0) -> dict:
    """Synthetic 6-DOF lattice system: row_ptr, col_idx, values, block_starts, b."""
    sz = lattice_sizes(side)
    rp = np.empty(sz["n"] + 1, np.uint32)
    ci = np.empty(sz["nnz"], np.uint32)
    v = np.empty(sz["nnz"], np.float32)
    bs = np.empty(sz["nodes"] + 1, np.uint32)
    b = np.empty(sz["n"], np.float32)
    _check(_lib_handle().wsb_lattice_generate(int(side), int(seed), float(aniso_log10), _p(rp, _lib.u32p),
                                              _p(ci, _lib.u32p), _p(v, _lib.f32p), _p(bs, _lib.u32p),
                                              _p(b, _lib.f32p)))
    return dict(row_ptr=rp, col_idx=ci, values=v, block_starts=bs, b=b, n=int(sz["n"]), nnz=int(sz["nnz"]))

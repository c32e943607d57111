"""ctypes declarations for libwsb.so (the C ABI in include/wsb.h)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwsb.so")

u32p = C.POINTER(C.c_uint32)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
u64p = C.POINTER(C.c_uint64)
vp = C.c_void_p

# Status codes (wsb_status)
OK, BAD_INPUT, ZERO_PIVOT, BREAKDOWN, NOT_CONVERGED, CUDA, OUT_OF_MEMORY, TIMEOUT, NO_DEVICE, UNSUPPORTED, PENDING = range(11)
STATUS_NAMES = {0: "OK", 1: "BAD_INPUT", 2: "ZERO_PIVOT", 3: "BREAKDOWN", 4: "NOT_CONVERGED", 5: "CUDA",
                6: "OUT_OF_MEMORY", 7: "TIMEOUT", 8: "NO_DEVICE", 9: "UNSUPPORTED", 10: "PENDING"}

PREC_F32_F64DOT, PREC_REFERENCE_F32, PREC_MIXED_F64_IR = 0, 1, 2
ALG_CLASSIC, ALG_SINGLE_REDUCTION = 0, 1
LAYOUT_AUTO, LAYOUT_CSR, LAYOUT_BSR6 = 0, 1, 2


class AdapterInfo(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("backend", C.c_char * 16), ("device_type", C.c_char * 32),
                ("vendor", C.c_uint32), ("device", C.c_uint32), ("sm_count", C.c_uint32), ("cc_major", C.c_int),
                ("cc_minor", C.c_int), ("total_mem_bytes", C.c_uint64)]


class SolveOpts(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("precision", C.c_int32), ("target_relres", C.c_double),
                ("inner_rel_tol", C.c_float), ("max_refine", C.c_uint32), ("history_capacity", C.c_uint64),
                ("history_out", f64p), ("always_write_x", C.c_int32), ("algorithm", C.c_int32), ("x64_out", f64p)]


class SolveResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("breakdown_kind", C.c_int32), ("iterations", C.c_uint64),
                ("refine_sweeps", C.c_uint32), ("reserved", C.c_uint32), ("b_norm2", C.c_double),
                ("final_r_norm2", C.c_double), ("final_relres", C.c_double), ("device_ms", C.c_double),
                ("total_ms", C.c_double), ("history_len", C.c_uint64), ("kernel_launches", C.c_uint64)]


class MatrixInfo(C.Structure):
    _fields_ = [("n", C.c_uint64), ("nnz", C.c_uint64), ("num_blocks", C.c_uint64), ("layout", C.c_int32),
                ("reserved", C.c_int32), ("device_bytes", C.c_uint64), ("spmv_bytes", C.c_uint64),
                ("iteration_bytes", C.c_uint64)]


class TuneResult(C.Structure):
    _fields_ = [("spmv_rows", C.c_uint32), ("spmv_cap", C.c_uint32), ("update_rows", C.c_uint32),
                ("update_blocks", C.c_uint32), ("spmv_ms", C.c_double), ("update_ms", C.c_double),
                ("default_spmv_ms", C.c_double), ("default_update_ms", C.c_double), ("candidates", C.c_uint32),
                ("reserved", C.c_uint32)]


SERVER_BORROW_INPUTS, SERVER_DEVICE_PREP = 1, 2


class ServerOpts(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("max_active", C.c_uint32), ("memory_budget_bytes", C.c_uint64),
                ("iters_per_step", C.c_uint32), ("flags", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("rejected", C.c_uint64), ("active", C.c_uint64), ("pending", C.c_uint64), ("steps", C.c_uint64),
                ("device_bytes_in_use", C.c_uint64), ("device_bytes_peak", C.c_uint64), ("busy_ms", C.c_double),
                ("kernel_launches", C.c_uint64), ("host_prep_ms", C.c_double), ("upload_ms", C.c_double),
                ("admit_ms", C.c_double), ("retire_ms", C.c_double), ("sched_idle_ms", C.c_double)]


class LatticeSizes(C.Structure):
    _fields_ = [("nodes", C.c_uint64), ("edges", C.c_uint64), ("n", C.c_uint64), ("nnz", C.c_uint64),
                ("num_blocks", C.c_uint64), ("bsr_blocks", C.c_uint64)]


# name -> (restype, argtypes)
SIGNATURES = {
    "wsb_context_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
    "wsb_context_destroy": (None, [vp]),
    "wsb_last_error": (C.c_char_p, [vp]),
    "wsb_context_describe": (C.c_int, [vp, C.c_char_p, C.c_size_t]),
    "wsb_context_adapter_info": (C.c_int, [vp, C.POINTER(AdapterInfo)]),
    "wsb_context_set_stream": (C.c_int, [vp, vp]),
    "wsb_context_synchronize": (C.c_int, [vp]),
    "wsb_buffer_create": (C.c_int, [vp, vp, C.c_size_t, C.POINTER(vp)]),
    "wsb_buffer_write": (C.c_int, [vp, vp, C.c_size_t, vp, C.c_size_t]),
    "wsb_buffer_read": (C.c_int, [vp, vp, C.c_size_t, vp, C.c_size_t]),
    "wsb_buffer_size": (C.c_size_t, [vp]),
    "wsb_buffer_device_ptr": (vp, [vp]),
    "wsb_buffer_destroy": (None, [vp]),
    "wsb_spmv_executor_create": (C.c_int, [vp, C.c_uint32, u32p, u32p, f32p, C.c_uint64, C.POINTER(vp)]),
    "wsb_spmv_executor_spmv": (C.c_int, [vp, vp, vp]),
    "wsb_spmv_executor_destroy": (None, [vp]),
    "wsb_dot_scalar_executor_create": (C.c_int, [vp, C.c_uint64, C.c_uint32, C.POINTER(vp)]),
    "wsb_dot_scalar_executor_dot_into": (C.c_int, [vp, vp, vp, C.c_uint32, C.c_uint32]),
    "wsb_dot_scalar_executor_scalar_results": (vp, [vp]),
    "wsb_dot_scalar_executor_readback": (C.c_int, [vp, f32p, C.c_uint32]),
    "wsb_dot_scalar_executor_destroy": (None, [vp]),
    "wsb_vec_axpy_inplace": (C.c_int, [vp, vp, vp, C.c_uint32, C.c_float]),
    "wsb_vec_axpy_inplace_from_scalar_results": (C.c_int, [vp, vp, vp, C.c_uint32, vp, C.c_uint32]),
    "wsb_vec_scale_inplace_from_scalar_results": (C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint32]),
    "wsb_block_jacobi_executor_create": (C.c_int, [vp, C.c_uint32, f32p, C.c_uint64, u32p, C.c_uint64, C.POINTER(vp)]),
    "wsb_block_jacobi_executor_apply": (C.c_int, [vp, vp, vp]),
    "wsb_block_jacobi_executor_destroy": (None, [vp]),
    "wsb_pcg_update_scalars": (C.c_int, [vp, vp] + [C.c_uint32] * 6),
    "wsb_dot_tree256_noalloc": (C.c_int, [vp, vp, vp, C.c_uint32, vp]),
    "wsb_lu_factor_inplace_6": (C.c_int, [f32p, C.c_uint64, C.c_uint32]),
    "wsb_build_lu_blocks_from_csr_block_starts_6": (C.c_int, [C.c_uint32, u32p, C.c_uint64, u32p, C.c_uint64, f32p,
                                                              C.c_uint64, u32p, C.c_uint64, f32p]),
    "wsb_solve_opts_default": (None, [C.POINTER(SolveOpts)]),
    "wsb_pcg_block_jacobi_csr": (C.c_int, [vp, C.c_uint64, f32p, C.c_uint64, f32p, C.c_uint64, C.c_uint64, C.c_float,
                                           C.c_float, vp, vp, C.POINTER(SolveOpts), u64p, C.POINTER(SolveResult)]),
    "wsb_matrix_create": (C.c_int, [vp, C.c_uint32, u32p, u32p, f32p, C.c_uint64, u32p, C.c_uint64, C.c_int32,
                                    C.POINTER(vp)]),
    "wsb_matrix_info_get": (C.c_int, [vp, C.POINTER(MatrixInfo)]),
    "wsb_matrix_destroy": (None, [vp]),
    "wsb_matrix_read_lu": (C.c_int, [vp, vp, f32p, C.c_uint64]),
    "wsb_matrix_autotune": (C.c_int, [vp, vp, C.c_uint32, C.POINTER(TuneResult)]),
    "wsb_autotune_clear": (None, []),
    "wsb_solve": (C.c_int, [vp, vp, f32p, f32p, C.c_uint64, C.c_float, C.c_float, C.POINTER(SolveOpts),
                            C.POINTER(SolveResult)]),
    "wsb_solve_device": (C.c_int, [vp, vp, vp, vp, C.c_uint64, C.c_float, C.c_float, C.POINTER(SolveOpts),
                                   C.POINTER(SolveResult)]),
    "wsb_matrix_spmv_device": (C.c_int, [vp, vp, vp, vp]),
    "wsb_matrix_spmv_check": (C.c_int, [vp, vp]),
    "wsb_context_set_wait_limit": (C.c_int, [vp, C.c_uint64]),
    "wsb_matrix_kernel_times": (C.c_int, [vp, vp, vp, C.c_uint32, f64p]),
    "wsb_batch_create": (C.c_int, [vp, C.POINTER(vp)]),
    "wsb_batch_add": (C.c_int, [vp, vp, f32p, f32p, C.c_uint64, C.c_float, C.c_float, C.POINTER(SolveOpts),
                                C.POINTER(C.c_uint32)]),
    "wsb_batch_solve": (C.c_int, [vp]),
    "wsb_batch_result": (C.c_int, [vp, C.c_uint32, f32p, C.POINTER(SolveResult)]),
    "wsb_batch_destroy": (None, [vp]),
    "wsb_server_create": (C.c_int, [vp, C.POINTER(ServerOpts), C.POINTER(vp)]),
    "wsb_server_submit": (C.c_int, [vp, C.c_uint32, u32p, u32p, f32p, C.c_uint64, u32p, C.c_uint64, f32p, f32p,
                                    C.c_uint64, C.c_float, C.c_float, C.POINTER(SolveOpts), u64p]),
    "wsb_server_poll": (C.c_int, [vp, C.c_uint64, f32p, C.POINTER(SolveResult)]),
    "wsb_server_wait": (C.c_int, [vp, C.c_uint64, f32p, C.POINTER(SolveResult), C.c_double]),
    "wsb_server_stats_get": (C.c_int, [vp, C.POINTER(ServerStats)]),
    "wsb_server_destroy": (None, [vp]),
    "wsb_lattice_sizes_get": (C.c_int, [C.c_uint32, C.POINTER(LatticeSizes)]),
    "wsb_lattice_generate": (C.c_int, [C.c_uint32, C.c_uint64, C.c_double, u32p, u32p, f32p, u32p, f32p]),
}

_lib = None


def load():
    """Load libwsb.so. Raises if the library has not been built: there is no
    fallback implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` "
                               "(or __graft_entry__.build()); there is no CPU fallback")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib

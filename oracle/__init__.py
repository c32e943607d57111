"""ctypes bindings to the CPU oracle (oracle/oracle.c).

Test infrastructure only: the parity tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module as the checker. The product
library never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")

OK, BAD_INPUT, ZERO_PIVOT, BREAKDOWN, MAXITER = 0, 1, 2, 3, 4

_u32p = C.POINTER(C.c_uint32)
_f32p = C.POINTER(C.c_float)
_f64p = C.POINTER(C.c_double)
_u64p = C.POINTER(C.c_uint64)
_i64p = C.POINTER(C.c_int64)
_ip = C.POINTER(C.c_int)


def build(force: bool = False) -> str:
    """Compile oracle.c into liboracle.so (gcc, OpenMP, no FMA contraction)."""
    src = os.path.join(_HERE, "oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_lu_factor_inplace_6.argtypes = [_f32p, C.c_int, _ip]
        L.orc_build_lu_blocks_6.argtypes = [C.c_uint32, _u32p, C.c_uint64, _u32p, C.c_uint64, _f32p,
                                            C.c_uint64, _u32p, C.c_uint64, _f32p, _i64p, _ip]
        L.orc_spmv_csr.argtypes = [C.c_uint32, _u32p, _u32p, _f32p, _f32p, _f32p]
        L.orc_spmv_csr.restype = None
        L.orc_dot_tree256.argtypes = [C.c_uint32, _f32p, _f32p]
        L.orc_dot_tree256.restype = C.c_float
        L.orc_block_jacobi_apply.argtypes = [C.c_uint32, C.c_uint32, _f32p, _u32p, _f32p, _f32p]
        L.orc_block_jacobi_apply.restype = None
        L.orc_axpy.argtypes = [C.c_uint32, C.c_float, _f32p, _f32p]
        L.orc_axpy.restype = None
        L.orc_scale.argtypes = [C.c_uint32, C.c_float, _f32p]
        L.orc_scale.restype = None
        L.orc_update_scalars.argtypes = [_f32p] + [C.c_uint32] * 6
        L.orc_update_scalars.restype = None
        L.orc_pcg_ref_f32.argtypes = [C.c_uint32, _u32p, _u32p, _f32p, C.c_uint32, _f32p, _u32p, _f32p,
                                      _f32p, C.c_uint64, C.c_float, C.c_float, _u64p, _f32p, _ip]
        L.orc_pcg_f64dot.argtypes = [C.c_uint32, _u32p, _u32p, _f32p, C.c_uint32, _f32p, _u32p, _f32p,
                                     _f32p, C.c_uint64, C.c_float, C.c_float, _u64p, _f64p, _ip]
        L.orc_pcg_single_reduction_f64dot.argtypes = [C.c_uint32, _u32p, _u32p, _f32p, C.c_uint32, _f32p, _u32p,
                                                      _f32p, _f32p, C.c_uint64, C.c_float, C.c_float, _u64p, _f64p]
        L.orc_pcg_f64.argtypes = [C.c_uint32, _u32p, _u32p, _f32p, C.c_uint32, _u32p, _f64p, _f64p,
                                  C.c_uint64, C.c_double, _u64p]
        L.orc_true_relres_f64.argtypes = [C.c_uint32, _u32p, _u32p, _f32p, _f32p, _f32p, _f64p]
        L.orc_true_relres_f64.restype = C.c_double
        L.orc_compare_x.argtypes = [C.c_uint64, _f32p, _f32p, _f64p]
        L.orc_compare_x.restype = None
        L.orc_num_threads.restype = C.c_int
        L.orc_lattice_sizes.argtypes = [C.c_uint32, _u64p]
        L.orc_lattice_generate.argtypes = [C.c_uint32, C.c_uint64, C.c_double, _u32p, _u32p, _f32p, _u32p, _f32p]
        _pp = C.POINTER(C.c_void_p)
        L.orc_pcg_ref_f32_many.argtypes = [C.c_uint32, _u32p, _pp, _pp, _pp, _u32p, _pp, _pp, _pp, _pp,
                                           C.c_uint64, C.c_float, C.c_float, C.c_uint32, _ip, _u64p]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def lu_factor_inplace_6(mat: np.ndarray, n: int):
    """compute.rs:37-71. Returns (status, pivot_k); mat (36 f32) is modified."""
    k = C.c_int(-1)
    st = lib().orc_lu_factor_inplace_6(_p(mat, _f32p), n, C.byref(k))
    return st, k.value


def build_lu_blocks_6(n, row_ptr, col_idx, values, block_starts):
    """compute.rs:84-181. Returns (status, lu f32[nb*36], bad_block, pivot_k)."""
    row_ptr, col_idx, values, bs = _u32(row_ptr), _u32(col_idx), _f32(values), _u32(block_starts)
    nb = max(len(bs) - 1, 0)
    out = np.zeros(max(nb, 1) * 36, np.float32)
    bad, pk = C.c_int64(-1), C.c_int(-1)
    if len(row_ptr) != n + 1:
        return BAD_INPUT, out[: nb * 36], -1, -1
    st = lib().orc_build_lu_blocks_6(n, _p(row_ptr, _u32p), len(row_ptr), _p(col_idx, _u32p), len(col_idx),
                                     _p(values, _f32p), len(values), _p(bs, _u32p), len(bs), _p(out, _f32p),
                                     C.byref(bad), C.byref(pk))
    return st, out[: nb * 36], bad.value, pk.value


def spmv(row_ptr, col_idx, values, x):
    n = len(row_ptr) - 1
    y = np.zeros(n, np.float32)
    lib().orc_spmv_csr(n, _p(_u32(row_ptr), _u32p), _p(_u32(col_idx), _u32p), _p(_f32(values), _f32p),
                       _p(_f32(x), _f32p), _p(y, _f32p))
    return y


def dot_tree256(a, b) -> np.float32:
    a, b = _f32(a), _f32(b)
    return np.float32(lib().orc_dot_tree256(len(a), _p(a, _f32p), _p(b, _f32p)))


def block_jacobi_apply(n, lu, block_starts, r, z=None):
    bs = _u32(block_starts)
    z = np.zeros(n, np.float32) if z is None else _f32(z).copy()
    lib().orc_block_jacobi_apply(n, max(len(bs) - 1, 0), _p(_f32(lu), _f32p), _p(bs, _u32p), _p(_f32(r), _f32p),
                                 _p(z, _f32p))
    return z


def axpy(alpha, x, y):
    y = _f32(y).copy()
    lib().orc_axpy(len(y), np.float32(alpha), _p(_f32(x), _f32p), _p(y, _f32p))
    return y


def scale(s, x):
    x = _f32(x).copy()
    lib().orc_scale(len(x), np.float32(s), _p(x, _f32p))
    return x


def update_scalars(s, p_ap, rz_new, rz_old, alpha, minus_alpha, beta):
    s = _f32(s).copy()
    lib().orc_update_scalars(_p(s, _f32p), p_ap, rz_new, rz_old, alpha, minus_alpha, beta)
    return s


def pcg_ref_f32(row_ptr, col_idx, values, lu, block_starts, b, x0, max_iter, rel_tol, abs_tol):
    """compute.rs:189-495. Returns dict(status, iterations, x, history, breakdown)."""
    n = len(row_ptr) - 1
    bs = _u32(block_starts)
    x = _f32(x0).copy()
    hist = np.zeros(max(int(max_iter), 1), np.float32)
    it, bk = C.c_uint64(0), C.c_int(0)
    st = lib().orc_pcg_ref_f32(n, _p(_u32(row_ptr), _u32p), _p(_u32(col_idx), _u32p), _p(_f32(values), _f32p),
                               max(len(bs) - 1, 0), _p(_f32(lu), _f32p), _p(bs, _u32p), _p(_f32(b), _f32p),
                               _p(x, _f32p), int(max_iter), np.float32(rel_tol), np.float32(abs_tol),
                               C.byref(it), _p(hist, _f32p), C.byref(bk))
    return dict(status=st, iterations=it.value, x=x, history=hist[: it.value], breakdown=bk.value)


def pcg_f64dot(row_ptr, col_idx, values, lu, block_starts, b, x0, max_iter, rel_tol, abs_tol):
    n = len(row_ptr) - 1
    bs = _u32(block_starts)
    x = _f32(x0).copy()
    hist = np.zeros(max(int(max_iter), 1), np.float64)
    it, bk = C.c_uint64(0), C.c_int(0)
    st = lib().orc_pcg_f64dot(n, _p(_u32(row_ptr), _u32p), _p(_u32(col_idx), _u32p), _p(_f32(values), _f32p),
                              max(len(bs) - 1, 0), _p(_f32(lu), _f32p), _p(bs, _u32p), _p(_f32(b), _f32p),
                              _p(x, _f32p), int(max_iter), np.float32(rel_tol), np.float32(abs_tol),
                              C.byref(it), _p(hist, _f64p), C.byref(bk))
    return dict(status=st, iterations=it.value, x=x, history=hist[: it.value], breakdown=bk.value)


def pcg_single_reduction_f64dot(row_ptr, col_idx, values, lu, block_starts, b, x0, max_iter, rel_tol, abs_tol):
    """The single-reduction (Chronopoulos-Gear) PCG recurrence with the
    product's arithmetic. Returns dict(status, iterations, x, history)."""
    n = len(row_ptr) - 1
    bs = _u32(block_starts)
    x = _f32(x0).copy()
    hist = np.zeros(max(int(max_iter), 1), np.float64)
    it = C.c_uint64(0)
    st = lib().orc_pcg_single_reduction_f64dot(n, _p(_u32(row_ptr), _u32p), _p(_u32(col_idx), _u32p),
                                               _p(_f32(values), _f32p), max(len(bs) - 1, 0), _p(_f32(lu), _f32p),
                                               _p(bs, _u32p), _p(_f32(b), _f32p), _p(x, _f32p), int(max_iter),
                                               np.float32(rel_tol), np.float32(abs_tol), C.byref(it),
                                               _p(hist, _f64p))
    return dict(status=st, iterations=it.value, x=x, history=hist[: it.value])


def pcg_f64(row_ptr, col_idx, values, block_starts, b, x0=None, max_iter=100000, rel_tol=1e-12):
    n = len(row_ptr) - 1
    bs = _u32(block_starts)
    b64 = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n, np.float64) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
    it = C.c_uint64(0)
    st = lib().orc_pcg_f64(n, _p(_u32(row_ptr), _u32p), _p(_u32(col_idx), _u32p), _p(_f32(values), _f32p),
                           max(len(bs) - 1, 0), _p(bs, _u32p), _p(b64, _f64p), _p(x, _f64p), int(max_iter),
                           float(rel_tol), C.byref(it))
    return dict(status=st, iterations=it.value, x=x)


def true_relres_f64(row_ptr, col_idx, values, b, x):
    n = len(row_ptr) - 1
    x32 = _f32(x) if np.asarray(x).dtype != np.float64 else None
    x64 = np.ascontiguousarray(x, dtype=np.float64) if x32 is None else None
    return lib().orc_true_relres_f64(n, _p(_u32(row_ptr), _u32p), _p(_u32(col_idx), _u32p),
                                     _p(_f32(values), _f32p), _p(_f32(b), _f32p), _p(x32, _f32p),
                                     _p(x64, _f64p))


def compare_x(x_ref, x):
    """main.rs:603-662 statistics: dict(l2_ref, l2_err, rel_l2, rmse, max_abs_err)."""
    x_ref, x = _f32(x_ref), _f32(x)
    out = np.zeros(5, np.float64)
    lib().orc_compare_x(min(len(x_ref), len(x)), _p(x_ref, _f32p), _p(x, _f32p), _p(out, _f64p))
    return dict(l2_ref=out[0], l2_err=out[1], rel_l2=out[2], rmse=out[3], max_abs_err=out[4])


def num_threads() -> int:
    return lib().orc_num_threads()


def lattice_generate(side: int, seed: int = 0, aniso_log10: float = 0.0) -> dict:
    """The synthetic 6-DOF lattice system of side `side` (row_ptr, col_idx,
    values, block_starts, b, n, nnz), generated by the oracle's own statement
    of the generator; bit-identical to the product's wsb_lattice_generate."""
    sz = np.zeros(3, np.uint64)
    if lib().orc_lattice_sizes(int(side), _p(sz, _u64p)) != OK:
        raise ValueError(f"lattice side {side} is too large")
    n, nnz, nodes = int(sz[0]), int(sz[1]), int(sz[2])
    rp = np.empty(n + 1, np.uint32)
    ci = np.empty(nnz, np.uint32)
    v = np.empty(nnz, np.float32)
    bs = np.empty(nodes + 1, np.uint32)
    b = np.empty(n, np.float32)
    st = lib().orc_lattice_generate(int(side), int(seed), float(aniso_log10), _p(rp, _u32p), _p(ci, _u32p),
                                    _p(v, _f32p), _p(bs, _u32p), _p(b, _f32p))
    if st != OK:
        raise RuntimeError(f"orc_lattice_generate failed with status {st}")
    return dict(row_ptr=rp, col_idx=ci, values=v, block_starts=bs, b=b, n=n, nnz=nnz)


def pcg_ref_f32_many(systems, max_iter, rel_tol, abs_tol=0.0, par_min_n=200_000):
    """Complete FP32 reference solves (orc_pcg_ref_f32) of many independent
    systems, each a dict with row_ptr, col_idx, values, block_starts, b and its
    `lu` (f32[36 nb]); x0 = 0. Systems with n >= par_min_n run one after the
    other with every host thread inside each solve, the smaller ones
    concurrently with one thread each. Returns a list of dict(status,
    iterations, x) in the order given."""
    cnt = len(systems)
    order = sorted(range(cnt), key=lambda i: -len(systems[i]["b"]))
    keep = []  # contiguous arrays that must outlive the call

    def ptr(a, dtype):
        a = np.ascontiguousarray(a, dtype=dtype)
        keep.append(a)
        return a.ctypes.data

    vp = C.c_void_p * cnt
    n_arr = np.zeros(cnt, np.uint32)
    nb_arr = np.zeros(cnt, np.uint32)
    rp, ci, va, lu, bs, bb, xx = vp(), vp(), vp(), vp(), vp(), vp(), vp()
    xs = []
    for j, i in enumerate(order):
        s = systems[i]
        n = len(s["b"])
        n_arr[j] = n
        nb_arr[j] = max(len(s["block_starts"]) - 1, 0)
        rp[j] = ptr(s["row_ptr"], np.uint32)
        ci[j] = ptr(s["col_idx"], np.uint32)
        va[j] = ptr(s["values"], np.float32)
        lu[j] = ptr(s["lu"], np.float32)
        bs[j] = ptr(s["block_starts"], np.uint32)
        bb[j] = ptr(s["b"], np.float32)
        x = np.zeros(n, np.float32)
        xs.append(x)
        xx[j] = x.ctypes.data
    status = np.zeros(cnt, np.int32)
    iters = np.zeros(cnt, np.uint64)
    cast = lambda a: C.cast(a, C.POINTER(C.c_void_p))  # noqa: E731
    lib().orc_pcg_ref_f32_many(cnt, _p(n_arr, _u32p), cast(rp), cast(ci), cast(va), _p(nb_arr, _u32p), cast(lu),
                               cast(bs), cast(bb), cast(xx), int(max_iter), np.float32(rel_tol),
                               np.float32(abs_tol), int(par_min_n), _p(status, _ip), _p(iters, _u64p))
    out = [None] * cnt
    for j, i in enumerate(order):
        out[i] = dict(status=int(status[j]), iterations=int(iters[j]), x=xs[j])
    return out

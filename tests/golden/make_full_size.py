"""Full-size oracle fixtures for the GPU parity tests (CPU only, run once).

Runs the oracle on the 80^3 lattice systems that the GPU tests solve and
keeps small summaries of the results:

  lattice80_f64dot.npz   orc_pcg_f64dot (FP32 vectors, FP64 reductions: the
                         product's default arithmetic) on side 80, seed 2024,
                         relative tolerance 1e-6: iterations, the FP64 residual
                         history, and x at 4096 evenly strided rows.
  lattice80_ref_f32.npz  orc_pcg_ref_f32 (the reference algorithm, compute.rs
                         189-495, bit for bit) on the same system: iterations,
                         the FP32 history, x at the strided rows and the
                         SHA-256 of all of x.
  aniso80_f64.npz        orc_pcg_f64 (full FP64 PCG) on side 80, seed 2024,
                         anisotropy 10^U(-3,3), to relative residual 1e-12:
                         iterations, x at the strided rows, ||x||_2 and the
                         FP64 true relative residual of the FP64 solution.

Usage: python tests/golden/make_full_size.py [--only NAME]
"""
import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

SIDE, SEED = 80, 2024
SAMPLE = 4096


def sample_rows(n):
    return np.linspace(0, n - 1, SAMPLE).astype(np.int64)


def system(aniso):
    s = oracle.lattice_generate(SIDE, SEED, aniso)
    st, lu, _, _ = oracle.build_lu_blocks_6(s["n"], s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
    assert st == oracle.OK
    return s, lu


def make_f64dot():
    s, lu = system(0.0)
    t = time.time()
    r = oracle.pcg_f64dot(s["row_ptr"], s["col_idx"], s["values"], lu, s["block_starts"], s["b"],
                          np.zeros(s["n"], np.float32), 20000, 1e-6, 0.0)
    assert r["status"] == oracle.OK, r["status"]
    idx = sample_rows(s["n"])
    np.savez_compressed(os.path.join(HERE, "lattice80_f64dot.npz"), iterations=r["iterations"], history=r["history"],
                        rows=idx, x=r["x"][idx], x_norm=np.linalg.norm(r["x"].astype(np.float64)))
    print("f64dot", r["iterations"], f"{time.time() - t:.0f} s", flush=True)


def make_ref_f32():
    s, lu = system(0.0)
    t = time.time()
    r = oracle.pcg_ref_f32(s["row_ptr"], s["col_idx"], s["values"], lu, s["block_starts"], s["b"],
                           np.zeros(s["n"], np.float32), 20000, 1e-6, 0.0)
    assert r["status"] == oracle.OK, r["status"]
    idx = sample_rows(s["n"])
    np.savez_compressed(os.path.join(HERE, "lattice80_ref_f32.npz"), iterations=r["iterations"],
                        history=r["history"], rows=idx, x=r["x"][idx],
                        x_sha256=hashlib.sha256(r["x"].tobytes()).hexdigest())
    print("ref_f32", r["iterations"], f"{time.time() - t:.0f} s", flush=True)


def make_aniso_f64():
    s, _ = system(3.0)
    t = time.time()
    r = oracle.pcg_f64(s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], s["b"], max_iter=200000,
                       rel_tol=1e-12)
    assert r["status"] == oracle.OK, r["status"]
    tr = oracle.true_relres_f64(s["row_ptr"], s["col_idx"], s["values"], s["b"], r["x"])
    idx = sample_rows(s["n"])
    np.savez_compressed(os.path.join(HERE, "aniso80_f64.npz"), iterations=r["iterations"], rows=idx, x=r["x"][idx],
                        x_norm=np.linalg.norm(r["x"]), true_relres=tr)
    print("aniso_f64", r["iterations"], tr, f"{time.time() - t:.0f} s", flush=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["f64dot", "ref_f32", "aniso_f64"])
    a = ap.parse_args()
    jobs = {"f64dot": make_f64dot, "ref_f32": make_ref_f32, "aniso_f64": make_aniso_f64}
    for name, fn in jobs.items():
        if a.only in (None, name):
            fn()

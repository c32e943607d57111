"""Iteration counts of the reference algorithm on the serving request set.

Runs the oracle's FP32 restatement of pcg_block_jacobi_csr_wgpu
(compute.rs:189-495) on every request of bench.py's serving workload at
relative tolerance 1e-8 and writes oracle/serve_reference_iterations.json.
bench.py's CPU-baseline and reference legs time a bounded number of oracle
iterations per request and scale by these counts.

Usage: python oracle/make_serve_reference.py
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

import bench  # noqa: E402
import oracle  # noqa: E402
import wgpu_solver_backend_b200 as wsb  # noqa: E402


def main():
    oracle.build()
    out = {"tolerance": bench.SERVE["target"], "requests": []}
    t0 = time.time()
    for side, seed in bench.serve_requests():
        s = bench.serve_system(side, seed)
        n = s["n"]
        lu = wsb.build_lu_blocks_from_csr_block_starts_6(n, s["row_ptr"], s["col_idx"], s["values"],
                                                         s["block_starts"])
        r = oracle.pcg_ref_f32(s["row_ptr"], s["col_idx"], s["values"], lu, s["block_starts"], s["b"],
                               np.zeros(n, np.float32), bench.SERVE["max_iter"], bench.SERVE["target"], 0.0)
        out["requests"].append({"side": side, "seed": seed, "n": n, "status": r["status"],
                                "iterations": int(r["iterations"])})
        print(side, seed, n, r["status"], r["iterations"], f"{time.time() - t0:.0f}s", flush=True)
    with open(os.path.join(HERE, "serve_reference_iterations.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()

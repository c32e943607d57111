"""Generate the golden fixtures under tests/golden/ from the reference's datasets.

Run where a checkout of the reference repository is available and pass its
root with --reference; the GPU tests only read the committed outputs.

For each of datasets/pcg_block_jacobi_dataset_{1,2,3}.txt this script
1. parses the fea_app text format (sections ``n``, ``nnz``, ``row_ptr_u32``,
   ``col_idx_u32``, ``values_f32``, ``b_f32``, ``x0_f32``, ``block_starts_u32``,
   ``x_ref_f32``; rules of wgpu_solver_backend_convert_cli/src/main.rs:104-401),
2. writes the binary case directory ``case_k/`` (convert_cli main.rs:407-494),
3. runs the FP32 oracle at the settings of commands.txt:26-54
   (max 2000 iterations, rel 1e-4, abs 1e-7) and stores its iteration count,
   residual history and solution in ``case_k/oracle_ref_f32.npz``.

Usage: python tests/golden/make_golden.py --reference PATH_TO_REFERENCE_CHECKOUT
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from wgpu_solver_backend_b200 import io as wio  # noqa: E402
import oracle  # noqa: E402


def parse_text_dataset(path):
    """Section parser following convert_cli main.rs:104-401."""
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    lines = [ln for ln in lines if ln and not ln.startswith("#")]
    out, i = {}, 0
    while i < len(lines):
        ln = lines[i]
        if ln.startswith("n "):
            out["n"] = int(ln[2:]); i += 1; continue
        if ln.startswith("nnz "):
            out["nnz"] = int(ln[4:]); i += 1; continue
        sec = ln
        need = int(lines[i + 1].split()[1])
        i += 2
        toks = []
        while len(toks) < need:
            toks.extend(lines[i].split())
            i += 1
        toks = toks[:need]
        if sec.endswith("_u32"):
            out[sec] = np.array([int(t) for t in toks], np.uint32)
        else:
            out[sec] = np.array([float(t) for t in toks], np.float64).astype(np.float32)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference repository checkout")
    args = ap.parse_args()
    oracle.build()
    summary = {}
    for k in (1, 2, 3):
        src = os.path.join(args.reference, "datasets", f"pcg_block_jacobi_dataset_{k}.txt")
        ds = parse_text_dataset(src)
        case = os.path.join(HERE, f"case_{k}")
        wio.write_case_dir(case, ds["row_ptr_u32"], ds["col_idx_u32"], ds["values_f32"], ds["b_f32"],
                           ds["x0_f32"], ds["block_starts_u32"], ds.get("x_ref_f32"))
        st, lu, bad, pk = oracle.build_lu_blocks_6(ds["n"], ds["row_ptr_u32"], ds["col_idx_u32"],
                                                   ds["values_f32"], ds["block_starts_u32"])
        assert st == 0, (k, st, bad, pk)
        res = oracle.pcg_ref_f32(ds["row_ptr_u32"], ds["col_idx_u32"], ds["values_f32"], lu,
                                 ds["block_starts_u32"], ds["b_f32"], ds["x0_f32"], 2000, 1e-4, 1e-7)
        assert res["status"] == 0, res["status"]
        cmp = oracle.compare_x(ds["x_ref_f32"], res["x"])
        np.savez(os.path.join(case, "oracle_ref_f32.npz"), x=res["x"], history=res["history"],
                 iterations=np.int64(res["iterations"]), lu=lu)
        summary[f"case_{k}"] = dict(n=int(ds["n"]), nnz=int(ds["nnz"]), iterations=int(res["iterations"]),
                                    rel_l2_vs_x_ref=float(cmp["rel_l2"]), rmse_vs_x_ref=float(cmp["rmse"]))
        print(k, summary[f"case_{k}"])
    with open(os.path.join(HERE, "oracle_summary.json"), "w") as f:
        json.dump(summary, f, indent=2)


if __name__ == "__main__":
    main()

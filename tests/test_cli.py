"""The command-line tools against the reference CLI's behaviour.

wgpu_solver_backend_convert_cli text-to-bin must write byte-identical case
directories to the committed fixtures (which follow convert_cli
main.rs:407-494) and fail with the reference's messages and exit code 1;
wgpu_solver_backend_cli compare-x must reproduce the statistics of
cli main.rs:603-662 (checked against the oracle), the pass rule rel_l2 <= rtol
or rmse <= atol, and exit 2 on failure; run-pcg-case and the five sanity
subcommands (main.rs:171-443) run on the GPU.
"""
import json
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from conftest import BIN, COMPARE_X_GATES, GOLDEN, load_case

CLI = os.path.join(BIN, "wgpu_solver_backend_cli")
CONVERT = os.path.join(BIN, "wgpu_solver_backend_convert_cli")
CASE_FILES = ("matrix.csr.bin", "rhs.bin", "x0.bin", "block_starts.bin", "x_ref.bin", "meta.json")


def run(*args, **kw):
    return subprocess.run([str(a) for a in args], capture_output=True, text=True, timeout=300, **kw)


def _tokens(arr, per_line=16):
    a = list(arr)
    if arr.dtype == np.float32:
        a = [str(np.float32(v)) for v in a]
    else:
        a = [str(int(v)) for v in a]
    return "\n".join(" ".join(a[i:i + per_line]) for i in range(0, len(a), per_line))


def write_text_dataset(path, case, x_ref=None, extra=""):
    """The dataset text bundle (sections as convert_cli main.rs:104-401 reads them)."""
    a = case.a
    parts = ["# dataset (text)", f"n {a.n_rows}", f"nnz {a.nnz}", ""]
    secs = [("row_ptr_u32", a.row_ptr), ("col_idx_u32", a.col_idx), ("values_f32", a.values),
            ("b_f32", case.b), ("x0_f32", case.x0), ("block_starts_u32", case.block_starts)]
    if x_ref is not None:
        secs.append(("x_ref_f32", x_ref))
    for name, arr in secs:
        parts += [name, f"len {len(arr)}", _tokens(np.asarray(arr)), ""]
    with open(path, "w") as f:
        f.write("\n".join(parts) + extra)


# ---------------------------------------------------------------------------
# text-to-bin (CPU)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("k", [1, 2, 3])
def test_text_to_bin_writes_the_fixture_bytes(tmp_path, k):
    case, x_ref, _ = load_case(k)
    txt = tmp_path / "ds.txt"
    write_text_dataset(txt, case, x_ref)
    out = tmp_path / "case"
    r = run(CONVERT, "text-to-bin", "--input", txt, "--out-dir", out)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == f"Wrote binaries into {out}"
    for f in CASE_FILES:
        with open(out / f, "rb") as a, open(os.path.join(GOLDEN, f"case_{k}", f), "rb") as b:
            assert a.read() == b.read(), f


def test_text_to_bin_without_x_ref_and_with_unknown_section(tmp_path):
    case, _, _ = load_case(1)
    txt = tmp_path / "ds.txt"
    write_text_dataset(txt, case, None, extra="\nextra_stuff\nlen 5\n1 2 3\n4 5\n")
    out = tmp_path / "case"
    r = run(CONVERT, "text-to-bin", "--input", txt, "--out-dir", out)
    assert r.returncode == 0, r.stderr
    assert "Warning: skipping unknown section: extra_stuff (len 5)" in r.stderr
    assert not (out / "x_ref.bin").exists()
    meta = json.loads((out / "meta.json").read_text())
    assert meta["x_ref_present"] is False and meta["format"] == "wgpu-solver-backend-text-v0"


def test_text_to_bin_refuses_an_existing_dir_without_force(tmp_path):
    case, x_ref, _ = load_case(1)
    txt = tmp_path / "ds.txt"
    write_text_dataset(txt, case, x_ref)
    out = tmp_path / "case"
    out.mkdir()
    (out / "stale.txt").write_text("x")
    r = run(CONVERT, "text-to-bin", "--input", txt, "--out-dir", out)
    assert r.returncode == 1
    assert r.stderr.strip() == f'Error: "Output dir {out} already exists. Use --force to overwrite."'
    r = run(CONVERT, "text-to-bin", "--input", txt, "--out-dir", out, "--force")
    assert r.returncode == 0 and not (out / "stale.txt").exists()


@pytest.mark.parametrize("seed", range(6))
def test_text_to_bin_round_trip_of_random_systems(tmp_path, seed):
    """Random lattice systems written with varying tokens per line (the
    parser reads whitespace-separated tokens, convert_cli main.rs:104-401):
    the binaries load back to the same arrays, bit for bit."""
    from types import SimpleNamespace

    from wgpu_solver_backend_b200 import io as wio
    import wgpu_solver_backend_b200 as wsb

    rng = np.random.default_rng(seed)
    s = wsb.lattice_generate(int(rng.integers(1, 5)), seed=seed)
    n = s["n"]
    a = SimpleNamespace(n_rows=n, nnz=len(s["values"]), row_ptr=s["row_ptr"], col_idx=s["col_idx"],
                        values=s["values"])
    x0 = rng.normal(size=n).astype(np.float32)
    x_ref = rng.normal(size=n).astype(np.float32)
    case = SimpleNamespace(a=a, b=s["b"], x0=x0, block_starts=s["block_starts"])
    txt = tmp_path / "ds.txt"
    per_line = int(rng.integers(1, 40))
    parts = ["# dataset (text)", f"n {n}", f"nnz {a.nnz}", ""]
    for name, arr in [("row_ptr_u32", a.row_ptr), ("col_idx_u32", a.col_idx), ("values_f32", a.values),
                      ("b_f32", case.b), ("x0_f32", x0), ("block_starts_u32", case.block_starts),
                      ("x_ref_f32", x_ref)]:
        parts += [name, f"len {len(arr)}", _tokens(np.asarray(arr), per_line), ""]
    txt.write_text("\n".join(parts))
    out = tmp_path / "case"
    r = run(CONVERT, "text-to-bin", "--input", txt, "--out-dir", out)
    assert r.returncode == 0, r.stderr
    c = wio.load_case_dir(str(out))
    for got, want in [(c.a.row_ptr, a.row_ptr), (c.a.col_idx, a.col_idx), (c.a.values, a.values), (c.b, case.b),
                      (c.x0, x0), (c.block_starts, case.block_starts), (wio.load_vector_bin(str(out / "x_ref.bin")),
                                                                          x_ref)]:
        assert np.array_equal(np.asarray(got).view(np.uint32), np.asarray(want).view(np.uint32))
    meta = json.loads((out / "meta.json").read_text())
    assert meta["n"] == n and meta["nnz"] == a.nnz and meta["x_ref_present"] is True


@pytest.mark.parametrize("text,msg", [
    ("nnz 1\nrow_ptr_u32\nlen 2\n0 1\n", "Missing 'n'"),
    ("n 1\nnnz 1\nrow_ptr_u32\nlen 3\n0 1\n", "Section row_ptr_u32: EOF while reading values (got 2, need 3)"),
    ("n 1\nnnz 1\nrow_ptr_u32\nlength 2\n", "Section row_ptr_u32: expected 'len N', got 'length 2'"),
    ("n 1\nnnz 1\nrow_ptr_u32\nlen 3\n0 1\ncol_idx_u32\n",
     "Section row_ptr_u32: hit unexpected header 'col_idx_u32' before collecting len=3 values"),
    ("n 1\nnnz 1\nvalues_f32\nlen 1\nabc\n", "Section values_f32: failed to parse f32 token 'abc': invalid float literal"),
    ("n 2\nnnz 1\nrow_ptr_u32\nlen 3\n0 1 1\ncol_idx_u32\nlen 1\n0\nvalues_f32\nlen 1\n1.0\nb_f32\nlen 2\n1 1\n"
     "x0_f32\nlen 2\n0 0\nblock_starts_u32\nlen 4\n0 1 1 2\n", "block_starts_u32 must be strictly increasing"),
    ("n 2\nnnz 1\nrow_ptr_u32\nlen 2\n0 1\ncol_idx_u32\nlen 1\n0\nvalues_f32\nlen 1\n1.0\nb_f32\nlen 2\n1 1\n"
     "x0_f32\nlen 2\n0 0\nblock_starts_u32\nlen 2\n0 2\n", "row_ptr_u32 len must be n+1 (3), got 2"),
])
def test_text_to_bin_errors_follow_the_reference(tmp_path, text, msg):
    txt = tmp_path / "bad.txt"
    txt.write_text(text)
    r = run(CONVERT, "text-to-bin", "--input", txt, "--out-dir", tmp_path / "o")
    assert r.returncode == 1
    assert r.stderr.strip() == f'Error: "{msg}"'


# ---------------------------------------------------------------------------
# compare-x (CPU)
# ---------------------------------------------------------------------------
def _stats(stdout):
    keys = {"||x_ref||_2": "l2_ref", "||x - x_ref||_2": "l2_err", "rel_l2": "rel_l2", "rmse": "rmse",
            "max_abs_err (diag)": "max_abs_err"}
    out = {}
    for line in stdout.splitlines():
        m = re.match(r"\s+(.+?)\s+: (\S+)$", line)
        if m and m.group(1) in keys:
            out[keys[m.group(1)]] = float(m.group(2))
    return out


def test_compare_x_statistics_match_the_oracle(tmp_path):
    import oracle
    from wgpu_solver_backend_b200 import io as wio

    x_ref = wio.load_vector_bin(os.path.join(GOLDEN, "case_3", "x_ref.bin"))
    rng = np.random.default_rng(5)
    x = (x_ref * (1 + 1e-4 * rng.standard_normal(len(x_ref)))).astype(np.float32)
    wio.write_vector_bin(str(tmp_path / "x.bin"), x)
    r = run(CLI, "compare-x", "--x-ref", os.path.join(GOLDEN, "case_3", "x_ref.bin"), "--x", tmp_path / "x.bin",
            "--top-k", "4")
    want = oracle.compare_x(x_ref, x)
    got = _stats(r.stdout)
    for k, v in want.items():
        assert got[k] == pytest.approx(v, rel=1e-9, abs=1e-300), k
    assert r.returncode == (0 if (want["rel_l2"] <= np.float32(1e-3) or want["rmse"] <= np.float32(1e-4)) else 2)
    worst = re.findall(r"i=(\d+)\s+x_ref=(\S+)\s+x=(\S+)\s+abs=(\S+)", r.stdout)
    err = np.abs(x - x_ref)
    assert [int(w[0]) for w in worst] == list(np.argsort(-err, kind="stable")[:4])


def test_compare_x_pass_rules_and_exit_codes(tmp_path):
    from wgpu_solver_backend_b200 import io as wio

    ref = os.path.join(GOLDEN, "case_2", "x_ref.bin")
    x_ref = wio.load_vector_bin(ref)
    same = run(CLI, "compare-x", "--x-ref", ref, "--x", ref)
    assert same.returncode == 0 and "  pass               : true" in same.stdout
    x = x_ref.copy()
    x[7] += np.float32(3.0)
    wio.write_vector_bin(str(tmp_path / "x.bin"), x)
    # rel_l2 is tiny (|x_ref| ~ 4e6) although one entry is off by 3: passes on rel_l2 alone.
    r = run(CLI, "compare-x", "--x-ref", ref, "--x", tmp_path / "x.bin", "--rel-tol", "1e-3", "--abs-tol", "1e-6")
    assert r.returncode == 0 and "  pass_rel_l2        : true" in r.stdout and "  pass_rmse          : false" in r.stdout
    r = run(CLI, "compare-x", "--x-ref", ref, "--x", tmp_path / "x.bin", "--rel-tol", "1e-9", "--abs-tol", "1e-6")
    assert r.returncode == 2 and r.stderr.strip() == "CompareX failed tolerances (rel_l2 and rmse)"
    assert "  rtol (rel L2)      : 1.000e-9" in r.stdout
    r = run(CLI, "compare-x", "--x-ref", ref, "--x", os.path.join(GOLDEN, "case_1", "x_ref.bin"))
    assert r.returncode == 2 and r.stderr.strip() == "Length mismatch: x_ref len 807 vs x len 48"
    r = run(CLI, "compare-x", "--x-ref", tmp_path / "missing.bin", "--x", ref)
    assert r.returncode == 2 and r.stderr.startswith(f"open {tmp_path / 'missing.bin'}: No such file or directory")


def test_cli_usage_errors_exit_2():
    assert run(CLI, "no-such-command").returncode == 2
    assert run(CLI, "run-pcg-case", "--case-dir", "x").returncode == 2
    r = run(CLI, "--version")
    assert r.returncode == 0 and r.stdout.strip() == "wgpu-solver-backend 0.1.0"


# ---------------------------------------------------------------------------
# GPU: run-pcg-case, info and the sanity subcommands
# ---------------------------------------------------------------------------
SANITY = {
    "vec-test": "VecTest OK: all y[i] == 7",
    "dot-test": "DotTest OK: got 32",
    "spmv-test": "SpmvTest OK: y == [16.0, 21.0, 38.0]",
    "block-jacobi-test": "BlockJacobiTest OK: z == r (identity blocks)",
    "pcg-update-scalars-test": "PcgUpdateScalarsTest OK: alpha=5, minus_alpha=-5, beta=0.5",
}
METRIC_KEYS = ["run_id", "command", "case_dir", "n", "nnz", "max_iters", "rel_tol", "abs_tol", "iterations",
               "converged", "error", "timings_ms", "gpu", "build"]


@pytest.mark.gpu
@pytest.mark.parametrize("cmd", list(SANITY))
def test_sanity_subcommands(cmd):
    r = run(CLI, "--backend", "vulkan", cmd)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == SANITY[cmd]


@pytest.mark.gpu
def test_info_prints_adapter_and_metrics():
    r = run(CLI, "info")
    assert r.returncode == 0, r.stderr
    desc, blob = r.stdout.split("\n", 1)
    assert "backend=Cuda" in desc
    m = json.loads(blob)
    assert list(m) == ["run_id", "command", "gpu", "build"] and m["command"] == "info"
    assert m["gpu"]["vendor"] == 0x10DE


@pytest.mark.gpu
@pytest.mark.parametrize("k", [1, 2, 3])
@pytest.mark.parametrize("precision", ["reference-f32", "f32-f64dot"])
def test_run_pcg_case_then_compare_x(tmp_path, k, precision):
    """commands.txt:26-78 end to end: solve at rel 1e-4, abs 1e-7, max 2000,
    then compare-x against x_ref with the dataset's gate."""
    case, _, fx = load_case(k)
    out_x, out_m = tmp_path / "out" / "x.bin", tmp_path / "out" / "metrics.json"
    r = run(CLI, "--backend", "auto", "run-pcg-case", "--case-dir", os.path.join(GOLDEN, f"case_{k}"),
            "--max-iters", "2000", "--rel-tol", "1e-4", "--abs-tol", "1e-7", "--out-x", out_x,
            "--out-metrics", out_m, "--precision", precision)
    assert r.returncode == 0, r.stderr
    m = json.loads(out_m.read_text())
    assert list(m)[: len(METRIC_KEYS)] == METRIC_KEYS
    assert m["converged"] is True and m["error"] is None and m["command"] == "run_pcg_case"
    assert m["rel_tol"] == 1e-4 and '"abs_tol": 1e-7' in out_m.read_text()
    it_oracle = int(fx["iterations"])
    if precision == "reference-f32":
        assert m["iterations"] == it_oracle
        from wgpu_solver_backend_b200 import io as wio

        np.testing.assert_array_equal(wio.load_vector_bin(str(out_x)), fx["x"])
    else:
        assert abs(m["iterations"] - it_oracle) <= max(2, 0.02 * it_oracle)
    # This implementation's result checks in the `solver` object: the true
    # FP64 residual of the written x and one iteration's algorithmic bytes.
    from wgpu_solver_backend_b200 import io as wio

    xs = wio.load_vector_bin(str(out_x))
    tr = oracle.true_relres_f64(case.a.row_ptr, case.a.col_idx, case.a.values, case.b, xs)
    assert m["solver"]["final_relres_true_f64"] == pytest.approx(tr, rel=1e-9)
    n, nnz, nb = case.a.n_rows, case.a.nnz, len(case.block_starts) - 1
    assert m["solver"]["iteration_bytes"] == 8 * nnz + 4 * (n + 1) + 48 * n + 144 * nb
    rel, atol = COMPARE_X_GATES[k]
    c = run(CLI, "compare-x", "--x-ref", os.path.join(GOLDEN, f"case_{k}", "x_ref.bin"), "--x", out_x,
            "--rel-tol", rel, "--abs-tol", atol, "--top-k", "10")
    assert c.returncode == 0, c.stdout + c.stderr


@pytest.mark.gpu
def test_run_pcg_case_failure_is_reported_in_metrics(tmp_path):
    """A solve that does not converge: exit 0, converged false, x.bin not written."""
    out_x, out_m = tmp_path / "x.bin", tmp_path / "m.json"
    r = run(CLI, "run-pcg-case", "--case-dir", os.path.join(GOLDEN, "case_3"), "--max-iters", "5",
            "--rel-tol", "1e-8", "--out-x", out_x, "--out-metrics", out_m)
    assert r.returncode == 0
    m = json.loads(out_m.read_text())
    assert m["converged"] is False and m["iterations"] is None and "did not converge" in m["error"]
    assert m["solver"]["final_relres_true_f64"] is None and m["solver"]["gbps"] is None
    assert not out_x.exists()
    assert r.stderr.startswith("Solve failed: ")


@pytest.mark.gpu
@pytest.mark.parametrize("k", [2, 3])
def test_run_pcg_case_single_reduction(tmp_path, k):
    """--algorithm single-reduction: the opt-in recurrence through the CLI
    passes the dataset's compare-x gate, and the metrics name it and count
    its extra vector (4 bytes per row more than the classic iteration)."""
    case, _, fx = load_case(k)
    out_x, out_m = tmp_path / "out" / "x.bin", tmp_path / "out" / "metrics.json"
    r = run(CLI, "run-pcg-case", "--case-dir", os.path.join(GOLDEN, f"case_{k}"), "--max-iters", "2000",
            "--rel-tol", "1e-4", "--abs-tol", "1e-7", "--out-x", out_x, "--out-metrics", out_m,
            "--algorithm", "single-reduction")
    assert r.returncode == 0, r.stderr
    m = json.loads(out_m.read_text())
    assert m["converged"] is True and m["solver"]["algorithm"] == "single-reduction"
    n, nnz, nb = case.a.n_rows, case.a.nnz, len(case.block_starts) - 1
    assert m["solver"]["iteration_bytes"] == 8 * nnz + 4 * (n + 1) + 52 * n + 144 * nb
    # A different recurrence: on the ill-conditioned third dataset it takes
    # 1,348 iterations where the reference's takes 1,273 (measured on B200).
    assert abs(m["iterations"] - int(fx["iterations"])) <= max(2, 0.10 * int(fx["iterations"]))
    rel, atol = COMPARE_X_GATES[k]
    c = run(CLI, "compare-x", "--x-ref", os.path.join(GOLDEN, f"case_{k}", "x_ref.bin"), "--x", out_x,
            "--rel-tol", str(rel), "--abs-tol", str(atol))
    assert c.returncode == 0, c.stdout + c.stderr

"""Multi-process logic of bench.py on CPU (gloo, world size 2): the path has
no exchange step, so ranks are independent replicas that only meet for the
barrier and the max-over-ranks time, and the reference arm runs on rank 0
alone. Also the reference arm's JSON line, which needs no GPU."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        w, r, _ = bench.dist_setup()
        bench.barrier(w)
        # Per-rank "timed region": rank r takes 1.5 + r seconds for 3 steps.
        slowest = bench.reduce_max(1.5 + r, w)
        value = bench.replica_rate(w, 3, slowest)
        bench.barrier(w)
        with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
            json.dump({"world": w, "rank": r, "slowest": slowest, "value": value}, f)
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_time_over_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r, g in enumerate(got):
        assert g["world"] == world and g["rank"] == r
        assert g["slowest"] == 2.5                 # max over ranks, on every rank
        assert g["value"] == pytest.approx(2 * 3 / 2.5)  # all ranks' units / slowest time


def test_replica_rate_is_weak_scaling():
    # Fixed work per rank: N ranks at the same time give N times the rate.
    assert bench.replica_rate(1, 64, 2.0) == 32.0
    assert bench.replica_rate(8, 64, 2.0) == 8 * 32.0


@pytest.mark.parametrize("workload", ["serve", "plain80"])
def test_reference_arm_runs_on_rank_zero_only(workload):
    # A non-zero rank of the reference arm exits 0 at once, without output or work.
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--workload", workload], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


def test_reference_arm_line_on_one_rank():
    # The reference arm runs on host cores only: its JSON line carries the
    # contract's keys, the CPU baseline it measured and a zero-copy e2e.
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE")}
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "3",
                        "--warmup", "1", "--max-side", "8"], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == "solves/s"
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 3
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert d["cpu_baseline"]["cores"] >= 1
    # Complete solves of every request of the (reduced) set, not a projection.
    n_req = len(bench.serve_set(8))
    assert d["reference_results"] == {**d["reference_results"], "converged": n_req, "of": n_req}
    assert "complete solves" in d["cpu_baseline"]["sample"]
    # The reference process maps the oracle and never the product library.
    assert d["repo_libraries_loaded"] == ["oracle/liboracle.so"]
    assert d["e2e"] == {"value": d["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_fcfs_replay_of_the_plain_path():
    # One request at a time in arrival order: a request waits for the one
    # before it to finish.
    lat = bench.fcfs_latencies([0.0, 0.1, 0.15, 2.0], [200.0, 50.0, 10.0, 5.0])
    assert lat == pytest.approx([200.0, 150.0, 110.0, 5.0])

"""Benchmark of the B200 block-Jacobi PCG.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload plain80|serve]

One JSON line on rank 0. Workloads (synthetic lattice systems, 6x6 blocks):
  plain80  one 80^3-node system (n = 3,072,000, nnz = 127,641,600), b ~ U[-1,1],
           relative tolerance 1e-6, max 20000 iterations; a step is one full
           solve with inputs resident in HBM.
  serve    an open-loop Poisson stream of solve requests (lattice side
           log-uniform in [4, 64], anisotropy 10^U(-2,2), tolerance 1e-6 or 1e-10
           with FP64 refinement), served by the continuous-batching server.
With N > 1 (torchrun) every rank runs the same workload on its own GPU as an
independent replica (the path has no exchange step); value sums the ranks'
work over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "served PCG solves/s & p99 latency vs plain per-solve PCG, 1 B200, relres 1e-8"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes per algorithmic byte of the SpMV kernel, from one ncu capture of
# k_spmv_loop on the 56^3 lattice (BSR6 tiles, 206 MB of matrix > L2; see
# profiles/k_spmv_loop_bsr6_side56.md): dram__bytes_read.sum 184.378112 MB +
# dram__bytes_write.sum 4.038656 MB over 188.285444 MB of algorithmic bytes.
# The kernel streams every byte once, so the traffic scales with the launch's
# algorithmic bytes.
SPMV_DRAM_PER_ALGO_BYTE = (184.378112e6 + 4.038656e6) / 188285444.0


def spmv_traffic(algo_bytes):
    return {"traffic": algo_bytes * SPMV_DRAM_PER_ALGO_BYTE,
            "traffic_note": "dram read+write bytes per launch, scaled from an ncu capture of the same kernel on "
                            "the 56^3 lattice (ratio %.4f to the algorithmic bytes)" % SPMV_DRAM_PER_ALGO_BYTE}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_max(val, world):
    """Maximum of a per-rank value over all ranks (the slowest rank's time)."""
    if world == 1:
        return val
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([val], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world, units_per_rank, slowest_s):
    """Whole-job rate of `world` independent replicas that each process
    `units_per_rank` units: all units over the slowest rank's time."""
    return world * units_per_rank / slowest_s


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ---------------------------------------------------------------------------
# serve: the request set
# ---------------------------------------------------------------------------
SERVE = dict(requests=64, side_min=4, side_max=64, aniso=2.0, target=1e-8, inner=1e-4, max_iter=60000, seed=7)


def serve_requests(n_req=None, seed=None):
    """(side, seed) per request: lattice side log-uniform on [4, 64], each
    system with its own seed (anisotropy 10^U(-2,2) per edge)."""
    n_req = SERVE["requests"] if n_req is None else n_req
    seed = SERVE["seed"] if seed is None else seed
    rng = np.random.default_rng(seed)
    u = rng.uniform(np.log(SERVE["side_min"]), np.log(SERVE["side_max"] + 1), n_req)
    sides = np.clip(np.floor(np.exp(u)).astype(int), SERVE["side_min"], SERVE["side_max"])
    return [(int(sd), 7_000_000 + 1000 * seed + i) for i, sd in enumerate(sides)]


def serve_system(side, seed):
    import wgpu_solver_backend_b200 as wsb

    return wsb.lattice_generate(side, seed=seed, aniso_log10=SERVE["aniso"])


# ---------------------------------------------------------------------------
# plain80
# ---------------------------------------------------------------------------
PLAIN = dict(side=80, seed=2024, rel_tol=1e-6, max_iter=20000)


def cpu_baseline_plain(sysm, lu, gpu_iters, sample_iters=600):
    """Times the oracle's FP32 restatement (all host threads) on a bounded
    sample of PCG iterations of the same system and scales to one solve."""
    import oracle

    n = sysm["n"]
    t0 = time.perf_counter()
    r = oracle.pcg_ref_f32(sysm["row_ptr"], sysm["col_idx"], sysm["values"], lu, sysm["block_starts"], sysm["b"],
                           np.zeros(n, np.float32), sample_iters, PLAIN["rel_tol"], 0.0)
    dt = time.perf_counter() - t0
    per_iter = dt / max(1, r["iterations"])
    solve_s = per_iter * gpu_iters
    return {"value": 1.0 / solve_s, "unit": "solves/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{r['iterations']} of {gpu_iters} PCG iterations of the 80^3 solve (oracle FP32, "
                      f"{oracle.num_threads()} threads), {dt:.2f} s, scaled by the GPU iteration count"}


def run_plain(args, world, rank, local):
    import torch

    import wgpu_solver_backend_b200 as wsb

    torch.cuda.set_device(local)
    ctx = wsb.GpuContext.create("auto", local)
    # A dedicated (non-default) stream shared by torch events and the library.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    s = wsb.lattice_generate(PLAIN["side"], seed=PLAIN["seed"])
    n = s["n"]
    m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], layout=wsb.LAYOUT_AUTO)
    info = m.info
    d_b = torch.from_numpy(s["b"]).cuda()
    d_x = torch.zeros(n, dtype=torch.float32, device="cuda")
    kw = dict(max_iter=PLAIN["max_iter"], rel_tol=PLAIN["rel_tol"])
    for _ in range(args.warmup):
        d_x.zero_()
        res = m.solve_device(d_b.data_ptr(), d_x.data_ptr(), **kw)
    iters = int(res["iterations"])
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        d_x.zero_()
        res = m.solve_device(d_b.data_ptr(), d_x.data_ptr(), **kw)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    dev_s = e0.elapsed_time(e1) / 1e3
    dev_s = reduce_max(dev_s, world)
    barrier(world)
    # Per-kernel device times of the solver's own loop kernels (CUDA events
    # around each launch, outside the graph), on the same matrix.
    kt = m.kernel_times(d_b.data_ptr(), iterations=20)
    spmv_s = kt["spmv_ms"] / 1e3
    peak, peak_kind = peaks()
    spmv_gbs = info["spmv_bytes"] / spmv_s / 1e9
    upd_bytes = 28 * n + 144 * info["num_blocks"]
    kernels = {"spmv": {"ms": kt["spmv_ms"], "bytes": info["spmv_bytes"], "gbs": spmv_gbs},
               "update": {"ms": kt["update_ms"], "bytes": upd_bytes, "gbs": upd_bytes / kt["update_ms"] / 1e6},
               "pupdate": {"ms": kt["pupdate_ms"], "bytes": 12 * n, "gbs": 12 * n / kt["pupdate_ms"] / 1e6}}
    iter_gbs = info["iteration_bytes"] * iters / (dev_s / args.steps) / 1e9
    # End to end through the C ABI with host buffers (copies in the timed region).
    x_host = np.zeros(n, np.float32)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        xh, r2 = m.solve(s["b"], x_host, **kw)
    torch.cuda.synchronize()
    e2e_s = reduce_max(time.perf_counter() - t0, world)
    line = {
        "metric": METRIC, "value": replica_rate(world, args.steps, dev_s), "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_s / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 reductions)",
        "data": "synthetic 80^3 6-DOF lattice, seeded",
        "config": {"workload": "plain80: one 80^3-node lattice system, n=3072000, nnz=127641600, tol 1e-6",
                   "layout": "BSR6" if info["layout"] == wsb.LAYOUT_BSR6 else "CSR",
                   "iterations": iters, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (matrix %.0f MB)" % (info["device_bytes"] / 1e6)},
        "e2e": {"value": replica_rate(world, args.steps, e2e_s), "unit": "solves/s", "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 4 * n},
        "roofline": {"bound": "hbm", "kernel": "spmv (BSR6 tiles)" if info["layout"] == wsb.LAYOUT_BSR6 else "spmv",
                     "achieved": spmv_gbs, "peak": peak, "unit": "GB/s", "frac": spmv_gbs / peak,
                     "peak_kind": peak_kind, **spmv_traffic(info["spmv_bytes"]),
                     "algorithmic_bytes_per_launch": info["spmv_bytes"], "launch_us": spmv_s * 1e6},
        "iteration_gbs": iter_gbs, "iteration_frac": iter_gbs / peak, "kernels": kernels,
        "gpu_launches": args.steps * (2 + 1 + 3 * iters),
        "clocks": clk,
    }
    if rank == 0 and world == 1:
        lu = wsb.build_lu_blocks_from_csr_block_starts_6(n, s["row_ptr"], s["col_idx"], s["values"],
                                                         s["block_starts"])
        line["cpu_baseline"] = cpu_baseline_plain(s, lu, iters)
    return line


def run_reference_plain(args, world, rank, local):
    import oracle

    import wgpu_solver_backend_b200 as wsb

    s = wsb.lattice_generate(PLAIN["side"], seed=PLAIN["seed"])
    lu = wsb.build_lu_blocks_from_csr_block_starts_6(s["n"], s["row_ptr"], s["col_idx"], s["values"],
                                                     s["block_starts"])
    # Iteration count of the full solve, from the oracle's FP64-dot variant on
    # a smaller budget is not available; the FP32 restatement's count on this
    # system is fixed by the seed (measured once, stored alongside).
    full_iters = int(os.environ.get("WSB_PLAIN80_ITERS", "0")) or 1000
    per = []
    for _ in range(args.warmup + args.steps):
        cb = cpu_baseline_plain(s, lu, full_iters, sample_iters=100)
        per.append(cb)
    vals = [c["value"] for c in per[args.warmup:]]
    v = float(np.mean(vals))
    return {"metric": METRIC, "impl": "reference", "value": v, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic 80^3 6-DOF lattice, seeded",
            "config": {"workload": "plain80: one 80^3-node lattice system, n=3072000, nnz=127641600, tol 1e-6"},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": per[-1]["cores"], "kind": "port",
                             "sample": per[-1]["sample"]},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# Server configuration of the e2e figure, and the others timed beside it
# (one burst pass each): borrow_inputs reads the caller's arrays in place
# instead of copying them at submit; device_prep builds each request's LU
# (and BSR6 form) on the GPU instead of the host.
SERVER_VARIANTS = {"copy+host_prep": dict(borrow_inputs=False, device_prep=False),
                   "borrow+host_prep": dict(borrow_inputs=True, device_prep=False),
                   "copy+device_prep": dict(borrow_inputs=False, device_prep=True),
                   "borrow+device_prep": dict(borrow_inputs=True, device_prep=True)}
SERVER_CFG = SERVER_VARIANTS["borrow+device_prep"]


def mixed_kw():
    import wgpu_solver_backend_b200 as wsb

    return dict(max_iter=SERVE["max_iter"], rel_tol=0.0, precision=wsb.PREC_MIXED_F64_IR,
                target_relres=SERVE["target"], inner_rel_tol=SERVE["inner"])


def served_pass(srv, pool, arrivals=None, targets=None):
    """Submits every request (at its arrival time, or all at once), waits for
    all. targets: per-request FP64 relative residual (default: the set's).
    Returns (makespan_s, latencies_ms, results)."""
    kw = mixed_kw()
    t0 = time.perf_counter()
    rids = []
    for i, s in enumerate(pool):
        if arrivals is not None:
            dt = t0 + arrivals[i] - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
        if targets is not None:
            kw["target_relres"] = float(targets[i])
        rids.append(srv.submit(s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], s["b"], **kw))
    res = [srv.wait(r, 600.0) for r in rids]
    mk = time.perf_counter() - t0
    return mk, [r[1]["total_ms"] for r in res], [r[1] for r in res]


def serve_set(max_side=None):
    """The requests of the serving set whose lattice side is at most max_side
    (all of them by default)."""
    max_side = SERVE["side_max"] if max_side is None else max_side
    return [(sd, seed) for sd, seed in serve_requests() if sd <= max_side]


def reference_pool(max_side=None):
    """The serving request set generated by the oracle's own statement of the
    lattice generator (bit-identical to the product's), so that the reference
    process never loads the product library."""
    import oracle

    pool = []
    for side, seed in serve_set(max_side):
        s = oracle.lattice_generate(side, seed, SERVE["aniso"])
        s["side"], s["seed"] = side, seed
        pool.append(s)
    return pool


REFERENCE_STOP = ("FP32 recursive residual r.r <= (1e-8)^2 b.b, the reference's stop test "
                  "(compute.rs:481), max 60000 iterations")


def reference_solve_requests(pool, idx):
    """Complete CPU solves of pool[i], i in idx, by the reference algorithm:
    the host LU build (compute.rs:37-181) and the FP32 PCG with the 256-wide
    tree reductions (compute.rs:189-495), both restated in the oracle; all host
    threads. Returns (seconds, lu_seconds, results)."""
    import oracle

    t0 = time.perf_counter()
    systems = []
    for i in idx:
        s = pool[i]
        st, lu, _, _ = oracle.build_lu_blocks_6(s["n"], s["row_ptr"], s["col_idx"], s["values"], s["block_starts"])
        if st != oracle.OK:
            raise RuntimeError(f"oracle LU failed on request {i} (status {st})")
        systems.append(dict(s, lu=lu))
    t1 = time.perf_counter()
    res = oracle.pcg_ref_f32_many(systems, SERVE["max_iter"], SERVE["target"], 0.0)
    return time.perf_counter() - t0, t1 - t0, res


def repo_libraries():
    """Shared objects of this repository mapped into the current process."""
    found = set()
    try:
        with open("/proc/self/maps") as f:
            for ln in f:
                path = ln.split()[-1] if ln.strip() else ""
                if path.startswith(ROOT) and ".so" in os.path.basename(path):
                    found.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(found)


def side_note(args):
    return "" if args.max_side >= SERVE["side_max"] else f", only sides <= {args.max_side}"


def step_groups(n_req, steps):
    """Requests solved by each of `steps` timed steps: contiguous groups that
    together cover the set once (or one request per step, cycling, when there
    are more steps than requests)."""
    if steps <= n_req:
        return [list(map(int, g)) for g in np.array_split(np.arange(n_req), steps)]
    return [[k % n_req] for k in range(steps)]


def cpu_baseline_serve(pool, stride=4):
    """The reference algorithm on the host cores (oracle, all threads):
    complete LU + FP32 PCG solves of every `stride`-th request of the set."""
    import oracle

    idx = list(range(0, len(pool), stride))
    dt, lu_s, res = reference_solve_requests(pool, idx)
    conv = sum(1 for r in res if r["status"] == oracle.OK)
    return {"value": len(idx) / dt, "unit": "solves/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"complete solves (LU + PCG) of every {stride}th request of the set ({len(idx)} requests, "
                      f"{sum(pool[i]['n'] for i in idx)} of {sum(p['n'] for p in pool)} unknowns), "
                      f"{dt:.1f} s ({lu_s:.2f} s LU), {oracle.num_threads()} threads; {conv} of {len(idx)} "
                      f"converged; stop: {REFERENCE_STOP}"}


def kernel_block(kt, info, n, peak):
    """Per-kernel mean launch time, algorithmic bytes, GB/s and fraction of
    the HBM peak for the three loop kernels of one matrix."""
    out = {}
    for k, b in (("spmv", info["spmv_bytes"]), ("update", 28 * n + 144 * info["num_blocks"]), ("pupdate", 12 * n)):
        ms = kt[k + "_ms"]
        out[k] = {"us": ms * 1e3, "bytes": int(b), "gbs": b / ms / 1e6, "frac": b / ms / 1e6 / peak}
    return out


def measure_c2(ctx, stream, peak):
    """The plain 80^3 system (n = 3,072,000, nnz = 127,641,600, tolerance
    1e-6) in both layouts: per-kernel times of the loop kernels (CUDA events
    per launch), whole solves (CUDA events, graph loop), per-iteration GB/s."""
    import torch

    import wgpu_solver_backend_b200 as wsb

    s = wsb.lattice_generate(PLAIN["side"], seed=PLAIN["seed"])
    n = s["n"]
    d_b = torch.from_numpy(s["b"]).cuda()
    d_x = torch.zeros(n, dtype=torch.float32, device="cuda")
    kw = dict(max_iter=PLAIN["max_iter"], rel_tol=PLAIN["rel_tol"])
    out = {"workload": "plain 80^3 lattice, n=3072000, nnz=127641600, b ~ U[-1,1], rel tol 1e-6"}
    for name, layout in (("bsr6", wsb.LAYOUT_BSR6), ("csr", wsb.LAYOUT_CSR)):
        m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], layout=layout)
        info = m.info
        torch.cuda.synchronize()
        kt = m.kernel_times(d_b.data_ptr(), iterations=20)
        d_x.zero_()
        m.solve_device(d_b.data_ptr(), d_x.data_ptr(), **kw)  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps, ms = 3, 0.0
        for _ in range(reps):
            d_x.zero_()
            torch.cuda.synchronize()
            e0.record(stream)
            r = m.solve_device(d_b.data_ptr(), d_x.data_ptr(), **kw)
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1) / reps
        it = int(r["iterations"])
        ib = info["iteration_bytes"]
        out[name] = {"kernels": kernel_block(kt, info, n, peak), "solve_ms": ms, "iterations": it,
                     "iteration_us": ms * 1e3 / it, "iteration_bytes": int(ib),
                     "iteration_gbs": ib * it / (ms / 1e3) / 1e9, "iteration_frac": ib * it / (ms / 1e3) / 1e9 / peak,
                     "matrix_bytes": int(info["device_bytes"])}
        # The opt-in single-reduction recurrence on the same matrix: two
        # kernels per iteration, SpMV + 68 n bytes (the update kernel also
        # reads and writes s and forms p = u + beta p).
        sr = dict(kw, algorithm=wsb.ALG_SINGLE_REDUCTION)
        d_x.zero_()
        m.solve_device(d_b.data_ptr(), d_x.data_ptr(), **sr)  # warm-up
        ms_sr = 0.0
        for _ in range(reps):
            d_x.zero_()
            torch.cuda.synchronize()
            e0.record(stream)
            r_sr = m.solve_device(d_b.data_ptr(), d_x.data_ptr(), **sr)
            e1.record(stream)
            torch.cuda.synchronize()
            ms_sr += e0.elapsed_time(e1) / reps
        it_sr = int(r_sr["iterations"])
        ib_sr = info["spmv_bytes"] + 68 * n
        out[name + "_single_reduction"] = {"solve_ms": ms_sr, "iterations": it_sr, "iteration_us": ms_sr * 1e3 / it_sr,
                                           "iteration_bytes": int(ib_sr),
                                           "iteration_gbs": ib_sr * it_sr / (ms_sr / 1e3) / 1e9,
                                           "iteration_frac": ib_sr * it_sr / (ms_sr / 1e3) / 1e9 / peak}
        del m
    return out


C4 = dict(systems=512, side_min=4, side_max=24, seed=512, rel_tol=1e-8, max_iter=20000)


def measure_c4(ctx, stream, peak):
    """512 independent systems (lattice side uniform in 4..24, own seeds and
    right-hand sides), tolerance 1e-8 with FP64 reductions, one batched
    solve (persistent kernels, graph loop, retire in place). Reports
    solves/s and the batch's algorithmic bytes (sum over systems of
    iterations x bytes per iteration) against the HBM peak."""
    import torch

    import wgpu_solver_backend_b200 as wsb

    rng = np.random.default_rng(C4["seed"])
    sides = rng.integers(C4["side_min"], C4["side_max"] + 1, C4["systems"])
    systems = [wsb.lattice_generate(int(sd), seed=50_000 + i) for i, sd in enumerate(sides)]
    mats = [wsb.Matrix.create(ctx, q["row_ptr"], q["col_idx"], q["values"], q["block_starts"]) for q in systems]
    kw = dict(max_iter=C4["max_iter"], rel_tol=C4["rel_tol"])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times, res = [], None
    for rep in range(3):  # the first is a warm-up
        bt = wsb.Batch(ctx)
        for m, q in zip(mats, systems):
            bt.add(m, q["b"], **kw)
        torch.cuda.synchronize()
        e0.record(stream)
        bt.solve()
        e1.record(stream)
        torch.cuda.synchronize()
        if rep:
            times.append(e0.elapsed_time(e1) / 1e3)
        res = [bt.result(i, q["n"])[1] for i, q in enumerate(systems)]
        del bt
    t = float(np.mean(times))
    iters = [int(r["iterations"]) for r in res]
    byts = sum(it * m.info["iteration_bytes"] for it, m in zip(iters, mats))
    return {"workload": f"{C4['systems']} systems, lattice side uniform {C4['side_min']}..{C4['side_max']} "
                        f"({sum(q['n'] for q in systems)} unknowns), rel tol 1e-8, FP64 reductions, one batch",
            "solves_per_s": C4["systems"] / t, "batch_ms": t * 1e3,
            "converged": sum(1 for r in res if r["rc"] == 0), "of": len(res),
            "iterations_min_median_max": [min(iters), int(np.median(iters)), max(iters)],
            "algorithmic_bytes": int(byts), "gbs": byts / t / 1e9, "frac": byts / t / 1e9 / peak}


def fcfs_latencies(arrivals_s, service_ms):
    """Latencies (ms) of requests served one at a time in arrival order, each
    starting when it has arrived and the previous one has finished."""
    t, out = 0.0, []
    for a, sv in zip(arrivals_s, service_ms):
        start = max(t, float(a))
        t = start + sv / 1e3
        out.append((t - float(a)) * 1e3)
    return out


def pinned_system(sysm):
    """The system's host arrays moved into page-locked (pinned) host memory,
    where requests come from in the end-to-end figure: host-to-device copies
    then run at DMA speed instead of through the driver's staging buffers."""
    import torch

    out = dict(sysm)
    for k in ("row_ptr", "col_idx", "values", "block_starts", "b"):
        a = np.ascontiguousarray(sysm[k])
        t = torch.empty(max(a.nbytes, 1), dtype=torch.uint8, pin_memory=True)
        v = t.numpy()[: a.nbytes].view(a.dtype)
        v[...] = a
        out[k] = v
        out["_pin_" + k] = t  # keeps the pinned buffer alive
    return out


def run_serve(args, world, rank, local):
    import torch

    import wgpu_solver_backend_b200 as wsb

    torch.cuda.set_device(local)
    ctx = wsb.GpuContext.create("auto", local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    reqs = serve_set(args.max_side)
    t_gen = time.perf_counter()
    pool = []
    for side, seed in reqs:
        sysm = pinned_system(serve_system(side, seed))
        sysm["side"], sysm["seed"] = side, seed
        pool.append(sysm)
    t_gen = time.perf_counter() - t_gen
    R = len(pool)
    n_total = sum(p["n"] for p in pool)
    kw = mixed_kw()
    srv = wsb.Server(ctx, memory_budget_bytes=120 << 30, iters_per_step=16, **SERVER_CFG)
    # Warm-up steps are full passes: besides the kernels and the graph, they
    # grow the server's stream-ordered memory pool to the set's size, which
    # the timed passes then reuse.
    for _ in range(args.warmup):
        served_pass(srv, pool)
    st0 = srv.stats()
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    mks, lats, results = [], [], []
    for _ in range(args.steps):
        mk, lat, res = served_pass(srv, pool)
        mks.append(mk)
        lats += lat
        results += res
    clk = clocks.stop()
    e2e_s = reduce_max(sum(mks), world)
    ok = sum(1 for r in results if r["rc"] == 0)
    failures = [{"path": "server", "side": pool[i % R]["side"], "seed": pool[i % R]["seed"], "rc": r["rc"],
                 "iterations": r["iterations"], "sweeps": r["refine_sweeps"], "relres": r["final_relres"],
                 "breakdown": r["breakdown_kind"]} for i, r in enumerate(results) if r["rc"] != 0]
    relres_max = max(r["final_relres"] for r in results)
    iters = [r["iterations"] for r in results[:R]]
    # Latency under open-loop Poisson arrivals at 70% of the measured capacity.
    lam = 0.7 * R / (sum(mks) / len(mks))
    rng = np.random.default_rng(11)
    arrivals = np.cumsum(rng.exponential(1.0 / lam, R)) - 0.0
    mk_p, lat_p, _ = served_pass(srv, pool, arrivals)
    # The tolerance mix of the serving configuration: each request's target
    # FP64 relative residual is 1e-6 or 1e-10 with probability 1/2.
    tmix = np.where(np.random.default_rng(13).random(R) < 0.5, 1e-6, 1e-10)
    mk_mix, lat_mix, res_mix = served_pass(srv, pool, targets=tmix)
    mix_ok = sum(1 for r, tg in zip(res_mix, tmix) if r["rc"] == 0 and r["final_relres"] <= tg)
    st = srv.stats()
    srv.close()
    # Where the server's time goes over the timed burst passes (and the two
    # passes after them): host preparation and copies in the uploader
    # threads, the scheduler's engine steps, admissions, retirements, idling.
    server_phases = {k: st[k] - st0[k] for k in ("busy_ms", "host_prep_ms", "upload_ms", "admit_ms", "retire_ms",
                                                 "sched_idle_ms", "steps")}
    # One burst pass of every other server configuration, for comparison.
    server_variants = {}
    for name, cfg in SERVER_VARIANTS.items():
        if cfg == SERVER_CFG:
            continue
        sv = wsb.Server(ctx, memory_budget_bytes=120 << 30, iters_per_step=16, **cfg)
        served_pass(sv, pool[: min(8, R)])
        mk_v, lat_v, _ = served_pass(sv, pool)
        sv.close()
        server_variants[name] = {"solves_per_s": R / mk_v, "burst_p99_ms": float(np.percentile(lat_v, 99))}
    # Resident batch: matrices already in HBM, one batched solve of the set.
    mats = [wsb.Matrix.create(ctx, p["row_ptr"], p["col_idx"], p["values"], p["block_starts"]) for p in pool]
    dev_s, batch_launches = 0.0, 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.steps):
        bt = wsb.Batch(ctx)
        for m, p in zip(mats, pool):
            bt.add(m, p["b"], **kw)
        torch.cuda.synchronize()
        e0.record(stream)
        bt.solve()
        e1.record(stream)
        torch.cuda.synchronize()
        dev_s += e0.elapsed_time(e1) / 1e3
        pass_bytes = 0
        for i, p in enumerate(pool):
            _, r = bt.result(i, p["n"])
            pass_bytes += int(r["iterations"]) * mats[i].info["iteration_bytes"]
            if i == 0:
                batch_launches += r["kernel_launches"]
            if r["rc"] != 0:
                failures.append({"path": "batch", "side": p["side"], "seed": p["seed"], "rc": r["rc"],
                                 "iterations": r["iterations"], "sweeps": r["refine_sweeps"],
                                 "relres": r["final_relres"], "breakdown": r["breakdown_kind"]})
        del bt
    pass_s = dev_s / args.steps
    dev_s = reduce_max(dev_s, world)
    # Plain baseline: the same requests one at a time (host arrays, matrix
    # upload and LU per request, then the solve), as a plain per-solve GPU PCG.
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain_lat = []
    for p in pool:
        t1 = time.perf_counter()
        m = wsb.Matrix.create(ctx, p["row_ptr"], p["col_idx"], p["values"], p["block_starts"])
        _, r = m.solve(p["b"], raise_on_error=False, **kw)
        if r["rc"] != 0:
            failures.append({"path": "plain", "side": p["side"], "seed": p["seed"], "rc": r["rc"],
                             "iterations": r["iterations"], "sweeps": r["refine_sweeps"],
                             "relres": r["final_relres"], "breakdown": r["breakdown_kind"]})
        del m
        plain_lat.append((time.perf_counter() - t1) * 1e3)
    plain_s = time.perf_counter() - t0
    # Plain resident: the matrices already in HBM, solved one after another.
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for m, p in zip(mats, pool):
        m.solve(p["b"], raise_on_error=False, **kw)
    torch.cuda.synchronize()
    plain_res_s = time.perf_counter() - t0
    # Latency at an arrival rate the plain path can sustain too (70 % of its
    # own capacity): the served latencies measured on a fresh server, and the
    # plain path's first-come-first-served latencies for the same arrivals,
    # replayed from its measured per-request times (one request at a time,
    # each starting when it has arrived and the previous one is done).
    lam2 = 0.7 * R / plain_s
    srv2 = wsb.Server(ctx, memory_budget_bytes=120 << 30, iters_per_step=16, **SERVER_CFG)
    served_pass(srv2, pool)  # warm-up: a full pass grows the server's memory pool
    # Two passes of arrivals (128 requests), so that p99 is not just the maximum.
    pool2 = pool + pool
    arrivals2 = np.cumsum(np.random.default_rng(12).exponential(1.0 / lam2, 2 * R))
    _, lat_p2, _ = served_pass(srv2, pool2, arrivals2)
    srv2.close()
    fcfs1 = fcfs_latencies(arrivals, plain_lat)
    fcfs2 = fcfs_latencies(arrivals2, plain_lat + plain_lat)
    # Dominant kernel (SpMV + p.Ap) on the largest system of the set.
    big = int(np.argmax([p["n"] for p in pool]))
    d_b = torch.from_numpy(pool[big]["b"]).cuda()
    torch.cuda.synchronize()
    kt = mats[big].kernel_times(d_b.data_ptr(), iterations=10)
    info = mats[big].info
    peak, peak_kind = peaks()
    serve_largest = kernel_block(kt, info, pool[big]["n"], peak)
    c2 = measure_c2(ctx, stream, peak)
    c4 = measure_c4(ctx, stream, peak)
    top = c2["bsr6"]["kernels"]["spmv"]
    e2e = replica_rate(world, args.steps * R, e2e_s)
    line = {
        "metric": METRIC, "value": replica_rate(world, args.steps * R, dev_s), "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_s / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 reductions + f64 refinement)",
        "data": "synthetic 6-DOF lattice systems, seeded",
        "config": {"workload": f"serve: {R} requests, lattice side log-uniform [4,64]{side_note(args)} "
                               f"(n 384..1,572,864, {n_total} unknowns in all), anisotropy 10^U(-2,2), true FP64 relres 1e-8 "
                               f"by FP64 refinement around FP32 PCG",
                   "step": "one pass over the request set", "value_path": "resident batch (wsb_batch)",
                   "e2e_path": "continuous-batching server (wsb_server, host arrays)",
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (%.1f GB of matrices)"
                   % (sum(m.info["device_bytes"] for m in mats) / 1e9)},
        "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": int(sum(
            4 * (len(p["row_ptr"]) + len(p["col_idx"]) + len(p["values"]) + len(p["block_starts"]) + 2 * p["n"])
            for p in pool)), "d2h_bytes_per_step": int(sum(4 * p["n"] for p in pool))},
        "latency_ms": {"p50": float(np.percentile(lat_p, 50)), "p99": float(np.percentile(lat_p, 99)),
                       "arrival_rate_per_s": lam, "burst_p50": float(np.percentile(lats, 50)),
                       "burst_p99": float(np.percentile(lats, 99)),
                       "plain_fcfs_same_arrivals_p50": float(np.percentile(fcfs1, 50)),
                       "plain_fcfs_same_arrivals_p99": float(np.percentile(fcfs1, 99)),
                       "at_plain_sustainable_rate": {
                           "arrival_rate_per_s": lam2, "served_p50": float(np.percentile(lat_p2, 50)),
                           "served_p99": float(np.percentile(lat_p2, 99)),
                           "plain_fcfs_p50": float(np.percentile(fcfs2, 50)),
                           "plain_fcfs_p99": float(np.percentile(fcfs2, 99))}},
        "plain_sequential": {"solves_per_s": R / plain_s, "resident_solves_per_s": R / plain_res_s,
                             "p50_ms": float(np.percentile(plain_lat, 50)), "p99_ms": float(np.percentile(plain_lat, 99))},
        "speedup_vs_plain": {"e2e": e2e / (world * R / plain_s), "resident": (world * args.steps * R / dev_s) /
                             (world * R / plain_res_s)},
        "results": {"ok": ok, "of": len(results), "max_final_relres": relres_max,
                    "iterations_min_median_max": [int(min(iters)), int(np.median(iters)), int(max(iters))]},
        "roofline": {"bound": "hbm", "kernel": "k_spmv_loop (SpMV + p.Ap) on the 3.07M-unknown 80^3 system, BSR6 "
                               "(the layout the library picks for it); CSR beside it in c2",
                     "achieved": top["gbs"], "peak": peak, "unit": "GB/s", "frac": top["frac"],
                     "peak_kind": peak_kind, **spmv_traffic(top["bytes"]),
                     "algorithmic_bytes_per_launch": top["bytes"], "launch_us": top["us"]},
        "resident_pass_hbm": {"algorithmic_bytes": pass_bytes, "gbs": pass_bytes / pass_s / 1e9,
                              "frac": pass_bytes / pass_s / 1e9 / peak,
                              "note": "sum over requests of PCG iterations x bytes per iteration; the FP64 "
                                      "refinement sweeps' residual and update passes are not counted"},
        "c2": c2,
        "c4": c4,
        "serve_largest_system_kernels": serve_largest,
        "serve_tolerance_mix": {"targets": "FP64 relres 1e-6 or 1e-10, p = 1/2 each (seeded)",
                                "solves_per_s": R / mk_mix, "met_target": mix_ok, "of": R,
                                "p50_ms": float(np.percentile(lat_mix, 50)), "p99_ms": float(np.percentile(lat_mix, 99)),
                                "path": "continuous-batching server, burst, host arrays"},
        "server": {"steps": st["steps"], "device_bytes_peak": st["device_bytes_peak"], "config": SERVER_CFG,
                   "phases_ms": server_phases, "other_configs_one_pass": server_variants},
        "failures": failures[:20],
        "host_generate_s": t_gen,
        "gpu_launches": batch_launches,
        "server_kernel_launches_all_passes": st["kernel_launches"],
        "clocks": clk,
    }
    if rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_baseline_serve(pool)
    return line


def run_reference_serve(args, world, rank, local):
    """The reference arm: the reference's own CPU algorithm (the oracle's
    restatement, no product code loaded) solving the serving request set
    completely on the host cores. Warm-up steps solve the smallest request;
    the timed steps solve contiguous groups of requests that together cover
    the set once."""
    import oracle

    pool = reference_pool(args.max_side)
    R = len(pool)
    smallest = int(np.argmin([p["n"] for p in pool]))
    for _ in range(args.warmup):
        reference_solve_requests(pool, [smallest])
    total_s, lu_s, solved, results = 0.0, 0.0, 0, []
    for g in step_groups(R, args.steps):
        dt, dlu, res = reference_solve_requests(pool, g)
        total_s += dt
        lu_s += dlu
        solved += len(g)
        results += res
    v = solved / total_s
    iters = [r["iterations"] for r in results]
    conv = sum(1 for r in results if r["status"] == oracle.OK)
    sample = (f"complete solves (LU + PCG) of {solved} requests ({len(set(sum(step_groups(R, args.steps), [])))} "
              f"distinct of {R}) in {args.steps} steps, {total_s:.1f} s ({lu_s:.2f} s LU), "
              f"{oracle.num_threads()} threads; stop: {REFERENCE_STOP}")
    return {"metric": METRIC, "impl": "reference", "value": v, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_s / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic 6-DOF lattice systems, seeded",
            "config": {"workload": f"serve: {R} requests, lattice side log-uniform [4,64]{side_note(args)}, "
                                   f"anisotropy 10^U(-2,2), relres 1e-8 on the reference's FP32 recursive residual",
                       "step": "complete solves of a contiguous group of the requests; the steps cover the set once",
                       "stop_rule": REFERENCE_STOP},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": oracle.num_threads(), "kind": "port",
                             "sample": sample},
            "repo_libraries_loaded": repo_libraries(),
            "reference_results": {"converged": conv, "of": len(results),
                                  "iterations_min_median_max": [int(min(iters)), int(np.median(iters)),
                                                                int(max(iters))]},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_kernels(args, world, rank, local):
    """Per-kernel device times of the three loop kernels on one lattice system
    (the small case used for profiler captures)."""
    import torch

    import wgpu_solver_backend_b200 as wsb

    torch.cuda.set_device(local)
    ctx = wsb.GpuContext.create("auto", local)
    s = wsb.lattice_generate(args.side, seed=PLAIN["seed"])
    m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"],
                          layout=wsb.LAYOUT_CSR if args.layout == "csr" else wsb.LAYOUT_AUTO)
    d_b = torch.from_numpy(s["b"]).cuda()
    torch.cuda.synchronize()
    try:
        kt = m.kernel_times(d_b.data_ptr(), iterations=args.iters)
    except Exception as e:  # report instead of a bogus timing
        return {"workload": f"kernels: {args.side}^3", "error": str(e)}
    info = m.info
    peak, kind = peaks()
    out = {"workload": f"kernels: {args.side}^3 lattice, n={s['n']}, layout {args.layout}", "iterations": args.iters,
           "matrix_bytes": info["device_bytes"]}
    for k, b in (("spmv", info["spmv_bytes"]), ("update", 28 * s["n"] + 144 * info["num_blocks"]),
                 ("pupdate", 12 * s["n"])):
        ms = kt[k + "_ms"]
        out[k] = {"us": ms * 1e3, "bytes": b, "gbs": b / ms / 1e6, "frac": b / ms / 1e6 / peak}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="serve", choices=["serve", "plain80", "kernels"])
    ap.add_argument("--side", type=int, default=56, help="kernels workload: lattice side")
    ap.add_argument("--iters", type=int, default=5, help="kernels workload: timed iterations")
    ap.add_argument("--layout", default="auto", choices=["auto", "csr"])
    ap.add_argument("--max-side", type=int, default=SERVE["side_max"],
                    help="serve workload: keep only the requests of lattice side <= this (default: all)")
    args = ap.parse_args()
    if args.workload == "kernels":
        world, rank, local = dist_setup()
        print(json.dumps(run_kernels(args, world, rank, local)), flush=True)
        return
    world, rank, local = dist_setup()
    if args.impl == "reference":
        if rank != 0:
            return
        line = (run_reference_serve if args.workload == "serve" else run_reference_plain)(args, world, rank, local)
        print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    line = (run_serve if args.workload == "serve" else run_plain)(args, world, rank, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()

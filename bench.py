#!/usr/bin/env python
"""Benchmark: triangle counting on R-MAT scale 24 (TC edges/s) on B200.

Workload (the single-GPU configuration the headline metric is quoted on):
R-MAT scale 24, edge factor 16, a/b/c/d = .57/.19/.19/.05, seeded,
symmetrised, self-loops and duplicates removed, oriented low degree -> high
degree (ties by id), int32 CSR, generated on the device (synthetic: the
reference's graph datasets are not available).

One step = the hot path over the whole graph: build the per-vertex bucketed
hash tables (hierarchical hash, alpha 0.2, 5 slots per bucket) emitting the
hash-ordered rows in the same pass, then count triangles by probing.
  value : TC edges/s with the CSR resident in HBM (device-timed, max over
          ranks), inputs (6+ GB of tables and rows) far larger than L2.
  e2e   : the same through the C ABI from pinned HOST buffers, with the
          H2D copy of the CSR and the D2H read of the count inside the timed
          region.
  roofline: the probe kernel (tc_kernel) against measured HBM bandwidth,
          with the algorithmic bytes sum_e (8*min(d+u, d+v) + 36) + 4(n+1).
  cpu_baseline: the CPU oracle (sorted-row merge, all host threads) on a
          bounded vertex sample of the same graph, rank 0 at N=1.

`--impl reference` times the reference path's CPU implementation -- the
reference ships none, so the CPU port of its algorithm (the oracle) --
on the same workload, with all host threads; rank 0 only.

Multi-GPU: the path does not exchange data; with N ranks every rank runs
its own replica of the workload (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TC edges/sec (R-MAT scale 24, table build + hash-probe count)"
UNIT = "edges/s"


def rmat_seed(scale: int) -> int:
    """0x5EED00SS, SS = the scale's decimal digits (scale 24 -> 0x5EED0024)."""
    return int(f"0x5EED00{scale:02d}", 16)


def oracle_count(scale: int, edge_factor: int):
    """The CPU oracle's exact triangle count of the seeded graph of this
    scale (tests/golden/tc_counts.json), or None if it was not computed."""
    try:
        rec = json.load(open(os.path.join(ROOT, "tests", "golden", "tc_counts.json")))
        if rec.get("edge_factor") != edge_factor:
            return None
        c = rec["counts"].get(str(scale))
        return c if c and int(c["seed"], 16) == rmat_seed(scale) else None
    except (OSError, ValueError, KeyError):
        return None


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the bounded CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--probe-rounds", type=int, default=0, choices=[0, 2, 4, 8])
    ap.add_argument("--warp-pair-min", type=int, default=0)
    ap.add_argument("--probe-variant", type=int, default=-1, choices=[-1, 0, 1],
                    help="-1 library default; 0 pipelined; 1 lean whole-warp pair loop")
    ap.add_argument("--tc-method", type=int, default=0, choices=[0, 1, 2, 3],
                    help="0 default (owner-grouped), 1 edge-flattened, 2 vertex-staged, "
                         "3 owner-grouped (probed tables staged in shared memory)")
    ap.add_argument("--alpha", type=float, default=0.2,
                    help="TC table load factor (with --no-autotune)")
    ap.add_argument("--bucket", type=int, default=5,
                    help="TC table slots per bucket (with --no-autotune)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep --alpha/--bucket and the library's probe knobs")
    ap.add_argument("--workload", default="tc",
                    choices=["tc", "sss-join", "ir-serve", "mixed-serve", "tc-batch", "pattern"],
                    help="tc: TC on R-MAT (default); sss-join: batched Jaccard self-join; "
                         "ir-serve: served conjunctive IR; mixed-serve: served mixed "
                         "intersections on R-MAT scale 22")
    # sss-join
    ap.add_argument("--sets", type=int, default=2_000_000)
    ap.add_argument("--size-hi", type=int, default=1024)
    ap.add_argument("--dup-frac", type=float, default=0.2)
    # serving
    ap.add_argument("--terms", type=int, default=1_000_000)
    ap.add_argument("--docs", type=int, default=20_000_000)
    ap.add_argument("--df-max", type=int, default=10_000_000)
    ap.add_argument("--requests", type=int, default=20000,
                    help="requests in the capacity burst of a serving workload")
    ap.add_argument("--serve-seconds", type=float, default=2.0,
                    help="length of each Poisson arrival phase")
    ap.add_argument("--streams", type=int, default=4)
    ap.add_argument("--max-batch", type=int, default=1024)
    ap.add_argument("--graphs", type=int, default=1024,
                    help="tc-batch: number of disjoint R-MAT graphs (scales 8..12)")
    ap.add_argument("--pattern-scale", type=int, default=14,
                    help="pattern: R-MAT scale of the graphs the patterns are counted on")
    ap.add_argument("--max-batch-cost", type=int, default=1 << 22,
                    help="served forms: estimated probes per batch at most (0 = no limit)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ------------------------------------------------------- rank aggregation --

def max_over_ranks(vals, world, device="cuda"):
    """Element-wise max of per-rank timings (every rank calls it in the same
    order; identity for one rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(vals), dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def weak_value(units_per_rank, world, ms):
    """Whole-job throughput of `world` replicas that each processed
    units_per_rank units, timed as the slowest rank's `ms`."""
    return world * units_per_rank / (ms / 1e3)


# ----------------------------------------------------------- clock sampler --

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p is not None:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        rows = []
        for line in (getattr(self, "out", "") or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append(dict(sm=float(f[1]), smax=float(f[2]), hw=f[5], hwt=f[6],
                                 swt=f[7], pcap=f[8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        reasons = set()
        for r in rows:
            if r["hw"].lower() == "active":
                reasons.add("hw_slowdown")
            if r["hwt"].lower() == "active":
                reasons.add("hw_thermal_slowdown")
            if r["swt"].lower() == "active":
                reasons.add("sw_thermal_slowdown")
            if r["pcap"].lower() == "active":
                reasons.add("sw_power_cap")
        return {"sm_mhz": statistics.median(r["sm"] for r in rows),
                "sm_max_mhz": max(r["smax"] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------ CPU legs -----

def cpu_sample_rate(off: np.ndarray, cols: np.ndarray, seconds: float, threads: int):
    """Oracle merge-TC over evenly spread vertex blocks until ~`seconds` of
    wall time; returns (edges/s, edges, vertices, wall)."""
    import oracle
    n = off.size - 1
    blocks = 64
    bsz = max(1, n // (blocks * 16))
    starts = [(i * n) // blocks for i in range(blocks)]
    edges = verts = 0
    t0 = time.perf_counter()
    rounds = 0
    while True:
        for s in starts:
            v0 = s + rounds * bsz
            v1 = min(v0 + bsz, n)
            if v0 >= n:
                continue
            oracle.tc_merge_range(off, cols, v0, v1, threads)
            edges += int(off[v1] - off[v0])
            verts += v1 - v0
        rounds += 1
        el = time.perf_counter() - t0
        if el >= seconds or rounds * bsz * blocks >= n:
            break
    return edges / el, edges, verts, el


# ------------------------------------------------------------ our arm -------

def run_ours(a, rank, world, local):
    import torch
    import torch.distributed as dist
    from reset_b200 import api, _lib

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    L = _lib.load()
    if a.probe_rounds or a.warp_pair_min or a.probe_variant >= 0:
        api.set_tuning(probe_rounds=a.probe_rounds or None,
                       warp_pair_min=a.warp_pair_min or None,
                       probe_variant=a.probe_variant if a.probe_variant >= 0 else None)

    off, cols = api.gen_rmat(a.scale, a.edge_factor, rmat_seed(a.scale))
    n, m = off.numel() - 1, cols.numel()
    deg = (off[1:] - off[:-1])
    src = torch.repeat_interleave(torch.arange(n, device="cuda", dtype=torch.int64), deg.long())
    s_e = torch.minimum(deg[src], deg[cols.long()]).to(torch.int64)
    sum_s = int(s_e.sum().item())
    del src, s_e
    alg_bytes = 8 * sum_s + 36 * m + 4 * (n + 1)
    h_off = off.cpu().pin_memory()
    h_cols = cols.cpu().pin_memory()

    # table and probe parameters: the autotuner ranks the reference grid with
    # its model, then builds + counts the whole graph with the best points
    # (and the reference default 0.2 / 5) on this GPU; untimed set-up
    tuned = None
    if not a.no_autotune and a.probe_rounds == 0 and a.warp_pair_min == 0 and a.probe_variant < 0:
        from reset_b200 import autotune

        def measure(hp):
            api.set_tuning(probe_rounds=hp.probe_rounds, warp_pair_min=hp.warp_pair_min,
                           probe_variant=1)

            def once():
                t = api.Table(off, cols, alpha=hp.alpha, bucket=hp.b, hierarchical=True,
                              hash_order=True)
                api.tc_count_async(t, off, t.hash_order, method=a.tc_method)
                t.free()
            once()
            return autotune.timed(once, reps=2)

        deg = (off[1:] - off[:-1]).cpu().numpy()
        samp = deg[np.random.default_rng(1).integers(0, deg.size, min(deg.size, 200_000))]
        # the probe-round and warp-pair knobs steer the edge-flattened kernel
        # only; the owner-grouped count is tuned over (alpha, b) alone
        edge = a.tc_method == 1
        hp = autotune.solve("tc", samp, measure=measure, measure_top=3,
                            rounds=(4, 8) if edge else (),
                            warp_pair_mins=(32, 64, 128) if edge else (), cache=None,
                            always=((0.2, 5), (0.25, 1), (0.4, 2), (0.5, 1), (0.5, 2)))
        api.set_tuning(probe_rounds=hp.probe_rounds, warp_pair_min=hp.warp_pair_min,
                       probe_variant=1)
        a.alpha, a.bucket = hp.alpha, hp.b
        tuned = {"alpha": hp.alpha, "bucket": hp.b, "probe_rounds": hp.probe_rounds,
                 "warp_pair_min": hp.warp_pair_min, "measured_ms": hp.measured_ms}
        torch.cuda.synchronize()

    # A step's build and count run back to back on one stream: both fill
    # every SM, and a build overlapped with the previous count only slowed
    # both.  e2e steps copy their CSR on a copy stream, so step k+1's H2D
    # overlaps step k's kernels.  The build's one sizing sync waits for the
    # previous count; the free is stream-ordered.
    stream = torch.cuda.current_stream()
    s_copy = torch.cuda.Stream()
    probe_ms = []
    counts = []
    in_flight = []   # done events of steps not yet known finished

    # e2e inputs land in two device buffers used in turn; a buffer is
    # rewritten only after the step that last read it has finished
    e2e_bufs = [(torch.empty_like(off), torch.empty_like(cols)) for _ in range(2)]
    buf_free = [None, None]
    n_e2e = [0]

    def step(record=False, off_d=off, cols_d=cols, inputs_from=None, out=None):
        # at most two steps' tables alive: the memory pool holds the same
        # working set in warm-up and in the timed region (no growth there)
        while len(in_flight) >= 2:
            in_flight.pop(0).synchronize()
        buf = None
        if inputs_from is not None:   # e2e: this step's CSR from pinned host memory
            buf = n_e2e[0] % 2
            n_e2e[0] += 1
            off_d, cols_d = e2e_bufs[buf]
            with torch.cuda.stream(s_copy):
                if buf_free[buf] is not None:
                    s_copy.wait_event(buf_free[buf])
                off_d.copy_(inputs_from[0], non_blocking=True)
                cols_d.copy_(inputs_from[1], non_blocking=True)
                copied = torch.cuda.Event()
                copied.record(s_copy)
            stream.wait_event(copied)
        t = api.Table(off_d, cols_d, alpha=a.alpha, bucket=a.bucket, hierarchical=True,
                      hash_order=True, stream=stream)
        if record:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        cnt = api.tc_count_async(t, off_d, t.hash_order, method=a.tc_method, stream=stream)
        if record:
            e1.record(stream)
            probe_ms.append((e0, e1))
        if out is not None:
            out.copy_(cnt, non_blocking=True)     # D2H of the step's result
        counts.append(cnt)
        t.free_async(stream)
        done = torch.cuda.Event()
        done.record(stream)
        in_flight.append(done)
        if buf is not None:
            buf_free[buf] = done

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    expect = int(counts[-1].item())
    counts.clear()
    # parity, outside the timed region: the exact count the CPU oracle
    # computed on the same seeded graph
    pinned = oracle_count(a.scale, a.edge_factor)
    if pinned is not None:
        assert pinned["vertices"] == n and pinned["oriented_edges"] == m, "graph differs"
        assert expect == pinned["triangles"], \
            f"triangle count {expect} != oracle {pinned['triangles']}"
    parity = ("equals the CPU oracle's count of the same graph (tests/golden/tc_counts.json)"
              if pinned is not None else "unpinned at this scale (no oracle count on file)")

    l0 = L.reset_kernel_launches()
    barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(a.steps):
            step(record=True)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    launches = L.reset_kernel_launches() - l0
    ms = ev0.elapsed_time(ev1)
    for c in counts:
        assert int(c.item()) == expect, "triangle count changed between steps"
    counts.clear()
    probe = [e0.elapsed_time(e1) for e0, e1 in probe_ms]
    probe_avg = sum(probe) / len(probe)

    # e2e: every step copies its CSR from pinned host memory, builds, counts
    # and copies the count back to pinned host memory (same pipelining)
    h_counts = torch.zeros(a.warmup + a.steps, dtype=torch.int64).pin_memory()
    for i in range(a.warmup):
        step(inputs_from=(h_off, h_cols), out=h_counts[i:i + 1])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(a.warmup, a.warmup + a.steps):
        step(inputs_from=(h_off, h_cols), out=h_counts[i:i + 1])
    torch.cuda.synchronize()
    e2e_step = (time.perf_counter() - t0) * 1e3 / a.steps
    assert all(int(x) == expect for x in h_counts.tolist()), "e2e count differs"
    counts.clear()

    ms, e2e_step, probe_avg = max_over_ranks([ms, e2e_step, probe_avg], world)
    step_ms = ms / a.steps
    value = weak_value(m, world, step_ms)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    achieved = alg_bytes / (probe_avg / 1e3) / 1e9
    # DRAM bytes per launch of the count kernel from a committed ncu record
    # of the same method, scale and slots per bucket (alpha within 0.05)
    traffic, traffic_note = None, None
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "tc_owner_kernel_traffic.json")))
        if a.tc_method in (0, 3):
            for rec in prof["records"]:
                if (rec["scale"] == a.scale and abs(rec["alpha"] - a.alpha) <= 0.05 + 1e-9
                        and rec["bucket"] == a.bucket):
                    traffic = rec["dram_bytes_per_launch"]
                    traffic_note = rec["how"]
    except Exception:
        pass

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic (seeded R-MAT generated on device)",
        "config": {"workload": f"tc_rmat_s{a.scale}_ef{a.edge_factor}",
                   "scale": a.scale, "edge_factor": a.edge_factor, "vertices": n,
                   "oriented_edges": m, "triangles": expect, "parity": parity,
                   "probes": sum_s,
                   "alpha": a.alpha, "bucket": a.bucket, "hash": "hierarchical",
                   "tc_method": ["owner-grouped", "edge-flattened", "vertex-staged",
                                 "owner-grouped"][a.tc_method],
                   "tuning": api.get_tuning(), "autotuned": tuned,
                   "vertex_ids": "relabeled by a seeded bijection (Graph500 convention)",
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (tables+rows > 6 GB); no flush"},
        "e2e": {"value": weak_value(m, world, e2e_step), "unit": UNIT,
                "h2d_bytes_per_step": 4 * (n + 1) + 4 * m, "d2h_bytes_per_step": 8,
                "ms_per_step": e2e_step},
        "probe_only": {"value": weak_value(m, world, probe_avg), "unit": UNIT,
                       "ms_per_launch": probe_avg},
        "roofline": {"bound": "hbm",
                     "kernel": ["tc_owner_kernel + its grouping passes", "tc_kernel",
                                "tc_staged_kernel",
                                "tc_owner_kernel + its grouping passes"][a.tc_method],
                     "timed": "the whole reset_tc_count_ex call (CUDA events on its stream)",
                     "achieved": achieved,
                     "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": peak_src, "traffic": traffic,
                     "traffic_source": traffic_note,
                     "algorithmic_bytes_per_launch": alg_bytes},
        "gpu_launches": launches,
    }
    line["clocks"] = clk.summary()
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        h_o, h_c = h_off.numpy(), h_cols.numpy()
        thr = host_threads()
        rate, edges, verts, wall = cpu_sample_rate(h_o, h_c, a.cpu_seconds, thr)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": thr, "kind": "port",
                                "sample": f"oracle sorted-row merge TC over {verts} vertices "
                                          f"({edges} oriented edges) in 64 evenly spread "
                                          f"blocks of the same graph, {wall:.1f} s wall"}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------ reference arm ------

def run_reference(a, rank, world):
    if rank != 0:
        return
    import oracle
    thr = host_threads()
    t0 = time.perf_counter()
    off, cols = oracle.rmat_graph(a.scale, a.edge_factor, rmat_seed(a.scale), oriented=True)
    gen_s = time.perf_counter() - t0
    rates = []
    info = None
    for i in range(a.warmup + a.steps):
        r = cpu_sample_rate(off, cols, max(2.0, a.cpu_seconds / 3), thr)
        if i >= a.warmup:
            rates.append(r[0])
            info = r
    v = statistics.mean(rates)
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": info[3] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded R-MAT, CPU generator)", "impl": "reference",
        "config": {"workload": f"tc_rmat_s{a.scale}_ef{a.edge_factor}", "scale": a.scale,
                   "edge_factor": a.edge_factor, "vertices": int(off.size - 1),
                   "oriented_edges": int(cols.size), "parallelism": "cpu",
                   "note": "the reference has no CPU implementation of this path; this is "
                           "the CPU port of its algorithm (oracle, sorted-row merge)"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": thr, "kind": "port",
                         "sample": f"{info[2]} vertices / {info[1]} edges per step in 64 "
                                   f"evenly spread blocks; graph generated in {gen_s:.1f} s"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    rank, world, local = dist_env()
    if a.workload != "tc":
        import bench_serving
        if a.impl == "reference":
            bench_serving.run_reference(a, rank, world)
        else:
            bench_serving.run_ours(a, rank, world, local)
        return
    if a.impl == "reference":
        run_reference(a, rank, world)
    else:
        run_ours(a, rank, world, local)


if __name__ == "__main__":
    main()

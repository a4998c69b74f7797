"""Workloads of bench.py beyond the default triangle count (imported by
bench.py for --workload sss-join | ir-serve | mixed-serve | tc-batch |
pattern; same JSON-line contract, same timing rules).

  sss-join    Batched Jaccard self-join (threshold 7/10, exact integer rule)
              over seeded token sets: prefix-filter candidates, then every
              candidate decided by one CUDA-graph replay of the persistent
              pair kernel (reset_batch_*), table parameters picked by the
              autotuner.  Beside it, the plain per-call form (reset_sss once
              per query set) on the same pairs.
  ir-serve    Conjunctive retrieval served with continuous batching over a
              resident inverted index; capacity, then Poisson arrivals at
              swept rates (p50/p99 latency), and the unbatched per-call form.
  mixed-serve A served mix on R-MAT scale 22: per-vertex triangle jobs,
              three-way (4-clique candidate) intersections and raw pairs
              with sizes log-uniform over 2^4..2^20.
  tc-batch    Many small graphs counted in one batched call.
  pattern     SMOG's query patterns Q0..Q8 (subgraph matching) on R-MAT.
Inputs are synthetic (seeded generators with the shapes of the reference's
datasets, which are not available).
"""
from __future__ import annotations

import json
import os
import statistics
import time

import numpy as np

import bench as B

SEED_SSS = 0x5EED0033
SEED_IR = 0x5EED0044
SEED_MIX = 0x5EED0022


def _setup(local, world):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return torch


def _maxr(vals, world):
    return B.max_over_ranks(vals, world)


def _finish(line, rank, world):
    import torch.distributed as dist
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def _peak():
    try:
        pk = json.load(open(os.path.join(B.ROOT, "MEASURED_PEAKS.json")))
        return pk["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def _pct(xs, q):
    if not xs:
        return None
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(q * len(xs)))]


# =============================================================== sss-join ==

def sss_join_ours(a, rank, world, local):
    torch = _setup(local, world)
    from reset_b200 import api, autotune, _lib
    L = _lib.load()
    ulog, num, den = 24, 7, 10
    off, tok = api.gen_token_sets(a.sets, ulog, 1.2, 8, a.size_hi, seed=SEED_SSS,
                                  dup_frac=a.dup_frac, keep_min=0.75)
    n, m = off.numel() - 1, tok.numel()
    sizes = off[1:] - off[:-1]
    pa, pb = api.prefix_candidates(off, tok, ulog, num, den)
    P = pa.numel()
    smin = torch.minimum(sizes[pa.long()], sizes[pb.long()]).long()
    probes = int(smin.sum().item())
    del smin
    alg_bytes = 8 * probes + 41 * P  # keys + first slot, ids/offsets, flag + size out

    # autotune (alpha, b, probe knobs) on a sample of the candidates
    samp = min(P, 2_000_000)
    sa, sb = pa[:samp].clone(), pb[:samp].clone()

    def measure(hp):
        api.set_tuning(probe_rounds=hp.probe_rounds, warp_pair_min=hp.warp_pair_min)
        t = api.Table(off, tok, alpha=hp.alpha, bucket=hp.b)
        bt = api.Batch(t, tok, capacity=max(1, samp), num=num, den=den, decisions_only=True)
        bt.pair_a[:samp].copy_(sa)
        bt.pair_b[:samp].copy_(sb)
        ms = autotune.timed(lambda: bt.run(samp), reps=3)
        bt.close()
        t.free()
        return ms

    hp = autotune.solve("sss", sizes.cpu().numpy(), measure=measure, measure_top=3,
                        rounds=(8,), cache=None) if samp else autotune.HyperParams()
    api.set_tuning(probe_rounds=hp.probe_rounds, warp_pair_min=hp.warp_pair_min)
    del sa, sb

    t = api.Table(off, tok, alpha=hp.alpha, bucket=hp.b)      # resident index
    cap = max(1, P)
    # the join needs decisions only: pairs stop as soon as they are settled
    bt = api.Batch(t, tok, capacity=cap, num=num, den=den, decisions_only=True)
    stream = torch.cuda.current_stream()
    results = []
    rep_ev = []

    def step(record=False):
        ca, cb = api.prefix_candidates(off, tok, ulog, num, den)
        k = ca.numel()
        bt.pair_a[:k].copy_(ca)
        bt.pair_b[:k].copy_(cb)
        if record:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        bt.run(k)
        if record:
            e1.record(stream)
            rep_ev.append((e0, e1))
        keep = bt.flags[:k].nonzero().squeeze(1)
        results.append((ca[keep], cb[keep]))

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    want = results[-1][0].numel()
    results.clear()
    l0 = L.reset_kernel_launches()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with B.Clocks(local) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(a.steps):
            step(record=True)
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = L.reset_kernel_launches() - l0
    ms = ev0.elapsed_time(ev1)
    for ra, _ in results:
        assert ra.numel() == want
    rep = statistics.mean(e0.elapsed_time(e1) for e0, e1 in rep_ev)
    # the same candidates decided with full intersection sizes (every key
    # probed): the launch the roofline's algorithmic bytes describe
    bfull = api.Batch(t, tok, capacity=cap, num=num, den=den, owner_grouped=True)
    bfull.pair_a[:P].copy_(pa)
    bfull.pair_b[:P].copy_(pb)
    full_ms = []
    for i in range(2 + a.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bfull.run(P)
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= 2:
            full_ms.append(e0.elapsed_time(e1))
    assert torch.equal(bfull.flags[:P], bt.flags[:P])   # same decisions
    full = statistics.mean(full_ms)
    bfull.close()

    # e2e: pinned host token sets -> index + candidates + decisions -> host pair list
    h_off, h_tok = off.cpu().pin_memory(), tok.cpu().pin_memory()
    e2e = []
    out_bytes = 0
    for i in range(a.warmup + a.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d_off = h_off.to("cuda", non_blocking=True)
        d_tok = h_tok.to("cuda", non_blocking=True)
        tt = api.Table(d_off, d_tok, alpha=hp.alpha, bucket=hp.b)
        ca, cb = api.prefix_candidates(d_off, d_tok, ulog, num, den)
        b2 = api.Batch(tt, d_tok, capacity=max(1, ca.numel()), num=num, den=den,
                       decisions_only=True)
        f, _ = b2(ca, cb)
        keep = f.nonzero().squeeze(1)
        pairs = torch.stack([ca[keep], cb[keep]], 1).cpu()
        el = (time.perf_counter() - t0) * 1e3
        out_bytes = pairs.numel() * 4
        b2.close()
        tt.free()
        assert pairs.shape[0] == want
        if i >= a.warmup:
            e2e.append(el)
    e2e_ms = statistics.mean(e2e)

    # plain per-call form: one reset_sss call per query set (its candidates)
    ha = pa.cpu().numpy()
    starts = np.flatnonzero(np.r_[True, ha[1:] != ha[:-1]])
    ends = np.r_[starts[1:], ha.size]
    pick = np.linspace(0, starts.size - 1, min(2000, starts.size)).astype(np.int64) if starts.size else []
    done = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for q in pick:
        s0, s1 = int(starts[q]), int(ends[q])
        f, _ = api.sss(t, off, tok, pa[s0:s1], pb[s0:s1], num, den)
        f.sum().item()
        done += s1 - s0
    plain_s = time.perf_counter() - t0
    plain_rate = done / plain_s if plain_s > 0 else None

    step_ms, e2e_ms, rep, full = _maxr([ms / a.steps, e2e_ms, rep, full], world)
    hbm, src = _peak()
    achieved = alg_bytes / (full / 1e3) / 1e9
    line = {
        "metric": "set-intersections/sec (Jaccard 0.7 self-join: prefix-filter candidates "
                  "decided by one graph-captured batch launch)",
        "value": world * P / (step_ms / 1e3), "unit": "intersections/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded token sets generated on device, planted near-duplicates)",
        "config": {"workload": f"sss_join_{n}_sets", "sets": n, "tokens": m,
                   "universe": 1 << ulog, "size_law": f"Zipf(1.2) on [8, {a.size_hi}]",
                   "token_law": "Zipf(1.0) by frequency rank", "dup_frac": a.dup_frac,
                   "threshold": f"{num}/{den} (10*I >= 7*U)", "candidates": P,
                   "similar_pairs": want, "probes": probes,
                   "autotuned": {"alpha": hp.alpha, "bucket": hp.b,
                                 "probe_rounds": hp.probe_rounds,
                                 "warp_pair_min": hp.warp_pair_min},
                   "step": "prefix-filter candidates + decisions-only batch replay + "
                           "pair-list compaction (index resident)",
                   "parallelism": f"replicas x{world}",
                   "l2": "token sets + tables larger than L2; no flush"},
        "batch_launch": {"value": world * P / (rep / 1e3), "unit": "intersections/s",
                         "ms_per_launch": rep, "mode": "decisions only (early exit)"},
        "batch_launch_full_sizes": {"value": world * P / (full / 1e3),
                                    "unit": "intersections/s", "ms_per_launch": full,
                                    "mode": "every key probed, |A ∩ B| written; pairs "
                                            "grouped by the larger set, its table staged "
                                            "in shared memory"},
        "plain_per_call": {"value": plain_rate, "unit": "intersections/s",
                           "calls": len(pick), "pairs": done,
                           "note": "reset_sss once per query set over its candidates"},
        "e2e": {"value": world * P / (e2e_ms / 1e3), "unit": "intersections/s",
                "h2d_bytes_per_step": 4 * (n + 1) + 4 * m, "d2h_bytes_per_step": out_bytes,
                "ms_per_step": e2e_ms,
                "note": "host token sets in; index build, candidates, decisions; pair list out"},
        "roofline": {"bound": "hbm",
                     "kernel": "owner-grouped pair decisions (batch replay, full sizes)",
                     "achieved": achieved,
                     "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_source": src,
                     "traffic": None, "algorithmic_bytes_per_launch": alg_bytes},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = _sss_cpu(off.cpu().numpy(), tok.cpu().numpy(),
                                        pa.cpu().numpy(), pb.cpu().numpy(), a.cpu_seconds,
                                        bt.flags[:P].cpu().numpy())
        line["config"]["pairs_checked_exactly"] = line["cpu_baseline"].pop("checked")
    bt.close()
    _finish(line, rank, world)


def _sss_cpu(off, tok, pa, pb, seconds, flags=None):
    """Oracle hash-probe decisions (one thread) on a bounded sample; with
    the GPU's decisions of the same candidates, every sampled one must be
    equal (returned as "checked")."""
    import oracle
    ot = oracle.Table(off, tok, hier=1)
    done, chunk = 0, 20000
    t0 = time.perf_counter()
    while done < pa.size and time.perf_counter() - t0 < seconds:
        f, _ = oracle.sss(ot, pa[done:done + chunk], pb[done:done + chunk], mode=1,
                          num=7, den=10)
        if flags is not None:
            assert np.array_equal(f, flags[done:done + f.size]), "self-join decision differs"
        done += min(chunk, pa.size - done)
    el = time.perf_counter() - t0
    return {"value": done / el, "unit": "intersections/s", "cores": 1, "kind": "port",
            "sample": f"first {done} candidate pairs decided by the oracle's hash probe "
                      f"in {el:.1f} s (table build not timed)",
            "checked": done if flags is not None else 0}


# ================================================================ serving ==

def _ir_queries(df, nq, rng):
    """2-6 terms drawn with probability proportional to df, deduped, ordered
    by df ascending (ties by id), as the reference's preprocessing orders a
    query (rarest term first)."""
    p = df / df.sum()
    ks = rng.integers(2, 7, nq)
    draws = rng.choice(df.size, size=int(ks.sum()), p=p)
    out, i = [], 0
    for k in ks:
        ts = np.unique(draws[i:i + k])
        i += k
        order = np.lexsort((ts, df[ts]))
        out.append(ts[order].astype(np.int32))
    return out


def _serve_phase(srv, reqs, submit, rate=None, seconds=None, rng=None, window=4096):
    """Submits `reqs` closed-loop with at most `window` outstanding (rate
    None: capacity), or Poisson at `rate`/s for `seconds`; waits for all;
    returns (results, wall seconds, list of requests used)."""
    from collections import deque
    from reset_b200.server import now_ns
    used = []
    t0 = time.perf_counter()
    if rate is None:
        res = []
        pend = deque()
        for q in reqs:
            if len(pend) >= window:
                res.append(srv.wait(pend.popleft()))
            pend.append(submit(q, 0))
            used.append(q)
        while pend:
            res.append(srv.wait(pend.popleft()))
        return res, time.perf_counter() - t0, used
    # Poisson arrivals: a consumer thread waits for the results in order and
    # releases each at once (as a client would), so completed results do not
    # pile up in the server's pinned result arena while requests arrive.
    # Result arrays are copied out for the first `checked` results only, and
    # the interpreter hands over between the threads every 0.2 ms, so the
    # consumer does not delay the submitting thread's arrivals.
    import queue
    import sys
    import threading
    ready = queue.Queue()
    res = []
    checked = 200

    def consume():
        while True:
            tk = ready.get()
            if tk is None:
                return
            res.append(srv.wait(tk, copy_out=len(res) < checked))

    import gc
    switch = sys.getswitchinterval()
    sys.setswitchinterval(0.0002)
    gc_was = gc.isenabled()
    gc.disable()   # a full collection over the results pauses the arrivals
    th = threading.Thread(target=consume, daemon=True)
    th.start()
    base = now_ns() + 2_000_000
    t = 0.0
    i = 0
    while t < seconds:
        t += rng.exponential(1.0 / rate)
        q = reqs[i % len(reqs)]
        i += 1
        at = base + int(t * 1e9)
        gap = at - now_ns()
        if gap > 400_000:   # sleep (releasing the interpreter) until ~0.2 ms before
            time.sleep((gap - 200_000) / 1e9)
        while now_ns() < at:
            pass
        ready.put(submit(q, at))
        used.append(q)
    ready.put(None)
    th.join()
    sys.setswitchinterval(switch)
    if gc_was:
        gc.enable()
    return res, time.perf_counter() - t0, used


def _lat(res):
    lat = [r.latency_us / 1e3 for r in res]
    return {"p50_ms": _pct(lat, 0.50), "p99_ms": _pct(lat, 0.99), "mean_ms": statistics.mean(lat)}


def _serve_report(srv_factory, reqs, submit, a, rng, check):
    """Capacity burst, per-call (unbatched) form, Poisson sweep."""
    with srv_factory(a.streams, a.max_batch) as srv:
        submit_b = submit(srv)
        _serve_phase(srv, reqs[:min(len(reqs), 2000)], submit_b)            # warm-up
        res, wall, used = _serve_phase(srv, reqs, submit_b)
        for q, r in zip(used, res):
            check(q, r)
        cap = len(res) / wall
        stats_cap = srv.stats()
        lat_cap = _lat(res)
        sweep = []
        for frac in (0.25, 0.5, 0.75, 0.9, 1.1):
            rate = frac * cap
            res, wall, used = _serve_phase(srv, reqs, submit_b, rate=rate,
                                           seconds=a.serve_seconds, rng=rng)
            for q, r in list(zip(used, res))[:200]:
                check(q, r)
            sweep.append({"offered_per_s": rate, "requests": len(res),
                          "achieved_per_s": len(res) / wall,
                          **_lat(res), "mean_batch": srv.stats()["mean_batch"]})
    with srv_factory(1, 1) as srv:
        submit_1 = submit(srv)
        n1 = min(len(reqs), 2000)
        res, wall, used = _serve_phase(srv, reqs[:200], submit_1)
        t0 = time.perf_counter()
        lat = []
        for q in reqs[:n1]:
            r = srv.wait(submit_1(q, 0))
            check(q, r)
            lat.append(r.latency_us / 1e3)
        per_call = {"value": n1 / (time.perf_counter() - t0), "p50_ms": _pct(lat, 0.5),
                    "p99_ms": _pct(lat, 0.99), "requests": n1,
                    "note": "the same kernels, one request per launch, each waited for"}
    return cap, lat_cap, stats_cap, sweep, per_call


def _ir_roofline(torch, api, t, toff, docs, h_toff, h_docs, qs):
    """The IR kernels' roofline on one reset_ir call over the queries `qs`
    (the kernels the served batches run: slice probe, slice scan, gather).
    Algorithmic bytes per query: 4 per candidate of the first list, 4 per
    probe (a candidate still alive at a further term reads one slot), 4
    per survivor written; the alive candidates come from exact host
    intersections."""
    qlist = np.concatenate(qs).astype(np.int32)
    qoff = np.zeros(len(qs) + 1, np.int32)
    qoff[1:] = np.cumsum([q.size for q in qs])
    dq = torch.from_numpy(qlist).cuda()
    dqo = torch.from_numpy(qoff).cuda()
    alg = 0
    for q in qs:
        alive = h_docs[h_toff[q[0]]:h_toff[q[0] + 1]]
        alg += 4 * alive.size
        for term in q[1:]:
            alg += 4 * alive.size
            alive = np.intersect1d(alive, h_docs[h_toff[term]:h_toff[term + 1]],
                                   assume_unique=True)
        alg += 4 * alive.size
    st = torch.cuda.current_stream()
    api.ir(t, toff, docs, dq, dqo)
    ms = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        api.ir(t, toff, docs, dq, dqo)
        e1.record(st)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    best = min(ms)
    peak, src = _peak()
    achieved = alg / (best / 1e3) / 1e9
    return {"bound": "hbm", "kernel": "ir_slice_kernel + slice scan + gather",
            "timed": f"one reset_ir call over {len(qs)} queries of the stream "
                     "(CUDA events on its stream; includes its host-side sizing read)",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": src, "traffic": None,
            "algorithmic_bytes_per_launch": int(alg), "ms_per_launch": best}


def ir_serve_ours(a, rank, world, local):
    torch = _setup(local, world)
    from reset_b200 import api, _lib
    from reset_b200.server import Server
    L = _lib.load()
    toff, docs = api.gen_inverted_index(a.terms, a.docs, 1.1, a.df_max, seed=SEED_IR)
    t = api.Table(toff, docs, hierarchical=True)
    h_toff = toff.cpu().numpy()
    h_docs = docs.cpu().numpy()
    df = np.diff(h_toff).astype(np.int64)
    rng = np.random.default_rng(SEED_IR + rank)
    reqs = _ir_queries(df, a.requests, rng)
    ix_holder = {}

    def factory(streams, mb):
        srv = Server(streams=streams, max_batch_requests=mb, max_batch_cost=a.max_batch_cost)
        ix_holder["ix"] = srv.add_index(t)
        return srv

    def submit(srv):
        return lambda q, at: srv.submit_ir(ix_holder["ix"], q, arrival_ns=at)

    checked = [0]

    def check(q, r):
        assert r.status == 0
        if checked[0] < 300:   # exact vs the merge intersection of the lists
            want = h_docs[h_toff[q[0]]:h_toff[q[0] + 1]]
            for term in q[1:]:
                want = np.intersect1d(want, h_docs[h_toff[term]:h_toff[term + 1]],
                                      assume_unique=True)
            got = r.docs if r.docs is not None else np.zeros(0, np.int32)
            assert np.array_equal(got, want), "served IR result differs"
            checked[0] += 1

    l0 = L.reset_kernel_launches()
    with B.Clocks(local) as clk:
        cap, lat_cap, st, sweep, per_call = _serve_report(factory, reqs, submit, a, rng, check)
    launches = L.reset_kernel_launches() - l0
    (cap,) = _maxr([cap], world)
    roof = _ir_roofline(torch, api, t, toff, docs, h_toff, h_docs, reqs[:512])
    qterms = sum(q.size for q in reqs) / len(reqs)
    res_ints = sum(int(df[q[0]]) for q in reqs) / len(reqs)
    line = {
        "metric": "IR queries/sec served (continuous batching), p50/p99 latency",
        "value": world * cap, "unit": "queries/s", "n_gpus": world,
        "steps": 1, "warmup": 1, "ms_per_step": 1e3 * a.requests / cap,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded inverted index generated on device; queries drawn by df)",
        "config": {"workload": f"ir_serve_{a.docs}_docs_{a.terms}_terms", "docs": a.docs,
                   "terms": a.terms, "postings": int(h_docs.size),
                   "df_law": f"Zipf(1.1), df(1) = {a.df_max}", "query_terms": "2-6, by df",
                   "mean_terms": qterms, "burst_requests": a.requests,
                   "streams": a.streams, "max_batch": a.max_batch,
                   "max_batch_cost": a.max_batch_cost,
                   "mean_batch_in_burst": st["mean_batch"],
                   "capacity_client": "closed loop, 4096 requests outstanding",
                   "server_counters_after_burst": st,
                   "results_checked_exactly": checked[0],
                   "parallelism": f"replicas x{world}"},
        "latency_at_capacity": lat_cap,
        "poisson_sweep": sweep,
        "plain_per_call": per_call,
        "e2e": {"value": world * cap, "unit": "queries/s",
                "h2d_bytes_per_step": int(4 * qterms * a.requests + 20 * a.requests),
                "d2h_bytes_per_step": int(4 * res_ints * a.requests + 4 * a.requests),
                "note": "serving is end to end by construction: host query arrays in, "
                        "host result lists out, through reset_server_*; d2h is an upper "
                        "bound (first-term lengths; only survivors are copied)"},
        "roofline": roof,
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if rank == 0:
        # exact total over all queries from one plain reset_ir call, for the
        # native client's check
        qd = torch.from_numpy(np.concatenate(reqs)).cuda()
        qo = torch.from_numpy(np.r_[0, np.cumsum([x.size for x in reqs])].astype(np.int32)).cuda()
        _, _, cnt = api.ir(t, toff, docs, qd, qo)
        exact = int(cnt.sum().item())
        del qd, qo, cnt
        # burst (capacity cross-check) and Poisson arrivals, C++ client
        nat = _ir_native(h_toff, h_docs, reqs, [4000, 8000, 12000])
        if nat is not None:
            for v in nat.values():
                if "total_results" in v:
                    assert v["total_results"] == exact, "native client totals differ"
        line["native_client"] = {"driver": "reset_b200/bin/reset_serve_ir", "runs": nat,
                                 "exact_total_results": exact,
                                 "note": "same queries and index, C++ client (4000 queries "
                                         "of warm-up, then all at once or Poisson; a waiter "
                                         "thread takes each result as it completes), table "
                                         "built by the driver (alpha 0.2, bucket 5)"}
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = _ir_cpu(h_toff, h_docs, reqs, a.cpu_seconds)
    t.free()
    _finish(line, rank, world)


def _ir_native(h_toff, h_docs, reqs, rates):
    """The same queries through the native serving driver
    (reset_b200/bin/reset_serve_ir, C++ client on reset_server_*), reading
    the index and queries in the reference's IR folder format: a burst and
    Poisson arrivals at `rates`.  Returns per-run throughput, p50/p99 and the
    total result count."""
    import re
    import shutil
    import subprocess
    import tempfile
    exe = os.path.join(B.ROOT, "reset_b200", "bin", "reset_serve_ir")
    if not os.path.exists(exe):
        return None
    d = tempfile.mkdtemp(prefix="reset_ir_")

    def arr(name, x):
        with open(os.path.join(d, name), "wb") as f:
            np.array([x.size], np.uint64).tofile(f)
            np.ascontiguousarray(x, np.int32).tofile(f)

    def scal(name, x):
        np.array([x], np.int32).tofile(os.path.join(d, name))

    try:
        arr("inverted_index_offsets.bin", h_toff)
        arr("inverted_index.bin", h_docs)
        scal("inverted_index_num.bin", h_toff.size - 1)
        arr("query.bin", np.concatenate(reqs))
        arr("query_offsets.bin", np.r_[0, np.cumsum([x.size for x in reqs])])
        scal("query_num.bin", len(reqs))
        out = {}
        runs = [("burst", [])] + [(f"poisson_{int(r)}_per_s", [f"--rate={r:.0f}"]) for r in rates]
        for label, extra in runs:
            p = subprocess.run([exe, d, "--warmup=4000"] + extra, capture_output=True,
                               text=True, timeout=900)
            if p.returncode != 0:
                out[label] = {"error": (p.stdout + p.stderr)[-300:]}
                continue
            m = re.search(r"served: ([0-9.]+) queries/s, latency p50 ([0-9.]+) ms, "
                          r"p99 ([0-9.]+) ms", p.stdout)
            tot = re.search(r"Total result count: (\d+)", p.stdout)
            out[label] = {"queries_per_s": float(m.group(1)), "p50_ms": float(m.group(2)),
                          "p99_ms": float(m.group(3)), "total_results": int(tot.group(1))}
        return out
    finally:
        shutil.rmtree(d, ignore_errors=True)


def _ir_cpu(toff, docs, reqs, seconds):
    """The oracle's hash-probe retrieval (one thread) on a bounded sample of
    the same queries."""
    import oracle
    t0 = time.perf_counter()
    ot = oracle.Table(toff, docs, hier=1)
    build = time.perf_counter() - t0
    done = 0
    t0 = time.perf_counter()
    for q in reqs:
        oracle.ir(ot, q, np.array([0, q.size], np.int32))
        done += 1
        if time.perf_counter() - t0 > seconds:
            break
    el = time.perf_counter() - t0
    return {"value": done / el, "unit": "queries/s", "cores": 1, "kind": "port",
            "sample": f"first {done} queries through the oracle's hash probe in {el:.1f} s "
                      f"(table build {build:.1f} s, not timed)"}


def _mixed_requests(s_off, s_cols, o_off, n_req, rng):
    n = s_off.size - 1
    sdeg = np.diff(s_off)
    odeg = np.diff(o_off)
    reqs = []
    cand_u = np.flatnonzero(sdeg >= 2)
    for _ in range(n_req):
        x = rng.random()
        if x < 0.4:
            k = int(rng.integers(1, 33))
            vs = rng.choice(np.flatnonzero(odeg > 0), k).astype(np.int32)
            reqs.append(("tc", vs))
        elif x < 0.8:
            k = int(rng.integers(1, 17))
            tri = []
            while len(tri) < k:
                u = int(rng.choice(cand_u))
                nu = s_cols[s_off[u]:s_off[u + 1]]
                v = int(rng.choice(nu))
                nv = s_cols[s_off[v]:s_off[v + 1]]
                pos = np.minimum(np.searchsorted(nv, nu), nv.size - 1)
                common = nu[nv[pos] == nu]
                if common.size:
                    tri.append((u, v, int(rng.choice(common))))
            reqs.append(("triples", np.array(tri, np.int32)))
        else:
            na, nb = (int(v) for v in np.exp(rng.uniform(np.log(16), np.log(1 << 20), 2)))
            reqs.append(("raw", (rng.integers(0, n, na).astype(np.int32),
                                 rng.integers(0, n, nb).astype(np.int32))))
    return reqs


def mixed_serve_ours(a, rank, world, local):
    torch = _setup(local, world)
    from reset_b200 import api, _lib
    from reset_b200.server import Server
    L = _lib.load()
    scale = 22
    o_off, o_cols = api.gen_rmat(scale, 16, SEED_MIX, oriented=True)
    s_off, s_cols = api.gen_rmat(scale, 16, SEED_MIX, oriented=False)
    to = api.Table(o_off, o_cols, hierarchical=True)
    ts = api.Table(s_off, s_cols, hierarchical=True)
    hs_off, hs_cols = s_off.cpu().numpy(), s_cols.cpu().numpy()
    ho_off, ho_cols = o_off.cpu().numpy(), o_cols.cpu().numpy()
    rng = np.random.default_rng(SEED_MIX + rank)
    reqs = _mixed_requests(hs_off, hs_cols, ho_off, a.requests, rng)
    ixs = {}

    def factory(streams, mb):
        srv = Server(streams=streams, max_batch_requests=mb, max_batch_cost=a.max_batch_cost)
        ixs["o"] = srv.add_index(to)
        ixs["s"] = srv.add_index(ts)
        return srv

    def submit(srv):
        def f(q, at):
            kind, args = q
            if kind == "tc":
                return srv.submit_tc_vertices(ixs["o"], args, arrival_ns=at)
            if kind == "triples":
                return srv.submit_triples(ixs["s"], args, arrival_ns=at)
            return srv.submit_raw(args[0], args[1], arrival_ns=at)
        return f

    checked = {"tc": 0, "triples": 0, "raw": 0}

    def check(q, r):
        kind, args = q
        assert r.status == 0
        if checked[kind] >= 40:
            return
        checked[kind] += 1
        if kind == "tc":
            want = [sum(np.intersect1d(ho_cols[ho_off[v]:ho_off[v + 1]],
                                       ho_cols[ho_off[w]:ho_off[w + 1]],
                                       assume_unique=True).size
                        for w in ho_cols[ho_off[v]:ho_off[v + 1]]) for v in args]
            assert list(r.values) == want
        elif kind == "triples":
            row = lambda v: hs_cols[hs_off[v]:hs_off[v + 1]]
            want = [np.intersect1d(np.intersect1d(row(u), row(v), assume_unique=True), row(w),
                                   assume_unique=True).size for u, v, w in args]
            assert list(r.values) == want
        else:
            A, Bs = args
            assert r.count == int(np.isin(A, Bs).sum())

    l0 = L.reset_kernel_launches()
    with B.Clocks(local) as clk:
        cap, lat_cap, st, sweep, per_call = _serve_report(factory, reqs, submit, a, rng, check)
    launches = L.reset_kernel_launches() - l0
    (cap,) = _maxr([cap], world)
    mix = {k: sum(1 for q in reqs if q[0] == k) for k in ("tc", "triples", "raw")}
    line = {
        "metric": "mixed intersection requests/sec served (continuous batching), p50/p99",
        "value": world * cap, "unit": "requests/s", "n_gpus": world,
        "steps": 1, "warmup": 1, "ms_per_step": 1e3 * a.requests / cap,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded R-MAT scale 22 generated on device; request mix drawn "
                "from it)",
        "config": {"workload": f"mixed_serve_rmat_s{scale}", "scale": scale,
                   "mix": mix, "tc": "1-32 vertices per job (oriented graph)",
                   "triples": "1-16 triangles (u,v,w) per job -> |N(u)∩N(v)∩N(w)|",
                   "raw": "|A|,|B| log-uniform over 2^4..2^20, ids in [0, 2^22)",
                   "streams": a.streams, "max_batch": a.max_batch,
                   "max_batch_cost": a.max_batch_cost,
                   "mean_batch_in_burst": st["mean_batch"], "checked_exactly": checked,
                   "server_counters_after_burst": st,
                   "parallelism": f"replicas x{world}"},
        "latency_at_capacity": lat_cap,
        "poisson_sweep": sweep,
        "plain_per_call": per_call,
        "e2e": {"value": world * cap, "unit": "requests/s", "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": None,
                "note": "serving is end to end by construction (host arrays in and out)"},
        "roofline": None,
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    to.free()
    ts.free()
    _finish(line, rank, world)


# ============================================================== dispatch ==

# =============================================================== tc-batch ==

SEED_TCB = 0x5EED0BA0


def tc_batch_ours(a, rank, world, local):
    """Batched TC: `graphs` disjoint seeded R-MAT graphs (scales cycling
    over 8..12), counted (1) by the plain per-call form -- per graph one
    table build and one reset_tc_count, each waited for -- and (2) batched:
    one block-diagonal CSR, one table build and one reset_tc_count_batch.
    Per-graph counts must be equal; both timed with CUDA events."""
    torch = _setup(local, world)
    from reset_b200 import api, _lib
    L = _lib.load()
    scales = [8 + (i % 5) for i in range(a.graphs)]
    gs = [api.gen_rmat(s, 16, SEED_TCB + i, oriented=True) for i, s in enumerate(scales)]
    nv = [int(o.numel() - 1) for o, _ in gs]
    ne = [int(c.numel()) for _, c in gs]
    vb = np.concatenate([[0], np.cumsum(nv)]).astype(np.int64)
    eb = np.concatenate([[0], np.cumsum(ne)]).astype(np.int64)
    off = torch.cat([torch.zeros(1, dtype=torch.int64, device="cuda")] +
                    [o[1:].long() + int(eb[i]) for i, (o, _) in enumerate(gs)]).int()
    cols = torch.cat([c.long() + int(vb[i]) for i, (_, c) in enumerate(gs)]).int()
    gro = torch.tensor(vb, dtype=torch.int32, device="cuda")
    m = int(cols.numel())
    alpha, bucket = 0.2, 5

    def plain():
        out = []
        for o, c in gs:
            t = api.Table(o, c, alpha=alpha, bucket=bucket, hierarchical=True, hash_order=True)
            out.append(api.tc_count(t, o, t.hash_order))
            t.free()
        return out

    def batched():
        t = api.Table(off, cols, alpha=alpha, bucket=bucket, hierarchical=True, hash_order=True)
        r = api.tc_count_batch(t, off, t.hash_order, gro)
        t.free_async()
        return r

    def timed(fn, reps):
        ms, res = [], None
        for _ in range(reps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            res = fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return statistics.median(ms), res

    for _ in range(a.warmup):
        want = plain()
        batched()
    l0 = L.reset_kernel_launches()
    with B.Clocks(local) as clk:
        ms_b, got = timed(batched, a.steps)
    launches = L.reset_kernel_launches() - l0
    ms_p, want = timed(plain, max(1, min(a.steps, 3)))
    assert got.cpu().tolist() == want, "batched per-graph counts differ from per-call counts"
    ms_b, ms_p = _maxr([ms_b, ms_p], world)
    line = {
        "metric": "TC edges/sec, batched (many graphs per launch) vs plain per-call",
        "value": world * m / (ms_b / 1e3), "unit": "edges/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_b, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded R-MAT graphs generated on device)",
        "config": {"workload": f"tc_batch_{a.graphs}_rmat_s8_12", "graphs": a.graphs,
                   "vertices": int(vb[-1]), "oriented_edges": m,
                   "triangles": int(sum(want)), "alpha": alpha, "bucket": bucket,
                   "parity": "per-graph counts of the batched call equal the per-call counts",
                   "parallelism": f"replicas x{world}"},
        "plain_per_call": {"value": world * m / (ms_p / 1e3), "unit": "edges/s",
                           "ms_per_pass": ms_p,
                           "note": "per graph: table build + reset_tc_count, each waited for"},
        "speedup_vs_plain": ms_p / ms_b,
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    _finish(line, rank, world)


SEED_PAT = 0x5EED7C00


def _pattern_checks(api, pattern):
    """Second encodings of the clique patterns, counted by other kernels:
    Q0 by the triangle count, Q3 by the 4-clique kernel, Q5 and Q7 listed
    level by level (no reuse) through the general pattern kernel."""
    def listed(k):
        offs = [0, 1] + [1 + sum(range(2, l + 1)) for l in range(2, k)]
        return api.PatternSpec(k, tuple(offs), tuple([0] + [j for l in range(2, k) for j in range(l)]))
    return {"Q0": lambda t, o, c: api.tc_count(t, o, c),
            "Q3": lambda t, o, c: api.clique4_count(t, o, c),
            "Q5": lambda t, o, c: api.pattern_count(t, o, c, listed(5)),
            "Q7": lambda t, o, c: api.pattern_count(t, o, c, listed(6))}.get(pattern)


def pattern_ours(a, rank, world, local):
    """SMOG's query patterns Q0..Q8 (reset_pattern_count) on seeded R-MAT
    graphs of scale a.pattern_scale, each on the graph the reference counts
    it on (oriented for the cliques, symmetric for the rest).  Per pattern,
    the median of a.steps calls (CUDA events around the whole call:
    row-order pass, scratch, kernel, count read back); the clique patterns'
    counts are checked against second encodings run by other kernels."""
    torch = _setup(local, world)
    from reset_b200 import api, _lib
    L = _lib.load()
    S = a.pattern_scale
    graphs = {}
    for g in ("oriented", "symmetric"):
        off, cols = api.gen_rmat(S, 16, SEED_PAT + S, oriented=(g == "oriented"))
        graphs[g] = (off, cols, api.Table(off, cols))
    rows, total_ms, launches = {}, 0.0, 0
    with B.Clocks(local) as clk:
        for name, p in api.PATTERNS.items():
            off, cols, t = graphs[p.graph]
            for _ in range(max(a.warmup, 1)):
                want = api.pattern_count(t, off, cols, name)
            ms = []
            l0 = L.reset_kernel_launches()
            for _ in range(a.steps):
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                got = api.pattern_count(t, off, cols, name)
                e1.record()
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
                assert got == want, name
            launches += L.reset_kernel_launches() - l0
            chk = _pattern_checks(api, name)
            rows[name] = {"graph": p.graph, "count": want, "ms": statistics.median(ms),
                          "start_edges": int(cols.numel())}
            if chk is not None:
                other = chk(t, off, cols)
                assert other == want, f"{name}: {want} vs {other}"
                rows[name]["checked_by_second_encoding"] = True
            total_ms += rows[name]["ms"]
    [total_ms] = _maxr([total_ms], world)
    line = {
        "metric": "SMOG query patterns Q0-Q8: summed time per call",
        "value": total_ms, "unit": "ms", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": total_ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded R-MAT graphs generated on device)",
        "config": {"workload": f"patterns_rmat_s{S}_ef16", "scale": S,
                   "vertices": 1 << S, "patterns": rows,
                   "parallelism": f"replicas x{world}"},
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    _finish(line, rank, world)


def run_ours(a, rank, world, local):
    {"sss-join": sss_join_ours, "ir-serve": ir_serve_ours,
     "mixed-serve": mixed_serve_ours, "tc-batch": tc_batch_ours,
     "pattern": pattern_ours}[a.workload](a, rank, world, local)


def run_reference(a, rank, world):
    """The reference has no CPU implementation of these paths; its algorithm
    restated on the CPU (the oracle) is timed on a bounded sample."""
    if rank != 0:
        return
    import oracle
    thr = 1
    if a.workload == "sss-join":
        # CPU generator stand-in: same law, smaller draw (the oracle has no
        # token-set generator); timed decisions on its prefix candidates
        rng = np.random.default_rng(SEED_SSS)
        n = min(a.sets, 200_000)
        w = 1.0 / np.arange(8, a.size_hi + 1) ** 1.2
        sz = rng.choice(np.arange(8, a.size_hi + 1), n, p=w / w.sum())
        U = 1 << 24
        rows = [np.unique(np.minimum((np.exp(rng.random(k) * np.log(U + 1)) - 1).astype(np.int64),
                                     U - 1)) for k in sz]
        off = np.zeros(n + 1, np.int32)
        off[1:] = np.cumsum([r.size for r in rows])
        tok = np.concatenate(rows).astype(np.int32)
        pa = rng.integers(0, n, 400_000).astype(np.int32)
        pb = rng.integers(0, n, 400_000).astype(np.int32)
        cb = _sss_cpu(off, tok, pa, pb, a.cpu_seconds)
        cb.pop("checked")
        unit, metric = "intersections/s", "set-intersections/sec (Jaccard 0.7 decisions)"
    elif a.workload == "ir-serve":
        rng = np.random.default_rng(SEED_IR)
        nt, nd = min(a.terms, 100_000), a.docs
        df = np.minimum(np.maximum(1, np.round(a.df_max * np.arange(1, nt + 1) ** -1.1)),
                        nd).astype(np.int64)
        lists = [np.unique(rng.integers(0, nd, int(k))) for k in df]
        toff = np.zeros(nt + 1, np.int32)
        toff[1:] = np.cumsum([x.size for x in lists])
        docs = np.concatenate(lists).astype(np.int32)
        reqs = _ir_queries(np.diff(toff).astype(np.int64), 5000, rng)
        cb = _ir_cpu(toff, docs, reqs, a.cpu_seconds)
        unit, metric = "queries/s", "IR queries/sec"
    elif a.workload == "pattern":
        # the oracle's count by definition (all host threads) per pattern on
        # the same seeded graphs, at a smaller scale (bounded CPU time)
        from reset_b200.api import PATTERNS
        S = min(a.pattern_scale, 11)
        per, el = {}, 0.0
        for name, p in PATTERNS.items():
            off, cols = oracle.rmat_graph(S, 16, SEED_PAT + S, oriented=(p.graph == "oriented"))
            t0 = time.perf_counter()
            c = oracle.pattern_count(off, cols, p.k, p.flags, p.offsets, p.backward,
                                     p.restriction, p.reuse)
            per[name] = {"count": c, "s": time.perf_counter() - t0}
            el += per[name]["s"]
        cores = os.cpu_count() or 1
        cb = {"value": el * 1e3, "unit": "ms", "cores": cores, "kind": "port",
              "sample": f"Q0-Q8 at scale {S} (GPU arm: scale {a.pattern_scale}), oracle by "
                        f"definition: " + ", ".join(f"{k} {v['s']:.2f} s" for k, v in per.items())}
        unit, metric = "ms", "SMOG query patterns Q0-Q8: summed time per call"
    elif a.workload == "tc-batch":
        t0 = time.perf_counter()
        edges, gi = 0, 0
        while time.perf_counter() - t0 < a.cpu_seconds and gi < a.graphs:
            o, c = oracle.rmat_graph(8 + (gi % 5), 16, SEED_TCB + gi, oriented=True)
            oracle.tc_merge(o, c, nthreads=1)
            edges += int(c.size)
            gi += 1
        el = time.perf_counter() - t0
        cb = {"value": edges / el, "unit": "edges/s", "cores": 1, "kind": "port",
              "sample": f"{gi} of the {a.graphs} graphs, oracle merge TC one by one, {el:.1f} s"}
        unit, metric = "edges/s", "TC edges/sec, batched (many graphs per launch) vs plain per-call"
    else:
        off, cols = oracle.rmat_graph(18, 16, SEED_MIX, oriented=False)
        rng = np.random.default_rng(SEED_MIX)
        t0 = time.perf_counter()
        done = 0
        while time.perf_counter() - t0 < a.cpu_seconds:
            na, nb = (int(v) for v in np.exp(rng.uniform(np.log(16), np.log(1 << 20), 2)))
            oracle.pair_count(rng.integers(0, 1 << 22, na).astype(np.int32),
                              rng.integers(0, 1 << 22, nb).astype(np.int32))
            done += 1
        el = time.perf_counter() - t0
        cb = {"value": done / el, "unit": "requests/s", "cores": 1, "kind": "port",
              "sample": f"{done} raw-pair requests through the oracle in {el:.1f} s"}
        unit, metric = "requests/s", "mixed intersection requests/sec"
    line = {"metric": metric, "value": cb["value"], "unit": unit, "n_gpus": world,
            "steps": 1, "warmup": 0, "ms_per_step": None,
            "higher_is_better": a.workload != "pattern",
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (CPU generators)", "impl": "reference",
            "config": {"workload": a.workload, "parallelism": "cpu",
                       "note": "the reference has no CPU implementation of this path; this "
                               "is the CPU port of its algorithm (oracle) on a sample"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": unit, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)

"""Autotuner for the table and probe parameters (load factor alpha, slots per
bucket b, probe rounds, warp-per-pair threshold).

Counterpart of the reference's hyperparameter_solver
(hyperparameter_solver/src/solver.py:132-188 cost model over the grid of
hyperparameter_solver/src/config.json; result type HyperParams{alpha, b,
cost} of hyperparameter_solver/cpp/hyper_solver.h:22-29).  The reference
ranks (alpha, b) with an analytic model of expected slot reads per lookup.
Here the model is only a prior: it ranks the grid, the best `measure_top`
points are built and timed on a sample of the actual workload on this GPU,
and the fastest wins.  Results are cached in a JSON file keyed by the GPU
name and a signature of the workload.
"""
from __future__ import annotations

import hashlib
import json
import os
import time
from dataclasses import asdict, dataclass
from typing import Callable, Dict, Iterable, List, Optional, Sequence, Tuple

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "reset_b200", "autotune.json")

# the reference's search grid (config.json: alpha 0.1..1 step 0.05, b 1..9)
ALPHAS = tuple(round(0.1 + 0.05 * i, 2) for i in range(19))
BUCKETS = tuple(range(1, 10))


@dataclass
class HyperParams:
    alpha: float = 0.2
    b: int = 5
    probe_rounds: int = 8
    warp_pair_min: int = 64
    cost: float = 0.0           # model cost (slot reads per probe) or measured ms
    measured_ms: Optional[float] = None


# ------------------------------------------------------------ cost model --

def calc_len(degree, alpha: float, bucket: int):
    """calculate_length (triangle-count/hashtable.cu:21-36) in float32;
    accepts a scalar or an array of degrees."""
    import numpy as np
    d = np.asarray(degree, dtype=np.int64)
    t = (d.astype(np.float32) / np.float32(alpha)).astype(np.int64)
    L = t // bucket
    nxt = np.left_shift(1, np.floor(np.log2(np.maximum(L, 1))).astype(np.int64) + 1)
    out = np.where(L == 0, 8, np.maximum(8, nxt))
    return int(out) if out.ndim == 0 else out


def _unique_weights(degrees):
    import numpy as np
    d = np.asarray(degrees, dtype=np.int64)
    d = d[d > 0]
    u, w = np.unique(d, return_counts=True)
    return u, w.astype(np.float64)


def slot_reads(alpha: float, b: int, degrees: Sequence[int], hit_rate: float = 0.15,
               kmax: int = 48) -> float:
    """Expected slots read per probe (each slot of a bucket is its own
    32-byte sector in the reference layout).  Keys per bucket ~ Poisson(lam),
    lam = d / len(d); a bucket holding j keys costs j+1 reads for a miss
    (the -1 slot ends it; keys past b spill into the following buckets and
    lengthen the walk) and about half that for a hit.  Averaged over the
    given degrees."""
    import numpy as np
    u, w = _unique_weights(degrees)
    if u.size == 0:
        return 0.0
    lam = u / calc_len(u, alpha, b)
    j = np.arange(kmax + 1, dtype=np.float64)
    # Poisson pmf, rows = degrees, cols = j
    logp = -lam[:, None] + j[None, :] * np.log(lam[:, None]) - np.cumsum(
        np.concatenate([[0.0], np.log(j[1:])]))[None, :]
    p = np.exp(logp)
    extra = np.maximum(j - b + 1, 0)
    miss = np.where(j < b, j + 1, b + 1 + extra)
    hit = np.where(j < b, np.maximum((j + 1) / 2.0, 1.0), (b + 1) / 2.0 + extra / 2.0)
    per = (p * (hit_rate * hit + (1 - hit_rate) * miss)[None, :]).sum(1)
    return float((per * w).sum() / w.sum())


def table_bytes(alpha: float, b: int, degrees: Sequence[int]) -> int:
    u, w = _unique_weights(degrees)
    return int(4 * b * (calc_len(u, alpha, b) * w).sum()) if u.size else 0


def model_rank(degrees: Sequence[int], alphas: Iterable[float] = ALPHAS,
               buckets: Iterable[int] = BUCKETS, mem_weight: float = 0.25,
               hit_rate: float = 0.15) -> List[HyperParams]:
    """The grid ranked by model cost = slot reads per probe plus a charge
    for table bytes per key (building and holding the table)."""
    u, w = _unique_weights(degrees)
    keys = max(1.0, float((u * w).sum()))
    out = []
    for a in alphas:
        for b in buckets:
            reads = slot_reads(a, b, degrees, hit_rate)
            mem = table_bytes(a, b, degrees) / keys / 32.0  # in sectors per key
            out.append(HyperParams(alpha=a, b=b, cost=reads + mem_weight * mem))
    out.sort(key=lambda h: h.cost)
    return out


# ----------------------------------------------------------------- cache --

def gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name()
    except Exception:
        return "unknown"


def signature(kind: str, degrees: Sequence[int], extra: str = "") -> str:
    import numpy as np
    d = np.asarray(degrees, dtype=np.int64)
    hist = np.bincount(np.minimum(np.log2(np.maximum(d, 1)).astype(np.int64), 40), minlength=41)
    h = hashlib.sha1((kind + extra).encode() + hist.tobytes()).hexdigest()[:16]
    return f"{kind}:{d.size}:{int(d.sum())}:{h}"


def _load(path: str) -> Dict[str, dict]:
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(path: str, data: Dict[str, dict]):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


# ----------------------------------------------------------------- solve --

def solve(kind: str, degrees: Sequence[int], measure: Optional[Callable[[HyperParams], float]] = None,
          measure_top: int = 6, rounds: Sequence[int] = (4, 8),
          warp_pair_mins: Sequence[int] = (32, 64, 128), cache: Optional[str] = DEFAULT_CACHE,
          alphas: Iterable[float] = ALPHAS, buckets: Iterable[int] = BUCKETS,
          extra_key: str = "",
          always: Sequence[Tuple[float, int]] = ((0.2, 5),)) -> HyperParams:
    """Pick parameters for a workload.

    degrees: set sizes of the table side (a sample is fine).
    measure(hp) -> milliseconds for one pass of the workload sample with hp
      (build + probe); None keeps the model's choice.
    The model's best `measure_top` (alpha, b) points, plus `always` (the
    reference default 0.2 / 5), are measured with the default probe knobs,
    then the probe knobs are swept at the best point.
    """
    key = f"{gpu_name()}|{signature(kind, degrees, extra_key)}"
    if cache:
        hit = _load(cache).get(key)
        if hit:
            return HyperParams(**hit)
    ranked = model_rank(degrees, alphas, buckets)
    best = ranked[0]
    if measure is not None:
        timed: List[Tuple[float, HyperParams]] = []
        pts = ranked[:max(1, measure_top)]
        for a, b in always:
            if all((h.alpha, h.b) != (a, b) for h in pts):
                pts.append(next((h for h in ranked if (h.alpha, h.b) == (a, b)),
                                HyperParams(alpha=a, b=b)))
        for hp in pts:
            ms = measure(hp)
            timed.append((ms, hp))
        timed.sort(key=lambda x: x[0])
        best_ms, best = timed[0]
        for r in rounds:
            for w in warp_pair_mins:
                hp = HyperParams(alpha=best.alpha, b=best.b, probe_rounds=r, warp_pair_min=w,
                                 cost=best.cost)
                if (r, w) == (best.probe_rounds, best.warp_pair_min):
                    continue
                ms = measure(hp)
                if ms < best_ms:
                    best_ms, best = ms, hp
        best.measured_ms = best_ms
    if cache:
        data = _load(cache)
        data[key] = asdict(best)
        _store(cache, data)
    return best


def timed(fn: Callable[[], None], reps: int = 3) -> float:
    """Median wall time (ms) of fn() with a device sync after each call."""
    import torch
    ts = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        ts.append((time.perf_counter() - t0) * 1e3)
    ts.sort()
    return ts[len(ts) // 2]

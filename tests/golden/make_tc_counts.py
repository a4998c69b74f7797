#!/usr/bin/env python
"""Exact triangle counts of the seeded R-MAT graphs the benchmark and the
GPU parity tests use, computed by the CPU oracle (sorted-row merge,
oracle.c ro_tc_merge, all host threads) -- test infrastructure.

The graphs are the R-MAT generator's (scale s, edge factor 16, a/b/c/d =
.57/.19/.19/.05, vertices relabeled by the seeded bijection, symmetrised,
self-loops and duplicates removed, oriented low degree -> high degree, ties
by id) with seed 0x5EED00SS (SS = the scale in decimal digits), the seed
bench.py uses at every scale.
The oracle's generator equals the device generator bit for bit (checked by
the GPU parity tests), so a count here pins the device count of the same
scale without running the oracle at benchmark time.

    python tests/golden/make_tc_counts.py 16 20 22 24
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

OUT = os.path.join(HERE, "tc_counts.json")


def rmat_seed(scale: int) -> int:
    """0x5EED00SS with the scale's decimal digits as the last two hex
    digits (scale 24 -> 0x5EED0024), the benchmark's seed convention."""
    return int(f"0x5EED00{scale:02d}", 16)


def main():
    import numpy as np
    import oracle
    scales = [int(x) for x in sys.argv[1:]] or [16, 20, 22, 24]
    try:
        rec = json.load(open(OUT))
    except FileNotFoundError:
        rec = {"generator": "R-MAT a/b/c/d .57/.19/.19/.05, relabeled, oriented by degree",
               "edge_factor": 16, "counts": {}}
    threads = os.cpu_count() or 1
    for s in scales:
        seed = rmat_seed(s)
        t0 = time.perf_counter()
        off, cols = oracle.rmat_graph(s, 16, seed, oriented=True)
        t1 = time.perf_counter()
        tri = oracle.tc_merge(off, cols, nthreads=threads)
        t2 = time.perf_counter()
        d = np.diff(off).astype(np.int64)
        src = np.repeat(np.arange(off.size - 1), d)
        probes = int(np.minimum(d[src], d[cols]).sum())
        rec["counts"][str(s)] = {"seed": hex(seed), "vertices": int(off.size - 1),
                                 "oriented_edges": int(cols.size), "triangles": int(tri),
                                 "probes": probes}
        print(f"scale {s}: n={off.size - 1} m={cols.size} triangles={tri} probes={probes} "
              f"(generate {t1 - t0:.1f} s, count {t2 - t1:.1f} s on {threads} threads)",
              flush=True)
        json.dump(rec, open(OUT, "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""Time the reference's own triangle-count kernel (oracle/_ref/ref_tc: the
reference's triangle-count/TC.cu + hashtable.cu compiled unchanged for
sm_100a) on the same seeded R-MAT graph bench.py uses, for a side-by-side
with this library's kernel on the same GPU.  Test/measurement
infrastructure: the graph comes from the CPU oracle's generator (identical
to the device generator), is written in the reference's TC input format
(triangle-count/TC.cu:236-245) to a scratch folder, and ref_tc prints the
kernel time of dynamic_triangle_count (TC.cu:128-190, launch shape of
TC.cu:268-275) in both hash modes, timed with CUDA events.

    python oracle/ref_bench.py --scale 24 [--alpha 0.2 --bucket 5] [--workdir DIR]

Before any kernel runs, the harness refuses graphs whose tables would
overflow the reference's 32-bit slot index (bucket + k * bucket_num); the
printed line gives bucket_num and the largest index.  Counts are compared
with the oracle's count of the same graph (tests/golden/tc_counts.json).
"""
import argparse
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def write_arr(path, a):
    with open(path, "wb") as f:
        np.array([a.size], np.uint64).tofile(f)
        np.ascontiguousarray(a).tofile(f)


def write_int(path, x):
    np.array([x], np.int32).tofile(path)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--seed", type=lambda s: int(s, 0), default=None,
                    help="default 0x5EED00SS, SS = the scale's decimal digits")
    ap.add_argument("--device-gen", action="store_true",
                    help="generate the graph with the library's device generator")
    ap.add_argument("--alpha", type=float, default=0.2)
    ap.add_argument("--bucket", type=int, default=5)
    ap.add_argument("--workdir", default=None)
    a = ap.parse_args()
    import oracle
    seed = a.seed if a.seed is not None else int(f"0x5EED00{a.scale:02d}", 16)
    exe = os.path.join(HERE, "_ref", "ref_tc")
    if not os.path.exists(exe):
        sys.exit("oracle/_ref/ref_tc is missing (build it with `make -C oracle ref`)")
    t0 = time.perf_counter()
    if a.device_gen:
        # the library's device generator: the same graph bit for bit (the
        # GPU parity tests compare it with the oracle's), minutes faster
        import torch
        from reset_b200 import api
        d_off, d_cols = api.gen_rmat(a.scale, a.edge_factor, seed, oriented=True)
        off, cols = d_off.cpu().numpy(), d_cols.cpu().numpy()
        del d_off, d_cols
        torch.cuda.empty_cache()
    else:
        off, cols = oracle.rmat_graph(a.scale, a.edge_factor, seed, oriented=True)
    gen = time.perf_counter() - t0
    work = a.workdir or tempfile.mkdtemp(prefix="reset_ref_tc_")
    ind, outd = os.path.join(work, "in"), os.path.join(work, "out")
    os.makedirs(ind, exist_ok=True)
    os.makedirs(outd, exist_ok=True)
    try:
        write_arr(os.path.join(ind, "csr_offsets_tri.bin"), off.astype(np.int32))
        write_arr(os.path.join(ind, "csr_cols_tri.bin"), cols.astype(np.int32))
        write_int(os.path.join(ind, "num_nodes_tri.bin"), off.size - 1)
        write_int(os.path.join(ind, "num_edges_tri.bin"), cols.size)
        print(f"graph: scale {a.scale} seed {seed:#x} n={off.size - 1} m={cols.size} "
              f"(CPU generator {gen:.1f} s)", flush=True)
        r = subprocess.run([exe, ind, outd, f"--alpha={a.alpha}", f"--bucket={a.bucket}",
                            "--no-dump"], capture_output=True, text=True)
        print(r.stdout.strip())
        if r.returncode != 0:
            print(r.stderr.strip(), file=sys.stderr)
            return r.returncode
        import json
        try:
            rec = json.load(open(os.path.join(os.path.dirname(HERE), "tests", "golden",
                                              "tc_counts.json")))["counts"].get(str(a.scale))
        except OSError:
            rec = None
        if rec and int(rec["seed"], 16) == seed:
            import re
            got = [int(x) for x in re.findall(r"(?:normal|hier)=(\d+)", r.stdout)]
            ok = bool(got) and all(g == rec["triangles"] for g in got)
            print(f"oracle count {rec['triangles']}: reference counts {got} "
                  f"{'equal' if ok else 'DIFFER'}")
            return 0 if ok else 1
        return 0
    finally:
        shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    sys.exit(main())

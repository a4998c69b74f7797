"""Generates the golden fixtures of tests/golden/ from the REFERENCE itself.

Runs the reference's own kernels (triangle-count/, set-similarity-search/,
information-retrieval/, set_size/ compiled unchanged for sm_100a into
oracle/_ref/ by `make -C oracle ref`) on small seeded inputs written in the
reference's .bin formats, and packs inputs + reference outputs into
compressed .npz files.  Needs a GPU:

    python tests/golden/make_golden.py --out /tmp/golden

and copy the .npz files into tests/golden/.  Inputs come from the oracle's
seeded generators, so they can be re-created anywhere.
"""
from __future__ import annotations

import argparse
import os
import struct
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")


def write_arr(path, a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", a.size))
        f.write(a.tobytes())


def write_int(path, v):
    with open(path, "wb") as f:
        f.write(struct.pack("<i", int(v)))


def read_arr(path, dtype=np.int32):
    with open(path, "rb") as f:
        n = struct.unpack("<Q", f.read(8))[0]
        return np.frombuffer(f.read(), dtype=dtype, count=n).copy()


def run(exe, *args):
    r = subprocess.run([os.path.join(REF, exe), *args], capture_output=True, text=True)
    sys.stdout.write(r.stdout)
    if r.returncode != 0:
        sys.stderr.write(r.stderr)
        raise SystemExit(f"{exe} failed ({r.returncode})")


def outputs(d, names):
    res = {}
    for nm in names:
        p = os.path.join(d, nm)
        key = nm.replace(".i64.bin", "").replace(".bin", "")
        res["ref_" + key] = read_arr(p, np.int64 if nm.endswith(".i64.bin") else np.int32)
    return res


def tc_case(work, name, scale, seed, alpha, bucket):
    # raw R-MAT ids (skewed bucket occupancy: long probe chains are exercised)
    off, cols = O.rmat_graph(scale, 16, seed, oriented=True, relabel=False)
    d = os.path.join(work, name)
    os.makedirs(d, exist_ok=True)
    write_arr(f"{d}/csr_offsets_tri.bin", off)
    write_arr(f"{d}/csr_cols_tri.bin", cols)
    write_int(f"{d}/num_nodes_tri.bin", off.size - 1)
    write_int(f"{d}/num_edges_tri.bin", cols.size)
    run("ref_tc", d, d, f"--alpha={alpha}", f"--bucket={bucket}")
    out = outputs(d, ["meta.i64.bin", "len.bin", "off64.i64.bin", "table_normal.bin",
                      "table_hier.bin", "cols_hier_sorted.bin"])
    return dict(off=off, cols=cols, alpha=np.float32(alpha), bucket=np.int32(bucket),
                scale=np.int32(scale), seed=np.int64(seed), **out)


def sss_case(work, name, scale, seed, thr):
    off, cols = O.rmat_graph(scale, 16, seed, oriented=False, relabel=False)
    n = off.size - 1
    vert = np.repeat(np.arange(n, dtype=np.int32), np.diff(off))
    d = os.path.join(work, name)
    os.makedirs(d, exist_ok=True)
    write_arr(f"{d}/csr_offsets.bin", off)
    write_arr(f"{d}/csr_cols.bin", cols)
    write_arr(f"{d}/vertexs.bin", vert)
    write_int(f"{d}/num_nodes.bin", n)
    write_int(f"{d}/num_edges.bin", cols.size)
    run("ref_sss", d, d, f"--thr={thr}")
    out = outputs(d, ["meta.i64.bin", "len.bin", "off64.i64.bin", "results_normal.bin",
                      "results_hier.bin", "cols_hier_sorted.bin"])
    return dict(off=off, cols=cols, thr=np.float32(thr), seed=np.int64(seed), **out)


def ir_index(nterms, ndocs, npost, nq, seed):
    """Small seeded inverted index + queries in the reference's conventions:
    posting lists sorted ascending, query terms distinct and ordered by
    (df, id) ascending (preprocess/preprocessor.py:345-349)."""
    rng = np.random.default_rng(seed)
    w = 1.0 / np.arange(1, nterms + 1) ** 1.1
    df = np.maximum(1, np.round(w / w.sum() * npost)).astype(np.int64)
    df = np.minimum(df, ndocs)
    lists = [np.sort(rng.choice(ndocs, size=int(k), replace=False)).astype(np.int32) for k in df]
    toff = np.zeros(nterms + 1, np.int32)
    toff[1:] = np.cumsum([l.size for l in lists])
    docs = np.concatenate(lists).astype(np.int32)
    p = df / df.sum()
    q, qoff = [], [0]
    for _ in range(nq):
        k = int(rng.integers(1, 6))
        ts = np.unique(rng.choice(nterms, size=k, p=p))
        ts = sorted(ts.tolist(), key=lambda t: (int(df[t]), t))
        q.extend(ts)
        qoff.append(len(q))
    return toff, docs, np.array(q, np.int32), np.array(qoff, np.int32)


def ir_case(work, name, seed):
    toff, docs, query, qoff = ir_index(300, 20000, 60000, 400, seed)
    d = os.path.join(work, name)
    os.makedirs(d, exist_ok=True)
    write_arr(f"{d}/inverted_index_offsets.bin", toff)
    write_arr(f"{d}/inverted_index.bin", docs)
    write_int(f"{d}/inverted_index_num.bin", toff.size - 1)
    write_arr(f"{d}/query.bin", query)
    write_arr(f"{d}/query_offsets.bin", qoff)
    write_int(f"{d}/query_num.bin", qoff.size - 1)
    run("ref_ir", d, d)
    out = outputs(d, ["meta.i64.bin", "len.bin", "off64.i64.bin", "result_normal.bin",
                      "count_normal.bin", "result_hier.bin", "count_hier.bin",
                      "result_offsets.i64.bin", "docs_hier_sorted.bin"])
    return dict(toff=toff, docs=docs, query=query, qoff=qoff, seed=np.int64(seed), **out)


def pair_case(work, name, na, nb, seed, universe):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, universe, size=na, dtype=np.int64).astype(np.int32)
    b = rng.integers(0, universe, size=nb, dtype=np.int64).astype(np.int32)
    d = os.path.join(work, name)
    os.makedirs(d, exist_ok=True)
    write_arr(f"{d}/a.bin", a)
    write_arr(f"{d}/b.bin", b)
    run("ref_pair", d, d)
    return dict(a=a, b=b, seed=np.int64(seed), **outputs(d, ["meta.i64.bin"]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    work = os.path.join(a.out, "work")
    os.makedirs(work, exist_ok=True)
    cases = {
        "tc_s10": lambda: tc_case(work, "tc_s10", 10, 0x5EED0010, 0.2, 5),
        "tc_s11_a05_b3": lambda: tc_case(work, "tc_s11_a05_b3", 11, 0x5EED0011, 0.5, 3),
        "sss_s9_t025": lambda: sss_case(work, "sss_s9_t025", 9, 0x5EED0009, 0.25),
        "sss_s9_t07": lambda: sss_case(work, "sss_s9_t07", 9, 0x5EED0109, 0.7),
        "ir_small": lambda: ir_case(work, "ir_small", 0x1A1A),
        "pair_1000_3000": lambda: pair_case(work, "pair_1000_3000", 1000, 3000, 7, 6000),
        "pair_4096_4096": lambda: pair_case(work, "pair_4096_4096", 4096, 4096, 11, 1 << 14),
        "pair_17_100": lambda: pair_case(work, "pair_17_100", 100, 17, 13, 64),
    }
    for name, fn in cases.items():
        np.savez_compressed(os.path.join(a.out, f"{name}.npz"), **fn())
        print("wrote", name)


if __name__ == "__main__":
    main()

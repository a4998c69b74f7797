"""Preprocessing drop-in: raw edge lists and JSONL corpora -> the reference's
`.bin` inputs for the triangle-count, set-similarity and retrieval paths.

Restates the rules of the reference's preprocess/ pipeline so that a user
with the reference's datasets produces byte-identical inputs through this
package (no torch, no GPU):

* `.bin` framing (preprocess/util.py:12-20): u64 element count + int32
  payload, or one bare int32;
* graph edge files (preprocessor.py:57-123): every `*.edges` / `*.txt`
  file of a folder in name order; lines starting with '#' skipped; the first
  two whitespace-separated integers of a line are an edge; self-loops and
  unparsable lines dropped;
* node ids (preprocessor.py:41-55, remap_nodes): distinct ids sorted and
  numbered densely, then scattered by i -> (i * step) mod N with step the
  first integer >= 10007 coprime to N;
* adjacency (preprocessor.py:129-145): symmetrised, de-duplicated, sorted;
* TC (preprocessor.py:187-210): row u keeps its neighbours v > u (oriented
  by id) -> csr_offsets_tri.bin, csr_cols_tri.bin, num_nodes_tri.bin,
  num_edges_tri.bin;
* SSS (preprocessor.py:161-184): the whole symmetric adjacency ->
  csr_offsets.bin, csr_cols.bin, vertexs.bin, num_nodes.bin, num_edges.bin;
* IR (preprocessor.py:212-380, util.py:55-66 and :122-134): tokens = the
  whitespace-split words of a document's "text" with every character that
  is neither a word character nor whitespace removed, lower-cased, empty ones
  dropped; terms numbered in sorted order; posting lists = sorted doc ids;
  the default high-frequency filter (strategy 3) removes the
  int(V * 0.0001) terms of lowest idf = log((D + 1) / (1 + df)) (stable
  order) and renumbers the rest in sorted-word order; a query keeps its
  known terms once each, ordered by (df, term id); finally every doc id x
  in the index becomes (x * step^2 mod D) with step the first integer >=
  10007 coprime to D (revise_inverted_index), so posting lists are no
  longer sorted -> inverted_index_offsets.bin, inverted_index.bin,
  inverted_index_num.bin, query.bin, query_offsets.bin, query_num.bin.

    python -m reset_b200.preprocess tc|sss|ir <dataset folder> [<output folder>]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import struct
import sys
from typing import Dict, Iterable, List, Tuple

import numpy as np

# ------------------------------------------------------------ .bin files --


def write_arr_bin(path: str, values) -> None:
    a = np.ascontiguousarray(np.asarray(values, dtype=np.int64))
    if a.size and (a.min() < -2**31 or a.max() >= 2**31):
        raise ValueError(f"{path}: values do not fit int32")
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", a.size))
        f.write(a.astype("<i4").tobytes())


def write_int_bin(path: str, value: int) -> None:
    with open(path, "wb") as f:
        f.write(struct.pack("<i", int(value)))


def read_arr_bin(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        (n,) = struct.unpack("<Q", f.read(8))
        return np.frombuffer(f.read(4 * n), dtype="<i4").astype(np.int32)


def read_int_bin(path: str) -> int:
    with open(path, "rb") as f:
        return struct.unpack("<i", f.read(4))[0]


# ----------------------------------------------------------------- graphs --


def _coprime_step(n: int, start: int = 10007) -> int:
    step = start
    while math.gcd(step, n) != 1:
        step += 1
    return step


def parse_edge_lines(lines: Iterable[str]) -> Tuple[List[int], List[int]]:
    """Edges of one file: first two integers of every non-comment line,
    self-loops dropped."""
    us, vs = [], []
    for line in lines:
        if not line or line[0] == "#":
            continue
        parts = line.split(None, 2)
        if len(parts) < 2:
            continue
        try:
            u, v = int(parts[0]), int(parts[1])
        except ValueError:
            continue
        if u != v:
            us.append(u)
            vs.append(v)
    return us, vs


def read_edge_folder(path: str) -> Tuple[np.ndarray, np.ndarray, int]:
    """All `.edges` / `.txt` files of `path` in name order -> (u, v) remapped
    to [0, N) by the reference's scatter, and N."""
    us: List[int] = []
    vs: List[int] = []
    for name in sorted(os.listdir(path)):
        if not (name.endswith(".edges") or name.endswith(".txt")):
            continue
        p = os.path.join(path, name)
        if os.path.getsize(p) == 0:
            continue
        with open(p, "r", encoding="utf-8", errors="ignore") as f:
            u, v = parse_edge_lines(f)
        us.extend(u)
        vs.extend(v)
    if not us:
        return np.zeros(0, np.int64), np.zeros(0, np.int64), 0
    # raw ids may exceed 64 bits in principle; real edge lists do not
    u = np.array(us, dtype=np.int64)
    v = np.array(vs, dtype=np.int64)
    nodes, inv = np.unique(np.concatenate([u, v]), return_inverse=True)
    n = int(nodes.size)
    step = _coprime_step(n)
    perm = (np.arange(n, dtype=np.int64) * step) % n
    inv = perm[inv]
    return inv[:u.size], inv[u.size:], n


def symmetric_adjacency(u: np.ndarray, v: np.ndarray, n: int) -> Tuple[np.ndarray, np.ndarray]:
    """Symmetrised, de-duplicated, sorted CSR -> (offsets[n+1], cols)."""
    src = np.concatenate([u, v])
    dst = np.concatenate([v, u])
    key = np.unique(src * n + dst)
    src, dst = key // n, key % n
    off = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(src, minlength=n), out=off[1:])
    return off, dst


def export_tc(folder: str, out: str) -> Dict[str, int]:
    u, v, n = read_edge_folder(folder)
    off, cols = symmetric_adjacency(u, v, n)
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
    keep = cols > src
    toff = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(src[keep], minlength=n), out=toff[1:])
    os.makedirs(out, exist_ok=True)
    write_arr_bin(os.path.join(out, "csr_cols_tri.bin"), cols[keep])
    write_arr_bin(os.path.join(out, "csr_offsets_tri.bin"), toff)
    write_int_bin(os.path.join(out, "num_nodes_tri.bin"), n)
    write_int_bin(os.path.join(out, "num_edges_tri.bin"), int(keep.sum()))
    return {"nodes": n, "edges": int(keep.sum())}


def export_sss(folder: str, out: str) -> Dict[str, int]:
    u, v, n = read_edge_folder(folder)
    off, cols = symmetric_adjacency(u, v, n)
    os.makedirs(out, exist_ok=True)
    write_arr_bin(os.path.join(out, "csr_cols.bin"), cols)
    write_arr_bin(os.path.join(out, "csr_offsets.bin"), off)
    write_arr_bin(os.path.join(out, "vertexs.bin"),
                  np.repeat(np.arange(n, dtype=np.int64), np.diff(off)))
    write_int_bin(os.path.join(out, "num_nodes.bin"), n)
    write_int_bin(os.path.join(out, "num_edges.bin"), int(cols.size))
    return {"nodes": n, "edges": int(cols.size)}


# -------------------------------------------------------------- retrieval --

_PUNCT = re.compile(r"[^\w\s]")


def tokenize(text: str) -> List[str]:
    out = []
    for tok in text.split():
        tok = _PUNCT.sub("", tok).lower()
        if tok:
            out.append(tok)
    return out


def _iter_jsonl(path: str):
    with open(path, "r", encoding="utf-8", errors="ignore") as f:
        for line in f:
            line = line.strip()
            if not line:
                continue
            try:
                yield json.loads(line)
            except json.JSONDecodeError:
                continue


def build_index(corpus: str, filter_ratio: float = 0.0001):
    """-> (word -> term id, offsets[T+1], doc ids (sorted per term), D)."""
    docs = [set(tokenize(d.get("text", ""))) for d in _iter_jsonl(corpus)]
    words = sorted(set().union(*docs)) if docs else []
    wid = {w: i for i, w in enumerate(words)}
    postings: List[List[int]] = [[] for _ in words]
    for d, toks in enumerate(docs):
        for t in toks:
            postings[wid[t]].append(d)
    D = len(docs)
    # strategy 3: drop the int(V * ratio) terms of lowest idf, stable order
    idf = [math.log((D + 1) / (1 + len(p))) for p in postings]
    order = sorted(range(len(idf)), key=lambda i: idf[i])
    removed = set(order[:int(len(order) * filter_ratio)])
    kept = [w for w in words if wid[w] not in removed]
    new_wid = {w: i for i, w in enumerate(kept)}
    off = np.zeros(len(kept) + 1, np.int64)
    lists = []
    for i, w in enumerate(kept):
        p = sorted(set(postings[wid[w]]))
        lists.append(p)
        off[i + 1] = off[i] + len(p)
    docs_arr = np.array([x for p in lists for x in p], dtype=np.int64)
    return new_wid, off, docs_arr, D


def build_queries(queries: str, wid: Dict[str, int], off: np.ndarray):
    df = np.diff(off)
    q: List[int] = []
    qoff = [0]
    for d in _iter_jsonl(queries):
        ids = {wid[w] for w in tokenize(d.get("text", "")) if w in wid}
        q.extend(sorted(ids, key=lambda t: (int(df[t]), t)))
        qoff.append(len(q))
    return np.array(q, np.int64), np.array(qoff, np.int64)


def scatter_doc_ids(docs: np.ndarray, D: int) -> np.ndarray:
    if D == 0:
        return docs
    step = _coprime_step(D)
    step2 = (step * step) % D
    return (docs * step2) % D


def export_ir(folder: str, out: str) -> Dict[str, int]:
    wid, off, docs, D = build_index(os.path.join(folder, "corpus.jsonl"))
    q, qoff = build_queries(os.path.join(folder, "queries.jsonl"), wid, off)
    docs = scatter_doc_ids(docs, D)
    os.makedirs(out, exist_ok=True)
    write_arr_bin(os.path.join(out, "inverted_index_offsets.bin"), off)
    write_arr_bin(os.path.join(out, "inverted_index.bin"), docs)
    write_int_bin(os.path.join(out, "inverted_index_num.bin"), off.size - 1)
    write_arr_bin(os.path.join(out, "query.bin"), q)
    write_arr_bin(os.path.join(out, "query_offsets.bin"), qoff)
    write_int_bin(os.path.join(out, "query_num.bin"), qoff.size - 1)
    return {"terms": int(off.size - 1), "docs": D, "queries": int(qoff.size - 1)}


EXPORTERS = {"tc": export_tc, "sss": export_sss, "ir": export_ir}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("mode", choices=sorted(EXPORTERS))
    ap.add_argument("folder", help="dataset folder (edge files, or corpus.jsonl + queries.jsonl)")
    ap.add_argument("out", nargs="?", help="output folder (default: the dataset folder)")
    a = ap.parse_args(argv)
    info = EXPORTERS[a.mode](a.folder, a.out or a.folder)
    print(json.dumps({"mode": a.mode, **info}))
    return 0


if __name__ == "__main__":
    sys.exit(main())

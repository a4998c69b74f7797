#!/usr/bin/env python
"""Golden vectors for the preprocessing drop-in (reset_b200/preprocess.py):
small seeded raw inputs -- edge-list folders with comments, tabs, weights,
duplicates, self-loops and unparsable lines; a JSONL corpus and queries with
punctuation, mixed case, unicode and unknown words -- run through the
reference's own preprocess/preprocessor.py (imported from the reference
checkout, outputs written to a temporary folder), stored with the inputs in
tests/golden/preprocess_small.npz.  Test infrastructure; needs the
reference checkout ($RESET_REFERENCE, default /root/reference).

    python tests/golden/make_preprocess_golden.py
"""
import io
import json
import os
import sys
import tempfile
from contextlib import redirect_stdout, redirect_stderr

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("RESET_REFERENCE", "/root/reference")


def edge_folder_files(rng, n_files, n_edges, id_space):
    """{file name: text} of one raw graph folder."""
    files = {}
    for k in range(n_files):
        lines = ["# synthetic edge list", "% not a comment marker here"]
        for _ in range(n_edges):
            u, v = (int(x) for x in rng.integers(0, id_space, 2))
            r = rng.random()
            if r < 0.05:
                v = u                                   # self-loop
            if r < 0.10:
                lines.append(f"{u}\t{v}")
            elif r < 0.15:
                lines.append(f"{u} {v} {rng.integers(1, 9)}")   # weighted
            elif r < 0.18:
                lines.append(f"  {u}  {v}")
            elif r < 0.20:
                lines.append(f"{u} x{v}")               # unparsable
            else:
                lines.append(f"{u} {v}")
        lines.append("")
        files[f"part{k}.edges" if k % 2 == 0 else f"part{k}.txt"] = "\n".join(lines)
    files["ignored.csv"] = "1 2\n3 4\n"
    return files


WORDS = ["Apple", "banana", "cherry", "delta", "echo", "fox", "golf", "hotel", "india",
         "juliet", "kilo", "lima", "mike", "nov", "oscar", "papa", "Québec", "romeo",
         "sierra", "tango", "über", "victor", "whisky", "x-ray", "yankee", "zulu", "the",
         "a", "of", "and"]


def corpus_lines(rng, n_docs):
    out = []
    p = 1.0 / np.arange(1, len(WORDS) + 1) ** 0.8
    p /= p.sum()
    for i in range(n_docs):
        k = int(rng.integers(1, 14))
        toks = [WORDS[j] for j in rng.choice(len(WORDS), size=k, p=p)]
        toks = [t + rng.choice(["", ",", ".", "!", "'s", "?"]) for t in toks]
        out.append(json.dumps({"_id": str(i), "text": " ".join(toks)}))
        if i % 17 == 0:
            out.append("")                              # blank line
    out.append("{not json")
    return "\n".join(out) + "\n"


def big_vocab_corpus(rng, n_docs, vocab):
    """A corpus whose vocabulary exceeds 10,000 words, so the reference's
    default high-frequency filter (int(V * 0.0001) terms) removes some."""
    out = []
    common = ["the", "of", "and"]
    for i in range(n_docs):
        k = int(rng.integers(3, 30))
        toks = [f"w{int(x)}" for x in rng.integers(0, vocab, size=k)]
        toks += [c for c in common if rng.random() < 0.9]
        out.append(json.dumps({"text": " ".join(toks)}))
    return "\n".join(out) + "\n"


def query_lines(rng, n_queries):
    out = []
    for i in range(n_queries):
        k = int(rng.integers(1, 6))
        toks = [WORDS[j] for j in rng.integers(0, len(WORDS), size=k)] + ["unknownword"]
        out.append(json.dumps({"_id": f"q{i}", "text": " ".join(toks) + "?"}))
    return "\n".join(out) + "\n"


def write_files(folder, files):
    os.makedirs(folder, exist_ok=True)
    for name, text in files.items():
        with open(os.path.join(folder, name), "w", encoding="utf-8") as f:
            f.write(text)


def main():
    sys.path.insert(0, os.path.join(REF, "preprocess"))
    import preprocessor as P   # the reference's own module
    from util import read_arr_bin, read_int_bin

    rng = np.random.default_rng(0x5EED0077)
    graph = edge_folder_files(rng, 3, 400, 300)
    corpus = corpus_lines(rng, 600)
    queries = query_lines(rng, 80)
    big_corpus = big_vocab_corpus(rng, 2500, 24000)
    big_queries = "\n".join(json.dumps({"text": f"w{a} w{b} the of"})
                            for a, b in rng.integers(0, 24000, size=(60, 2))) + "\n"
    rec = {"graph_files": np.array(json.dumps(graph)),
           "corpus": np.array(corpus), "queries": np.array(queries),
           "big_corpus": np.array(big_corpus), "big_queries": np.array(big_queries)}
    with tempfile.TemporaryDirectory() as tmp:
        gdir = os.path.join(tmp, "graph")
        write_files(gdir, graph)
        sink = io.StringIO()
        for mode, names in [("tc", ["csr_cols_tri", "csr_offsets_tri"]),
                            ("sss", ["csr_cols", "csr_offsets", "vertexs"])]:
            out = os.path.join(tmp, "out_" + mode)
            with redirect_stdout(sink), redirect_stderr(sink):
                P.processor_factory(mode, out).build_all(gdir)
            for nm in names:
                rec[f"{mode}_{nm}"] = np.array(read_arr_bin(os.path.join(out, nm + ".bin")), np.int32)
            for nm in ["num_nodes_tri", "num_edges_tri"] if mode == "tc" else ["num_nodes", "num_edges"]:
                rec[f"{mode}_{nm}"] = np.array(read_int_bin(os.path.join(out, nm + ".bin")))
        for tag, c, q in [("ir", corpus, queries), ("irbig", big_corpus, big_queries)]:
            idir = os.path.join(tmp, tag)
            write_files(idir, {"corpus.jsonl": c, "queries.jsonl": q})
            out = os.path.join(tmp, "out_" + tag)
            with redirect_stdout(sink), redirect_stderr(sink):
                P.processor_factory("ir", out).build_all(idir)
            for nm in ["inverted_index_offsets", "inverted_index", "query", "query_offsets"]:
                rec[f"{tag}_{nm}"] = np.array(read_arr_bin(os.path.join(out, nm + ".bin")),
                                              np.int32)
            for nm in ["inverted_index_num", "query_num"]:
                rec[f"{tag}_{nm}"] = np.array(read_int_bin(os.path.join(out, nm + ".bin")))
    np.savez_compressed(os.path.join(HERE, "preprocess_small.npz"), **rec)
    print({k: (v.shape if v.ndim else v.item() if v.dtype != object else "") for k, v in rec.items()
           if k not in ("graph_files", "corpus", "queries", "big_corpus", "big_queries")})


if __name__ == "__main__":
    main()

"""The preprocessing drop-in (reset_b200/preprocess.py) against the outputs
of the reference's own preprocess/preprocessor.py on the same raw inputs
(tests/golden/preprocess_small.npz, made by make_preprocess_golden.py):
TC and SSS graph files, and IR index + queries -- including the
high-frequency filter (a vocabulary above 10,000 words) and the doc-id
scatter that leaves posting lists unsorted.  CPU only."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

from reset_b200 import preprocess as PP


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(os.path.join(GOLDEN, "preprocess_small.npz")))


def _write(folder, files):
    os.makedirs(folder, exist_ok=True)
    for name, text in files.items():
        with open(os.path.join(folder, name), "w", encoding="utf-8") as f:
            f.write(text)


def test_graph_exports_equal_reference(golden, tmp_path):
    src = tmp_path / "graph"
    _write(src, json.loads(str(golden["graph_files"])))
    for mode, arrays, scalars in [
            ("tc", ["csr_cols_tri", "csr_offsets_tri"], ["num_nodes_tri", "num_edges_tri"]),
            ("sss", ["csr_cols", "csr_offsets", "vertexs"], ["num_nodes", "num_edges"])]:
        out = tmp_path / ("out_" + mode)
        PP.EXPORTERS[mode](str(src), str(out))
        for nm in arrays:
            got = PP.read_arr_bin(str(out / (nm + ".bin")))
            assert np.array_equal(got, golden[f"{mode}_{nm}"]), (mode, nm)
        for nm in scalars:
            assert PP.read_int_bin(str(out / (nm + ".bin"))) == int(golden[f"{mode}_{nm}"])


@pytest.mark.parametrize("tag,corpus,queries", [("ir", "corpus", "queries"),
                                                ("irbig", "big_corpus", "big_queries")])
def test_ir_export_equals_reference(golden, tmp_path, tag, corpus, queries):
    src = tmp_path / tag
    _write(src, {"corpus.jsonl": str(golden[corpus]), "queries.jsonl": str(golden[queries])})
    out = tmp_path / "out"
    info = PP.export_ir(str(src), str(out))
    for nm in ["inverted_index_offsets", "inverted_index", "query", "query_offsets"]:
        got = PP.read_arr_bin(str(out / (nm + ".bin")))
        assert np.array_equal(got, golden[f"{tag}_{nm}"]), nm
    for nm in ["inverted_index_num", "query_num"]:
        assert PP.read_int_bin(str(out / (nm + ".bin"))) == int(golden[f"{tag}_{nm}"])
    if tag == "irbig":
        # the filter removed int(V * 0.0001) >= 1 term of the 19,630-word vocabulary
        assert info["terms"] < 19630


def test_ir_posting_lists_are_scattered_not_sorted(golden):
    """After revise_inverted_index the doc ids of a term are a permutation
    image of a sorted list: distinct, but in general not ascending."""
    off, docs = golden["ir_inverted_index_offsets"], golden["ir_inverted_index"]
    unsorted = 0
    for t in range(off.size - 1):
        row = docs[off[t]:off[t + 1]]
        assert np.unique(row).size == row.size
        unsorted += int(np.any(np.diff(row) < 0))
    assert unsorted > 0


def test_tc_export_feeds_the_checker(golden, tmp_path, oracle_mod):
    """The exported TC files are a CSR the oracle counts: by-id orientation
    (v > u) gives the same triangles as the symmetric SSS adjacency / 6."""
    off = golden["tc_csr_offsets_tri"]
    cols = golden["tc_csr_cols_tri"]
    src = np.repeat(np.arange(off.size - 1), np.diff(off))
    assert np.all(cols > src)
    soff, scols = golden["sss_csr_offsets"], golden["sss_csr_cols"]
    n = soff.size - 1
    adj = [set(scols[soff[u]:soff[u + 1]].tolist()) for u in range(n)]
    brute = sum(len(adj[u] & adj[v]) for u in range(n) for v in adj[u] if v > u) // 3
    assert oracle_mod.tc_merge(off.astype(np.int32), cols.astype(np.int32)) == brute


def test_bin_roundtrip_and_range(tmp_path):
    p = str(tmp_path / "a.bin")
    PP.write_arr_bin(p, [0, -1, 2**31 - 1])
    assert PP.read_arr_bin(p).tolist() == [0, -1, 2**31 - 1]
    with pytest.raises(ValueError):
        PP.write_arr_bin(p, [2**31])
    PP.write_int_bin(p, -7)
    assert PP.read_int_bin(p) == -7

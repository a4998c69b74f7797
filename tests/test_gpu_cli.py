"""The C++ drop-in drivers (reset_b200/bin/*) run on the reference's own input
file formats and print the reference's result lines; their numbers must
equal the reference's outputs stored in the golden fixtures."""
import os
import re
import struct
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu
BIN = os.path.join(ROOT, "reset_b200", "bin")


def write_arr(path, a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", a.size))
        f.write(a.tobytes())


def write_int(path, v):
    with open(path, "wb") as f:
        f.write(struct.pack("<i", int(v)))


def run(exe, *args):
    r = subprocess.run([os.path.join(BIN, exe), *map(str, args)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.mark.parametrize("name", ["tc_s10", "tc_s11_a05_b3"])
def test_reset_tc_cli(cuda, libreset, tmp_path, name):
    g = load(name)
    d = str(tmp_path)
    write_arr(f"{d}/csr_offsets_tri.bin", g["off"])
    write_arr(f"{d}/csr_cols_tri.bin", g["cols"])
    write_int(f"{d}/num_nodes_tri.bin", g["off"].size - 1)
    write_int(f"{d}/num_edges_tri.bin", g["cols"].size)
    out = run("reset_tc", d, f"--alpha={float(g['alpha'])}", f"--bucket={int(g['bucket'])}")
    ref = g["ref_meta"]
    assert int(re.search(r"Normal hash - Triangles: (\d+)", out).group(1)) == ref[2]
    assert int(re.search(r"Hierarchical hash - Triangles: (\d+)", out).group(1)) == ref[3]
    assert int(re.search(r"Max length: (\d+)", out).group(1)) == ref[0]
    assert int(re.search(r"Total buckets: (\d+)", out).group(1)) == ref[1]
    assert "[RESET]" in out and "[Native]" in out


@pytest.mark.parametrize("name", ["sss_s9_t025", "sss_s9_t07"])
def test_reset_sss_cli(cuda, libreset, tmp_path, name):
    g = load(name)
    d = str(tmp_path)
    off, cols = g["off"], g["cols"]
    n = off.size - 1
    write_arr(f"{d}/csr_offsets.bin", off)
    write_arr(f"{d}/csr_cols.bin", cols)
    write_arr(f"{d}/vertexs.bin", np.repeat(np.arange(n, dtype=np.int32), np.diff(off)))
    write_int(f"{d}/num_nodes.bin", n)
    write_int(f"{d}/num_edges.bin", cols.size)
    out = run("reset_sss", d, f"--thr={float(g['thr'])}")
    got = int(re.search(r"greater than threshold: (\d+)", out).group(1))
    assert got == g["ref_meta"][2] == int(g["ref_results_normal"].sum())


def test_reset_ir_cli(cuda, libreset, tmp_path):
    g = load("ir_small")
    d = str(tmp_path)
    write_arr(f"{d}/inverted_index_offsets.bin", g["toff"])
    write_arr(f"{d}/inverted_index.bin", g["docs"])
    write_int(f"{d}/inverted_index_num.bin", g["toff"].size - 1)
    write_arr(f"{d}/query.bin", g["query"])
    write_arr(f"{d}/query_offsets.bin", g["qoff"])
    write_int(f"{d}/query_num.bin", g["qoff"].size - 1)
    out = run("reset_ir", d)
    got = int(re.search(r"Total result count: (\d+)", out).group(1))
    assert got == int(g["ref_count_normal"].sum()) == int(g["ref_count_hier"].sum())
    # the same queries through the native serving driver, burst and Poisson
    for extra in ([], ["--rate=20000", "--streams=2", "--max-batch=8"]):
        out = run("reset_serve_ir", d, *extra)
        served = int(re.search(r"Total result count: (\d+)", out).group(1))
        assert served == got
        assert re.search(r"served: [0-9.]+ queries/s, latency p50", out)


@pytest.mark.parametrize("name", ["pair_1000_3000", "pair_4096_4096", "pair_17_100"])
def test_reset_intersection_cli(cuda, libreset, tmp_path, name):
    g = load(name)
    write_arr(f"{tmp_path}/a.bin", g["a"])
    write_arr(f"{tmp_path}/b.bin", g["b"])
    out = run("reset_intersection", "--files", f"{tmp_path}/a.bin", f"{tmp_path}/b.bin")
    got = int(re.search(r"Intersection Result Count: (\d+)", out).group(1))
    assert got == g["ref_meta"][1]


def _write_smog_graph(d, prefix, off, cols):
    """SMOG's graph folder files (SMOG/SMOG_hie/common_hie.cu:61-129): raw
    int32 arrays, no header."""
    n = off.size - 1
    vtx = np.repeat(np.arange(n, dtype=np.int32), np.diff(off))
    for name, a in (("begin", off), ("adjacent", cols), ("vertex", vtx),
                    ("md", [int(np.diff(off).max())])):
        np.asarray(a, dtype=np.int32).tofile(f"{d}/{prefix}{name}.bin")


def test_reset_smog_cli(cuda, libreset, oracle_mod, tmp_path):
    """SMOG's executable interface: its graph folder (oriented files for the
    clique patterns, generic_ ones for the rest), its positional arguments
    and its result line, for every pattern of its table, against the
    oracle's count by definition."""
    from reset_b200.api import PATTERNS
    d = str(tmp_path)
    o_off, o_cols = oracle_mod.rmat_graph(9, 16, 0x5EED5309, oriented=True)
    s_off, s_cols = oracle_mod.rmat_graph(9, 16, 0x5EED5309, oriented=False)
    _write_smog_graph(d, "", o_off, o_cols)
    _write_smog_graph(d, "generic_", s_off, s_cols)
    for name, p in PATTERNS.items():
        off, cols = (o_off, o_cols) if p.graph == "oriented" else (s_off, s_cols)
        want = oracle_mod.pattern_count(off, cols, p.k, p.flags, p.offsets, p.backward,
                                        p.restriction, p.reuse)
        out = run("reset_smog", d, name, 1, 0.2, 5, 1024, 216, 1)
        assert int(re.search(rf"{name} count is (\d+)", out).group(1)) == want, name
        assert f"graph vertex number is : {off.size - 1}" in out
        assert re.search(r"Hierarchical time: [0-9.e+-]+ ms", out)

"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Integer work, so every comparison is exact: generated graphs, table layout
(byte for byte), hash-ordered rows, triangle counts, set-similarity flags and
intersection sizes, retrieval result lists and raw intersection counts.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def R(cuda, libreset):
    from reset_b200 import api
    return api


def dev(x, torch):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def host(t):
    return t.detach().cpu().numpy()


# ------------------------------------------------------------- generator --

@pytest.mark.parametrize("scale,oriented,relabel", [
    (6, True, True), (10, True, True), (12, False, True), (16, True, True),
    (10, True, False), (12, False, False), (1, True, True), (2, False, True)])
def test_gen_rmat_matches_oracle(R, cuda, oracle_mod, scale, oriented, relabel):
    seed = 0x5EED0000 + scale
    off, cols = R.gen_rmat(scale, 16, seed, oriented=oriented, relabel=relabel)
    o_off, o_cols = oracle_mod.rmat_graph(scale, 16, seed, oriented=oriented, relabel=relabel)
    assert np.array_equal(host(off), o_off)
    assert np.array_equal(host(cols), o_cols)


# ----------------------------------------------------------- table build --

def _synthetic_csr(rng, sizes, universe):
    off = np.zeros(len(sizes) + 1, np.int32)
    off[1:] = np.cumsum(sizes)
    rows = [np.sort(rng.choice(universe, size=s, replace=False)) if s else np.zeros(0, np.int64)
            for s in sizes]
    elems = np.concatenate(rows).astype(np.int32) if off[-1] else np.zeros(0, np.int32)
    return off, elems


def _check_table(R, cuda, O, off, elems, alpha, bucket, hier):
    t = R.Table(dev(off, cuda), dev(elems, cuda), alpha=alpha, bucket=bucket,
                hierarchical=hier, hash_order=True)
    t.check()
    ot = O.Table(off, elems, alpha=alpha, bucket=bucket, hier=hier)
    slots, ln, o64 = t.tensors()
    assert t.bucket_num == ot.bucket_num and t.max_len == ot.max_len
    assert np.array_equal(host(ln), ot.len)
    assert np.array_equal(host(o64), ot.off64)
    assert np.array_equal(host(slots), ot.table), "table layout differs from CSR-order insertion"
    assert np.array_equal(host(t.hash_order), ot.hash_order())
    assert np.array_equal(host(t.csr_hash_order()), ot.hash_order())
    return t, ot


@pytest.mark.parametrize("hier", [True, False])
@pytest.mark.parametrize("alpha,bucket", [(1.0, 1), (0.9, 2), (0.2, 5)])
def test_table_layout_huge_sets(R, cuda, oracle_mod, hier, alpha, bucket):
    """Sets of 2^16 keys and more are built in parallel (final fills by a
    scan, clusters replayed in CSR order) and must equal sequential CSR-order
    insertion byte for byte: dense tables (long clusters), repeated keys,
    keys crowding the last buckets (a cluster that wraps to bucket 0), and
    small sets around them."""
    rng = np.random.default_rng(11)
    big = rng.integers(0, 1 << 24, 70000)
    big[:20000] = big[0]               # one key repeated: a cluster of 20000 keys
    big[20000:23000] = (1 << 20) - 1 - rng.integers(0, 4, 3000)  # high buckets
    rng.shuffle(big)
    other = rng.integers(0, 1 << 20, 80000)
    rows = [np.sort(rng.choice(1 << 20, 40, replace=False)), big, other,
            np.zeros(0, np.int64), np.sort(rng.choice(1 << 20, 300, replace=False))]
    off = np.zeros(len(rows) + 1, np.int32)
    off[1:] = np.cumsum([r.size for r in rows])
    elems = np.concatenate(rows).astype(np.int32)
    _check_table(R, cuda, oracle_mod, off, elems, alpha, bucket, hier)


@pytest.mark.parametrize("hier", [True, False])
@pytest.mark.parametrize("alpha,bucket", [(0.2, 5), (0.5, 3), (1.0, 1), (0.1, 9), (0.25, 4)])
def test_table_layout_rmat(R, cuda, oracle_mod, hier, alpha, bucket):
    off, cols = oracle_mod.rmat_graph(12, 16, 0x5EED0012, oriented=False)
    _check_table(R, cuda, oracle_mod, off, cols, alpha, bucket, hier)


@pytest.mark.parametrize("hier", [True, False])
def test_table_layout_ragged_sizes(R, cuda, oracle_mod, hier):
    """Empty sets, 1-element sets, the thread/warp boundary (8/9), exact
    powers of two (the strict next-power quirk), tile-sized and big sets,
    and one set whose fill counts do not fit shared memory."""
    rng = np.random.default_rng(5)
    sizes = [0, 1, 0, 5, 8, 9, 16, 31, 32, 33, 100, 0, 1000, 1023, 1024, 1025, 4000,
             70000, 3, 0, 2]
    off, elems = _synthetic_csr(rng, sizes, 1 << 22)
    _check_table(R, cuda, oracle_mod, off, elems, 0.2, 5, hier)


def test_table_layout_collisions(R, cuda, oracle_mod):
    """Keys crowded into few buckets: bucket overflow, spill chains and the
    wrap-around from the last bucket to bucket 0."""
    rng = np.random.default_rng(9)
    sizes = [40, 200, 7, 64, 500]
    off = np.zeros(len(sizes) + 1, np.int32)
    off[1:] = np.cumsum(sizes)
    parts = []
    for s in sizes:
        # multiples of a large power of two all share a normal-hash bucket;
        # values near the top of the id range crowd the last hierarchical bucket
        base = rng.choice(4096, size=s, replace=False).astype(np.int64)
        parts.append(np.where(np.arange(s) % 2 == 0, base * 1024, (1 << 30) - 1 - base))
    elems = np.concatenate(parts).astype(np.int32)
    for hier in (True, False):
        for alpha, bucket in [(0.2, 5), (1.0, 2), (1.0, 1)]:
            _check_table(R, cuda, oracle_mod, off, elems, alpha, bucket, hier)


def test_table_empty_inputs(R, cuda, oracle_mod):
    off = np.zeros(4, np.int32)
    elems = np.zeros(0, np.int32)
    _check_table(R, cuda, oracle_mod, off, elems, 0.2, 5, True)


def test_table_duplicates_inserted_twice(R, cuda, oracle_mod):
    # hashtable.cu inserts duplicates as separate slots (no dedupe)
    off = np.array([0, 6, 6, 9], np.int32)
    elems = np.array([3, 3, 3, 7, 7, 11, 2, 2, 2], np.int32)
    _check_table(R, cuda, oracle_mod, off, elems, 0.2, 5, True)
    _check_table(R, cuda, oracle_mod, off, elems, 1.0, 1, False)


# -------------------------------------------------------------------- TC --

@pytest.mark.parametrize("scale", [8, 12, 16])
@pytest.mark.parametrize("hier", [True, False])
def test_tc_count_matches_oracle(R, cuda, oracle_mod, scale, hier):
    off, cols = oracle_mod.rmat_graph(scale, 16, 0x5EED0000 + scale, oriented=True)
    want = oracle_mod.tc_merge(off, cols)
    doff, dcols = dev(off, cuda), dev(cols, cuda)
    t = R.Table(doff, dcols, hierarchical=hier, hash_order=True)
    assert R.tc_count(t, doff, dcols) == want
    assert R.tc_count(t, doff, t.hash_order) == want
    # same offsets in a different buffer: descriptors are rebuilt
    assert R.tc_count(t, doff.clone(), t.hash_order) == want
    t.check()
    ot = oracle_mod.Table(off, cols, hier=hier)
    assert oracle_mod.tc_hash(ot, ot.hash_order()) == want


def test_tc_params_and_generator(R, cuda, oracle_mod):
    off, cols = R.gen_rmat(14, 16, 0xABCDEF, oriented=True)
    o_off, o_cols = host(off), host(cols)
    want = oracle_mod.tc_merge(o_off, o_cols)
    for alpha, bucket in [(0.2, 5), (0.5, 2), (1.0, 1)]:
        for hier in (True, False):
            t = R.Table(off, cols, alpha=alpha, bucket=bucket, hierarchical=hier, hash_order=True)
            assert R.tc_count(t, off, t.hash_order) == want


def test_tc_empty_graph(R, cuda):
    off = cuda.zeros(9, dtype=cuda.int32, device="cuda")
    cols = cuda.zeros(0, dtype=cuda.int32, device="cuda")
    t = R.Table(off, cols)
    assert R.tc_count(t, off, cols) == 0


# ------------------------------------------------------------------- SSS --

@pytest.mark.parametrize("hier", [True, False])
def test_sss_graph_pairs(R, cuda, oracle_mod, hier):
    """Reference SSS setting: pairs are the CSR entries (sss.cu:104-105)."""
    off, cols = oracle_mod.rmat_graph(11, 16, 0x5EED0111, oriented=False)
    n = off.size - 1
    pa = np.repeat(np.arange(n, dtype=np.int32), np.diff(off))
    pb = cols
    doff, dcols, dpa, dpb = (dev(x, cuda) for x in (off, cols, pa, pb))
    t = R.Table(doff, dcols, hierarchical=hier)
    ot = oracle_mod.Table(off, cols, hier=hier)
    for num, den in [(7, 10), (1, 4), (0, 1), (1, 1)]:
        f, i = R.sss(t, doff, dcols, dpa, dpb, num, den)
        of, oi = oracle_mod.sss(ot, pa, pb, mode=1, num=num, den=den)
        assert np.array_equal(host(i), oi)
        assert np.array_equal(host(f), of)
    for thr in [0.25, 0.7, 0.5, 1.0 / 3.0]:
        f, i = R.sss_float(t, doff, dcols, dpa, dpb, thr)
        of, oi = oracle_mod.sss(ot, pa, pb, mode=0, thr=thr)
        assert np.array_equal(host(f), of)


def test_sss_random_pairs_and_empty_sets(R, cuda, oracle_mod):
    rng = np.random.default_rng(3)
    sizes = rng.integers(0, 300, size=500)
    sizes[::17] = 0
    off, elems = _synthetic_csr(rng, sizes, 2000)
    P = 20000
    pa = rng.integers(0, 500, size=P).astype(np.int32)
    pb = rng.integers(0, 500, size=P).astype(np.int32)
    pb[:50] = pa[:50]  # identical sets: Jaccard 1 (or U = 0 for empty sets)
    doff, de, dpa, dpb = (dev(x, cuda) for x in (off, elems, pa, pb))
    for hier in (True, False):
        t = R.Table(doff, de, hierarchical=hier, hash_order=True)
        ot = oracle_mod.Table(off, elems, hier=hier)
        f, i = R.sss(t, doff, t.hash_order, dpa, dpb, 7, 10)
        of, oi = oracle_mod.sss(ot, pa, pb, mode=1, num=7, den=10)
        assert np.array_equal(host(i), oi) and np.array_equal(host(f), of)
        f, i = R.sss_float(t, doff, de, dpa, dpb, 0.7)
        of, _ = oracle_mod.sss(ot, pa, pb, mode=0, thr=0.7)
        assert np.array_equal(host(f), of)


@pytest.mark.parametrize("hier", [True, False])
def test_sss_pair_methods_agree(R, cuda, oracle_mod, hier):
    """The owner-grouped pair path (tables staged in shared memory, every bin:
    CTA units with more than 512 probers, warp owners, direct owners with
    tables too large to stage) and the pair-flattened path give the oracle's
    sizes and decisions, integer and float rule, with and without sizes, on
    sets with repeated entries (the probe direction matters there)."""
    rng = np.random.default_rng(11)
    sizes = rng.integers(0, 120, size=3000)
    sizes[::23] = 0
    sizes[:4] = [9000, 3000, 700, 2048]          # 9000 keys: table too large to stage
    off, elems = _synthetic_csr(rng, sizes, 20000)
    # repeated entries in every 5th set
    rows = [elems[off[u]:off[u + 1]] for u in range(sizes.size)]
    rows = [np.concatenate([r, r[: r.size // 4]]) if u % 5 == 0 else r for u, r in enumerate(rows)]
    off = np.concatenate([[0], np.cumsum([r.size for r in rows])]).astype(np.int32)
    elems = np.concatenate(rows).astype(np.int32)
    P = 60000
    pa = rng.integers(0, sizes.size, size=P).astype(np.int32)
    pb = rng.integers(0, sizes.size, size=P).astype(np.int32)
    pa[:4000] = rng.integers(0, 4, size=4000)     # ~1000 probers for each big set
    pb[4000:4100] = pa[4000:4100]
    doff, de, dpa, dpb = (dev(x, cuda) for x in (off, elems, pa, pb))
    t = R.Table(doff, de, hierarchical=hier)
    ot = oracle_mod.Table(off, elems, hier=hier)
    of, oi = oracle_mod.sss(ot, pa, pb, mode=1, num=3, den=10)
    off_f, _ = oracle_mod.sss(ot, pa, pb, mode=0, thr=0.3)
    before = R.get_tuning()
    try:
        for method in (R.PAIR_OWNER, R.PAIR_FLAT, R.PAIR_DEFAULT):
            R.set_tuning(pair_method=method)
            f, i = R.sss(t, doff, de, dpa, dpb, 3, 10)
            assert np.array_equal(host(i), oi) and np.array_equal(host(f), of), method
            f, _ = R.sss(t, doff, de, dpa, dpb, 3, 10, with_inter=False)
            assert np.array_equal(host(f), of), method
            f, _ = R.sss_float(t, doff, de, dpa, dpb, 0.3)
            assert np.array_equal(host(f), off_f), method
        t.check()
    finally:
        R.set_tuning(**before)


# -------------------------------------------------------------------- IR --

def _ir_index(rng, nterms, ndocs, npost, nq, empty_every=0):
    w = 1.0 / np.arange(1, nterms + 1) ** 1.1
    df = np.minimum(np.maximum(1, np.round(w / w.sum() * npost)), ndocs).astype(np.int64)
    df[::11] = 0  # terms with no postings
    lists = [np.sort(rng.choice(ndocs, size=int(k), replace=False)).astype(np.int32) for k in df]
    toff = np.zeros(nterms + 1, np.int32)
    toff[1:] = np.cumsum([l.size for l in lists])
    docs = np.concatenate(lists).astype(np.int32)
    p = (df + 1) / (df + 1).sum()
    q, qoff = [], [0]
    for i in range(nq):
        k = 0 if (empty_every and i % empty_every == 0) else int(rng.integers(1, 7))
        ts = np.unique(rng.choice(nterms, size=k, p=p)) if k else []
        ts = sorted(list(ts), key=lambda t: (int(df[t]), int(t)))
        q.extend(ts)
        qoff.append(len(q))
    return toff, docs, np.array(q, np.int32), np.array(qoff, np.int32)


@pytest.mark.parametrize("hier", [True, False])
def test_ir_matches_oracle(R, cuda, oracle_mod, hier):
    rng = np.random.default_rng(21)
    toff, docs, query, qoff = _ir_index(rng, 400, 60000, 300000, 700, empty_every=50)
    dt, dd, dq, dqo = (dev(x, cuda) for x in (toff, docs, query, qoff))
    t = R.Table(dt, dd, hierarchical=hier, hash_order=True)
    ot = oracle_mod.Table(toff, docs, hier=hier)
    for dsrc, osrc in [(dd, docs), (t.hash_order, ot.hash_order())]:
        roff, res, cnt = R.ir(t, dt, dsrc, dq, dqo)
        oroff, ores, ocnt = oracle_mod.ir(ot, query, qoff, docs=osrc)
        assert np.array_equal(host(roff), oroff)
        assert np.array_equal(host(cnt), ocnt)
        hr = host(res)
        for qi in range(qoff.size - 1):
            a, c = oroff[qi], ocnt[qi]
            assert np.array_equal(hr[a:a + c], ores[a:a + c]), f"query {qi}"
    t.check()


def test_ir_long_first_lists(R, cuda, oracle_mod):
    """First-term lists longer than one work slice (several slices per query)."""
    rng = np.random.default_rng(4)
    ndocs = 200000
    lists = [np.sort(rng.choice(ndocs, size=s, replace=False)).astype(np.int32)
             for s in [50000, 60000, 9000, 120000, 7]]
    toff = np.zeros(len(lists) + 1, np.int32)
    toff[1:] = np.cumsum([l.size for l in lists])
    docs = np.concatenate(lists)
    query = np.array([0, 1, 3, 1, 3, 0, 1, 2, 3, 1], np.int32)
    qoff = np.array([0, 3, 5, 7, 9, 10], np.int32)
    dt, dd, dq, dqo = (dev(x, cuda) for x in (toff, docs, query, qoff))
    t = R.Table(dt, dd)
    ot = oracle_mod.Table(toff, docs)
    roff, res, cnt = R.ir(t, dt, dd, dq, dqo)
    oroff, ores, ocnt = oracle_mod.ir(ot, query, qoff)
    assert np.array_equal(host(cnt), ocnt)
    hr = host(res)
    for qi in range(qoff.size - 1):
        a, c = oroff[qi], ocnt[qi]
        assert np.array_equal(hr[a:a + c], ores[a:a + c])


# -------------------------------------------------------------- raw pair --

@pytest.mark.parametrize("na,nb,universe", [
    (1, 1, 4), (16, 100, 64), (1000, 3000, 6000), (4096, 4096, 1 << 14),
    (1 << 20, 1 << 16, 1 << 22), (1 << 16, 1 << 20, 1 << 21), (0, 10, 10), (10, 0, 10)])
def test_intersect_count(R, cuda, oracle_mod, na, nb, universe):
    rng = np.random.default_rng(na * 7 + nb)
    a = rng.integers(0, universe, size=na).astype(np.int32)
    b = rng.integers(0, universe, size=nb).astype(np.int32)
    got = R.intersect_count(dev(a, cuda), dev(b, cuda))
    assert got == oracle_mod.pair_count(a, b)


# ------------------------------------------------- TC methods, odd shapes --

def _random_rows(rng, sizes, n, dup_every=0):
    rows = []
    for i, s in enumerate(sizes):
        r = rng.choice(n, size=min(s, n), replace=False) if s else np.zeros(0, np.int64)
        if dup_every and i % dup_every == 0 and r.size > 1:
            r = np.concatenate([r, r[: max(1, r.size // 3)]])  # repeated entries
        rows.append(np.sort(r).astype(np.int32))
    off = np.zeros(len(rows) + 1, np.int32)
    off[1:] = np.cumsum([r.size for r in rows])
    return off, np.concatenate(rows).astype(np.int32)


@pytest.mark.parametrize("hier", [True, False])
def test_tc_methods_on_ragged_rows(R, cuda, oracle_mod, hier):
    """Row lengths at every class boundary of the staged kernel (tiny < 32,
    warp-staged <= 256, CTA-staged <= 4096, unstaged above), rows with
    repeated entries and equal-length pairs (the probe direction decides the
    count there), against the oracle's restatement of TC.cu:143-183."""
    rng = np.random.default_rng(17)
    n = 9000
    sizes = list(rng.integers(0, 40, size=n))
    for i, s in zip(range(0, 60, 5), [31, 32, 33, 255, 256, 257, 300, 4095, 4096, 4097, 6000, 8000]):
        sizes[i] = s
    off, cols = _random_rows(rng, sizes, n, dup_every=7)
    ot = oracle_mod.Table(off, cols, hier=hier)
    want = oracle_mod.tc_hash(ot)
    doff, dcols = dev(off, cuda), dev(cols, cuda)
    t = R.Table(doff, dcols, hierarchical=hier, hash_order=True)
    for method in (R.TC_EDGE, R.TC_STAGED, R.TC_OWNER):
        assert R.tc_count(t, doff, dcols, method=method) == want
        assert R.tc_count(t, doff, t.hash_order, method=method) == oracle_mod.tc_hash(ot, ot.hash_order())
    t.check()


@pytest.mark.parametrize("scale", [10, 14, 17])
def test_tc_methods_agree_rmat(R, cuda, oracle_mod, scale):
    off, cols = R.gen_rmat(scale, 16, 0x5EED0100 + scale, oriented=True)
    want = oracle_mod.tc_merge(off.cpu().numpy(), cols.cpu().numpy())
    t = R.Table(off, cols, hash_order=True)
    for method in (R.TC_EDGE, R.TC_STAGED, R.TC_OWNER):
        assert R.tc_count(t, off, t.hash_order, method=method) == want


def _fixture_counts():
    import json
    import os
    p = os.path.join(os.path.dirname(__file__), "golden", "tc_counts.json")
    return json.load(open(p))["counts"]


@pytest.mark.parametrize("scale", [16, 18, 20, 22, 24])
def test_tc_benchmark_graphs_match_oracle_counts(R, cuda, scale):
    """The benchmark's graphs at full size (scale 24: 16.8M vertices, 260M
    oriented edges): the device generator's graph, its tables (the
    reference's alpha 0.2 / 5 slots, and 0.4 / 2) and every TC method give
    the triangle count the CPU oracle computed on the same seeded graph
    (tests/golden/tc_counts.json, made by make_tc_counts.py)."""
    rec = _fixture_counts()[str(scale)]
    off, cols = R.gen_rmat(scale, 16, int(rec["seed"], 16), oriented=True)
    assert off.numel() - 1 == rec["vertices"] and cols.numel() == rec["oriented_edges"]
    methods = (R.TC_OWNER, R.TC_EDGE) if scale >= 22 else (R.TC_OWNER, R.TC_EDGE, R.TC_STAGED)
    for alpha, bucket in [(0.2, 5), (0.4, 2)]:
        t = R.Table(off, cols, alpha=alpha, bucket=bucket, hierarchical=True, hash_order=True)
        for method in methods:
            assert R.tc_count(t, off, t.hash_order, method=method) == rec["triangles"], \
                (alpha, bucket, method)
        t.check()
        t.free()


def test_tc_owner_alignment_rules(R, cuda, oracle_mod):
    """Method 3 streams rows with 16-byte loads: a column array that is not
    16-byte aligned is refused by method 3 and counted by method 1 under the
    default method."""
    torch = cuda
    off, cols = oracle_mod.rmat_graph(10, 16, 0x5EED0010, oriented=True)
    want = oracle_mod.tc_merge(off, cols)
    doff = dev(off, torch)
    buf = torch.zeros(cols.size + 1, dtype=torch.int32, device="cuda")
    buf[1:] = dev(cols, torch)
    shifted = buf[1:]                      # 4-byte offset from a 256-byte aligned base
    assert shifted.data_ptr() % 16 == 4
    t = R.Table(doff, shifted, hierarchical=True)
    assert R.tc_count(t, doff, shifted) == want
    from reset_b200._lib import ResetError
    with pytest.raises(ResetError):
        R.tc_count(t, doff, shifted, method=R.TC_OWNER)


# --------------------------------------------------------- tuning knobs --

@pytest.mark.parametrize("variant,rounds,wpm,alpha,bucket", [
    (0, 2, 64, 0.2, 5), (0, 4, 1, 0.2, 5), (1, 2, 32, 0.2, 5), (1, 4, 64, 0.2, 5),
    (1, 8, 64, 0.2, 5), (1, 8, 1, 0.2, 5), (1, 8, 100000, 0.2, 5),
    (1, 8, 64, 0.4, 2), (1, 8, 1, 0.4, 2), (1, 8, 64, 0.25, 1), (1, 4, 32, 0.9, 1),
    (1, 8, 64, 1.0, 2), (0, 4, 64, 0.4, 2)])
def test_every_probe_variant_counts_the_same(R, cuda, oracle_mod, variant, rounds, wpm,
                                             alpha, bucket):
    """The probe knobs change scheduling only: TC counts, SSS flags and sizes
    equal the oracle for every variant, both hashes."""
    torch = cuda
    before = R.get_tuning()
    try:
        R.set_tuning(probe_rounds=4 if rounds != 8 else None, warp_pair_min=wpm,
                     probe_variant=variant)
        R.set_tuning(probe_rounds=rounds)
        off, cols = R.gen_rmat(13, 16, 0x5EED7000, oriented=True)
        want = oracle_mod.tc_merge(host(off), host(cols))
        for hier in (True, False):
            t = R.Table(off, cols, alpha=alpha, bucket=bucket, hierarchical=hier,
                        hash_order=True)
            assert R.tc_count(t, off, t.hash_order) == want
            assert R.tc_count(t, off, cols) == want
        s_off, s_cols = R.gen_rmat(11, 16, 0x5EED7001, oriented=False)
        st = R.Table(s_off, s_cols, hierarchical=True)
        n = s_off.numel() - 1
        g = torch.Generator(device="cuda").manual_seed(3)
        pa = torch.randint(0, n, (20000,), device="cuda", dtype=torch.int32, generator=g)
        pb = torch.randint(0, n, (20000,), device="cuda", dtype=torch.int32, generator=g)
        f, i = R.sss(st, s_off, s_cols, pa, pb, num=1, den=5)
        of, oi = oracle_mod.sss(oracle_mod.Table(host(s_off), host(s_cols), hier=1),
                                host(pa), host(pb), mode=1, num=1, den=5)
        assert np.array_equal(host(f), of.astype(np.uint8)) and np.array_equal(host(i), oi)
    finally:
        R.set_tuning(probe_rounds=4, probe_variant=before["probe_variant"])
        R.set_tuning(**before)


def test_free_async_across_streams(R, cuda, oracle_mod):
    """Build on one stream, count on another, free stream-ordered on the
    counting stream; repeated back to back without host syncs."""
    torch = cuda
    off, cols = R.gen_rmat(14, 16, 0x5EED7100, oriented=True)
    want = oracle_mod.tc_merge(host(off), host(cols))
    s_build, s_probe = torch.cuda.Stream(), torch.cuda.Stream()
    outs = []
    for _ in range(6):
        with torch.cuda.stream(s_build):
            t = R.Table(off, cols, hierarchical=True, hash_order=True, stream=s_build)
            ev = torch.cuda.Event()
            ev.record(s_build)
        s_probe.wait_event(ev)
        with torch.cuda.stream(s_probe):
            c = R.tc_count_async(t, off, t.hash_order, stream=s_probe)
        t.hash_order.record_stream(s_probe)
        t.free_async(s_probe)
        outs.append(c)
    torch.cuda.synchronize()
    assert [int(c.item()) for c in outs] == [want] * 6


# ------------------------------------------------------------ 4-cliques --

@pytest.mark.parametrize("scale,hier", [(8, True), (11, True), (11, False), (14, True)])
def test_clique4_matches_oracle(R, cuda, oracle_mod, scale, hier):
    off, cols = R.gen_rmat(scale, 16, 0x5EED4C00 + scale, oriented=True)
    want = oracle_mod.clique4(host(off), host(cols))
    t = R.Table(off, cols, hierarchical=hier)
    assert R.clique4_count(t, off, cols) == want
    t.check()


def test_clique4_complete_graph(R, cuda):
    torch = cuda
    from math import comb
    n = 40
    rows = [list(range(u + 1, n)) for u in range(n)]
    off = np.zeros(n + 1, np.int32)
    off[1:] = np.cumsum([len(r) for r in rows])
    cols = np.array(sum(rows, []), np.int32)
    d_off, d_cols = dev(off, torch), dev(cols, torch)
    t = R.Table(d_off, d_cols)
    assert R.clique4_count(t, d_off, d_cols) == comb(n, 4)


@pytest.mark.parametrize("scale,hier", [(10, True), (12, False), (13, True)])
def test_clique_k_matches_oracle(R, cuda, oracle_mod, scale, hier):
    """k-cliques (SMOG's clique search over hash probes) equal the oracle's
    depth-first merge restatement for k = 3..7; k = 3 and 4 also equal the
    triangle and 4-clique counts."""
    torch = cuda
    off, cols = oracle_mod.rmat_graph(scale, 16, 0x5EED0500 + scale, oriented=True)
    d_off, d_cols = dev(off, torch), dev(cols, torch)
    t = R.Table(d_off, d_cols, hierarchical=hier)
    for k in range(3, 8):
        assert R.clique_count(t, d_off, d_cols, k) == oracle_mod.clique_k(off, cols, k), k
    assert R.clique_count(t, d_off, d_cols, 3) == oracle_mod.tc_merge(off, cols)
    assert R.clique_count(t, d_off, d_cols, 4) == R.clique4_count(t, d_off, d_cols)
    t.check()


def test_clique_k_complete_graph_and_limits(R, cuda):
    torch = cuda
    from math import comb
    from reset_b200._lib import ResetError
    n = 24
    rows = [list(range(u + 1, n)) for u in range(n)]
    off = np.zeros(n + 1, np.int32)
    off[1:] = np.cumsum([len(r) for r in rows])
    cols = np.array(sum(rows, []), np.int32)
    d_off, d_cols = dev(off, torch), dev(cols, torch)
    t = R.Table(d_off, d_cols)
    for k in (3, 5, 9, 16):
        assert R.clique_count(t, d_off, d_cols, k) == comb(n, k), k
    for k in (2, 17):
        with pytest.raises(ResetError):
            R.clique_count(t, d_off, d_cols, k)


# ------------------------------------------------------------- patterns --

def _extra_patterns(R):
    """Hand-made patterns beside SMOG's: reuse with restriction and
    distinctness mixed; last levels that list one vertex (the vertex just
    picked, bounded by it, or distinct from all earlier ones)."""
    P = R.PatternSpec
    return {
        "mixed": P(5, (0, 1, 2, 4, 6), (0, 0, 1, -1, 3, 0), (-1, 0, -1, 1, -1),
                   (-1, -1, -1, 2, -1), 3),
        "tail_bound": P(4, (0, 1, 3, 4), (0, 0, 1, 2), (-1, 0, -1, 2), None, 3),
        "tail_distinct": P(4, (0, 1, 3, 4), (0, 0, 1, 2), (-1, 0, -1, -1), None, 3),
        "tail_fixed": P(4, (0, 1, 3, 4), (0, 0, 1, 0), (-1, 0, 1, 1), None, 1),
    }


def _oracle_pattern(oracle_mod, off, cols, p):
    return oracle_mod.pattern_count(off, cols, p.k, p.flags, p.offsets, p.backward,
                                    p.restriction, p.reuse)


@pytest.mark.parametrize("scale,hier", [(9, True), (10, False), (11, True)])
def test_pattern_count_matches_oracle(R, cuda, oracle_mod, scale, hier):
    """SMOG's query patterns (the general and the reusing form, with
    restrictions and distinctness) equal the oracle's count by definition,
    each on the graph the reference counts it on (oriented for the cliques
    Q0, Q3, Q5, Q7; symmetric for the rest).  Q6 stops at scale 10, where
    the oracle still takes seconds."""
    torch = cuda
    graphs = {}
    for name, p in R.PATTERNS.items():
        if name == "Q6" and scale > 10:
            continue
        if p.graph not in graphs:
            off, cols = oracle_mod.rmat_graph(scale, 16, 0x5EED7B00 + scale,
                                              oriented=(p.graph == "oriented"))
            d_off, d_cols = dev(off, torch), dev(cols, torch)
            graphs[p.graph] = (off, cols, d_off, d_cols, R.Table(d_off, d_cols, hierarchical=hier))
        off, cols, d_off, d_cols, t = graphs[p.graph]
        assert R.pattern_count(t, d_off, d_cols, name) == _oracle_pattern(oracle_mod, off, cols, p), name
    off, cols, d_off, d_cols, t = graphs["symmetric"]
    for name, p in _extra_patterns(R).items():
        assert R.pattern_count(t, d_off, d_cols, p) == _oracle_pattern(oracle_mod, off, cols, p), name
    for g in graphs.values():
        g[4].check()


def test_pattern_count_complete_graphs_and_cliques(R, cuda, oracle_mod):
    """Complete graphs (every candidate set full, distinctness and
    restrictions decide alone), a hand-made pattern mixing reuse,
    restriction and distinctness, an 8-vertex reusing clique chain equal to
    the 8-clique count, and Q5 equal to the 5-clique kernel's count."""
    torch = cuda
    from math import comb
    P = R.PatternSpec
    chain8 = P(8, (0, 1, 3, 5, 7, 9, 11, 13), (0, 0, 1, -1, 2, -1, 3, -1, 4, -1, 5, -1, 6),
               None, (-1, -1, -1, 2, 3, 4, 5, 6))
    n = 12
    for oriented in (True, False):
        rows = [[v for v in range(n) if (v > u if oriented else v != u)] for u in range(n)]
        off = np.zeros(n + 1, np.int32)
        off[1:] = np.cumsum([len(r) for r in rows])
        cols = np.array(sum(rows, []), np.int32)
        d_off, d_cols = dev(off, torch), dev(cols, torch)
        t = R.Table(d_off, d_cols)
        for name, p in (list(R.PATTERNS.items()) + list(_extra_patterns(R).items()) +
                        [("chain8", chain8)]):
            want = _oracle_pattern(oracle_mod, off, cols, p)
            assert R.pattern_count(t, d_off, d_cols, p) == want, (name, oriented)
        if oriented:
            assert R.pattern_count(t, d_off, d_cols, chain8) == comb(n, 8)
    off, cols = oracle_mod.rmat_graph(12, 16, 0x5EED7B0C, oriented=True)
    d_off, d_cols = dev(off, torch), dev(cols, torch)
    t = R.Table(d_off, d_cols)
    assert R.pattern_count(t, d_off, d_cols, "Q5") == R.clique_count(t, d_off, d_cols, 5)
    assert R.pattern_count(t, d_off, d_cols, chain8) == R.clique_count(t, d_off, d_cols, 8)
    # the same cliques listed level by level (no reuse) run the general
    # kernel, the reusing chains the k-clique kernel
    for name, k in (("Q3", 4), ("Q5", 5), ("Q7", 6)):
        offs = [0, 1] + [1 + sum(range(2, l + 1)) for l in range(2, k)]
        listed = P(k, tuple(offs), tuple([0] + [j for l in range(2, k) for j in range(l)]))
        assert R.pattern_count(t, d_off, d_cols, listed) == R.pattern_count(t, d_off, d_cols, name), name
    # an empty edge list counts nothing
    e_off = dev(np.zeros(5, np.int32), torch)
    e_cols = torch.empty(0, dtype=torch.int32, device="cuda")
    assert R.pattern_count(R.Table(e_off, e_cols), e_off, e_cols, "Q4") == 0


def test_pattern_count_unsorted_rows(R, cuda, oracle_mod):
    """Rows in shuffled order (no ascending-row shortcuts: every key
    scanned) count what the sorted rows count, for every pattern."""
    torch = cuda
    rng = np.random.default_rng(0x5EED7B0A)
    for g in ("symmetric", "oriented"):
        off, cols = oracle_mod.rmat_graph(10, 16, 0x5EED7B0A, oriented=(g == "oriented"))
        sh = cols.copy()
        for u in range(off.size - 1):
            rng.shuffle(sh[off[u]:off[u + 1]])
        d_off, d_cols = dev(off, torch), dev(sh, torch)
        t = R.Table(d_off, d_cols, hierarchical=(g == "symmetric"))
        for name, p in R.PATTERNS.items():
            if p.graph == g:
                assert R.pattern_count(t, d_off, d_cols, name) == \
                    _oracle_pattern(oracle_mod, off, cols, p), name
        if g == "symmetric":
            for name, p in _extra_patterns(R).items():
                assert R.pattern_count(t, d_off, d_cols, p) == \
                    _oracle_pattern(oracle_mod, off, cols, p), name


def block_diagonal(graphs):
    """Disjoint oriented graphs [(off, cols)] -> one CSR + vertex offsets."""
    offs, colss, gro = [np.zeros(1, np.int64)], [], [0]
    vbase = ebase = 0
    for off, cols in graphs:
        offs.append(off[1:].astype(np.int64) + ebase)
        colss.append(cols.astype(np.int64) + vbase)
        vbase += off.size - 1
        ebase += cols.size
        gro.append(vbase)
    return (np.concatenate(offs).astype(np.int32), np.concatenate(colss).astype(np.int32),
            np.array(gro, np.int32))


@pytest.mark.parametrize("hier", [True, False])
def test_tc_count_batch_per_graph(R, cuda, oracle_mod, hier):
    """One owner-grouped count over a batch of disjoint graphs of different
    sizes (including empty and edgeless ones) gives every graph's own
    triangle count, as the oracle counts them one by one."""
    torch = cuda
    graphs = []
    for i, scale in enumerate([6, 9, 1, 11, 8, 7, 10, 5]):
        if i == 2:
            graphs.append((np.zeros(4, np.int32), np.zeros(0, np.int32)))  # edgeless
            continue
        graphs.append(oracle_mod.rmat_graph(scale, 16, 0x5EED0600 + i, oriented=True))
    off, cols, gro = block_diagonal(graphs)
    want = [oracle_mod.tc_merge(o, c) if c.size else 0 for o, c in graphs]
    d_off, d_cols, d_gro = dev(off, torch), dev(cols, torch), dev(gro, torch)
    t = R.Table(d_off, d_cols, hierarchical=hier, hash_order=True)
    for c in (d_cols, t.hash_order):
        got = host(R.tc_count_batch(t, d_off, c, d_gro)).tolist()
        assert got == want
    assert R.tc_count(t, d_off, t.hash_order) == sum(want)
    t.check()

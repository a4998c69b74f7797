"""The served form (reset_server_*): every request kind against the oracle,
each result identical alone and in a concurrent mix, admission by the
device-memory budget, and argument errors."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def R(cuda, libreset):
    from reset_b200 import api
    return api


@pytest.fixture(scope="module")
def S(cuda, libreset):
    from reset_b200 import server
    return server


def host(t):
    return t.detach().cpu().numpy()


def _ir_index(rng, nterms, ndocs, npost):
    w = 1.0 / np.arange(1, nterms + 1) ** 1.1
    df = np.minimum(np.maximum(1, np.round(w / w.sum() * npost)), ndocs).astype(np.int64)
    df[::13] = 0
    lists = [np.sort(rng.choice(ndocs, size=int(k), replace=False)).astype(np.int32) for k in df]
    toff = np.zeros(nterms + 1, np.int32)
    toff[1:] = np.cumsum([l.size for l in lists])
    return toff, np.concatenate(lists).astype(np.int32), df


def _queries(rng, df, nq):
    p = (df + 1) / (df + 1).sum()
    out = []
    for _ in range(nq):
        k = int(rng.integers(1, 7))
        ts = np.unique(rng.choice(df.size, size=k, p=p))
        out.append(np.array(sorted(ts.tolist(), key=lambda t: (int(df[t]), t)), np.int32))
    return out


def _sets(off, el, v):
    return el[off[v]:off[v + 1]]


@pytest.fixture(scope="module")
def world(R, cuda, oracle_mod):
    """An IR index, a symmetric graph (pairs, triples) and an oriented graph
    (per-vertex triangles), with the expected answers of a request mix."""
    torch = cuda
    rng = np.random.default_rng(7)
    toff, docs, df = _ir_index(rng, 300, 50000, 250000)
    ir_t = R.Table(torch.from_numpy(toff).cuda(), torch.from_numpy(docs).cuda(), hierarchical=True)
    s_off, s_cols = R.gen_rmat(11, 16, 0x5EED5001, oriented=False)
    sym_t = R.Table(s_off, s_cols, hierarchical=True)
    o_off, o_cols = R.gen_rmat(11, 16, 0x5EED5002, oriented=True)
    ori_t = R.Table(o_off, o_cols, hierarchical=False)
    so, sc = host(s_off), host(s_cols)
    oo, oc = host(o_off), host(o_cols)
    n = so.size - 1
    reqs = []
    ot = oracle_mod.Table(toff, docs, hier=1)
    for q in _queries(rng, df, 120):
        _, res, cnt = oracle_mod.ir(ot, q, np.array([0, q.size], np.int32))
        reqs.append(("ir", q, res[:cnt[0]]))
    for _ in range(40):
        k = int(rng.integers(1, 300))
        pa = rng.integers(0, n, k).astype(np.int32)
        pb = rng.integers(0, n, k).astype(np.int32)
        inter = np.array([np.intersect1d(_sets(so, sc, a), _sets(so, sc, b)).size
                          for a, b in zip(pa, pb)], np.int64)
        U = np.diff(so)[pa] + np.diff(so)[pb] - inter
        flags = ((U > 0) & (4 * inter >= 1 * U)).astype(np.uint8)
        reqs.append(("pairs", (pa, pb), (inter, flags)))
    for _ in range(40):
        k = int(rng.integers(1, 50))
        tri = rng.integers(0, n, (k, 3)).astype(np.int32)
        tri[::3, 1] = tri[::3, 0]
        want = np.array([np.intersect1d(np.intersect1d(_sets(so, sc, a), _sets(so, sc, b)),
                                        _sets(so, sc, c)).size for a, b, c in tri], np.int64)
        reqs.append(("triples", tri, want))
    for _ in range(30):
        vs = rng.integers(0, n, int(rng.integers(1, 20))).astype(np.int32)
        want = np.array([sum(np.intersect1d(_sets(oo, oc, v), _sets(oo, oc, w)).size
                             for w in _sets(oo, oc, v)) for v in vs], np.int64)
        reqs.append(("tc", vs, want))
    for _ in range(25):
        na, nb = (int(x) for x in np.exp(rng.uniform(np.log(16), np.log(40000), 2)))
        a = rng.integers(0, 60000, na).astype(np.int32)
        b = rng.integers(0, 60000, nb).astype(np.int32)
        reqs.append(("raw", (a, b), oracle_mod.pair_count(a, b)))
    rng.shuffle(reqs)
    return dict(ir=ir_t, sym=sym_t, ori=ori_t, reqs=reqs)


def _submit(srv, ix, req):
    kind, args, _ = req
    if kind == "ir":
        return srv.submit_ir(ix["ir"], args)
    if kind == "pairs":
        return srv.submit_pairs(ix["sym"], args[0], args[1], num=1, den=4)
    if kind == "triples":
        return srv.submit_triples(ix["sym"], args)
    if kind == "tc":
        return srv.submit_tc_vertices(ix["ori"], args)
    return srv.submit_raw(args[0], args[1])


def _check(req, r):
    kind, args, want = req
    assert r.status == 0, (kind, r.status)
    if kind == "ir":
        got = r.docs if r.docs is not None else np.zeros(0, np.int32)
        assert np.array_equal(got, want) and r.count == want.size
    elif kind == "pairs":
        assert np.array_equal(r.values, want[0]) and np.array_equal(r.flags, want[1])
        assert r.count == int(want[1].sum())
    elif kind in ("triples", "tc"):
        assert np.array_equal(r.values, want) and r.count == int(want.sum())
    else:
        assert r.count == want


def _register(srv, world):
    return {k: srv.add_index(world[k]) for k in ("ir", "sym", "ori")}


def test_mix_matches_oracle_and_alone(S, world):
    reqs = world["reqs"]
    with S.Server(streams=4, max_batch_requests=64) as srv:
        ix = _register(srv, world)
        tickets = [_submit(srv, ix, q) for q in reqs]       # all in flight at once
        mixed = [srv.wait(t) for t in tickets]
        st = srv.stats()
    for q, r in zip(reqs, mixed):
        _check(q, r)
    assert st["completed"] == len(reqs) and st["batches"] >= 2
    assert max(r.batch_size for r in mixed) > 1
    with S.Server(streams=1, max_batch_requests=1) as srv:
        ix = _register(srv, world)
        for q, rm in zip(reqs, mixed):
            ra = srv.wait(_submit(srv, ix, q))               # alone: batch of one
            assert ra.batch_size == 1
            _check(q, ra)
            for f in ("count",):
                assert getattr(ra, f) == getattr(rm, f)
            for f in ("docs", "values", "flags"):
                a, b = getattr(ra, f), getattr(rm, f)
                assert (a is None and b is None) or np.array_equal(a, b)


def test_results_when_the_pinned_arena_is_full(S, world):
    """IR results land in the pinned result arena and are handed out without
    a copy; while clients hold the arena full, later results land in
    pageable buffers instead.  Both give the oracle's lists, including when
    a second thread waits and releases while requests are submitted."""
    import queue
    import threading
    reqs = [q for q in world["reqs"] if q[0] == "ir"]
    assert sum(q[2].size for q in reqs) * 4 > 8192      # the arena cannot hold all
    with S.Server(streams=4, max_batch_requests=8, pinned_result_bytes=8192) as srv:
        ix = _register(srv, world)
        held = [srv.wait(_submit(srv, ix, q), release=False) for q in reqs[:4]]
        tickets = [_submit(srv, ix, q) for q in reqs]
        for q, t in zip(reqs, tickets):
            _check(q, srv.wait(t))
        for q, r in zip(reqs[:4], held):
            _check(q, r)
    with S.Server(streams=4, max_batch_requests=8, pinned_result_bytes=1 << 16) as srv:
        ix = _register(srv, world)
        ready, got = queue.Queue(), []

        def consume():
            while (tk := ready.get()) is not None:
                got.append(srv.wait(tk))
        th = threading.Thread(target=consume)
        th.start()
        for q in reqs * 3:
            ready.put(_submit(srv, ix, q))
        ready.put(None)
        th.join()
    for q, r in zip(reqs * 3, got):
        _check(q, r)


def test_memory_budget_admission(S, world):
    reqs = [q for q in world["reqs"] if q[0] != "raw"]
    budget = 256 * 1024
    with S.Server(streams=3, max_batch_requests=1000, mem_budget_bytes=budget) as srv:
        ix = _register(srv, world)
        tickets = [_submit(srv, ix, q) for q in reqs]
        for q, t in zip(reqs, tickets):
            r = srv.wait(t)
            if r.status == 2:        # a request larger than the whole budget
                continue
            _check(q, r)
        st = srv.stats()
        assert st["max_in_use_bytes"] <= budget
        assert st["in_use_bytes"] == 0
        big = srv.submit_raw(np.arange(100000, dtype=np.int32), np.arange(100000, dtype=np.int32))
        assert srv.wait(big).status == 2   # RESET_ERR_OOM: can never fit


def test_empty_and_invalid_requests(S, world):
    from reset_b200._lib import ResetError
    with S.Server(streams=2) as srv:
        ix = _register(srv, world)
        r = srv.wait(srv.submit_ir(ix["ir"], []))
        assert r.status == 0 and r.count == 0
        r = srv.wait(srv.submit_raw([], [1, 2]))
        assert r.status == 0 and r.count == 0
        with pytest.raises(ResetError):
            srv.submit_ir(ix["ir"], [10 ** 6])
        with pytest.raises(ResetError):
            srv.submit_pairs(99, [0], [1])
        with pytest.raises(ResetError):
            srv.submit_triples(ix["sym"], [[0, 1, -1]])
        with pytest.raises(ResetError):
            srv.submit_raw([-1], [1])
        with pytest.raises(ResetError):
            srv.wait(123456789)

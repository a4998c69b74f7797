"""The set-similarity self-join pipeline on the GPU, checked against the
oracle: seeded token sets, prefix-filter candidates (exactly the oracle's
restated filter, and a superset of the brute-force join), and the batched
CUDA-graph form of the pair kernel (equal to reset_sss and to the oracle's
decisions, across replays of different sizes)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def R(cuda, libreset):
    from reset_b200 import api
    return api


def host(t):
    return t.detach().cpu().numpy()


def _pairs(a, b):
    return set(zip(host(a).tolist(), host(b).tolist())) if not isinstance(a, np.ndarray) \
        else set(zip(a.tolist(), b.tolist()))


@pytest.mark.parametrize("n,ulog,lo,hi", [(1, 4, 1, 1), (300, 8, 1, 40),
                                          (5000, 16, 8, 300), (20000, 20, 8, 64)])
def test_token_sets_properties(R, n, ulog, lo, hi):
    off, tok = R.gen_token_sets(n, ulog, 1.6, lo, hi, seed=0x5EED0000 + n)
    o, t = host(off), host(tok)
    assert o[0] == 0 and o[-1] == t.size and o.size == n + 1
    sz = np.diff(o)
    assert sz.min() >= 1 and sz.max() <= hi
    assert t.min() >= 0 and t.max() < (1 << ulog)
    row = np.repeat(np.arange(n), sz)
    key = row.astype(np.int64) << 32 | t
    assert np.all(np.diff(key) > 0)             # rows sorted, no duplicates
    off2, tok2 = R.gen_token_sets(n, ulog, 1.6, lo, hi, seed=0x5EED0000 + n)
    assert np.array_equal(host(off2), o) and np.array_equal(host(tok2), t)


def test_planted_near_duplicates(R):
    off, tok = R.gen_token_sets(3000, 24, 1.2, 8, 200, seed=0x5EED0D0D, dup_frac=0.4, keep_min=0.9)
    o, t = host(off), host(tok)
    rows = [set(t[o[i]:o[i + 1]].tolist()) for i in range(o.size - 1)]
    close = sum(1 for i in range(1, len(rows)) if any(
        len(rows[i] & rows[k]) >= 0.7 * len(rows[i] | rows[k]) for k in range(max(0, i - 8), i)))
    assert close > 0.2 * len(rows)       # a large share of sets has a near twin
    off0, tok0 = R.gen_token_sets(3000, 24, 1.2, 8, 200, seed=0x5EED0D0D)
    assert not np.array_equal(host(tok0), t)


def test_token_sets_rejects_bad_arguments(R):
    from reset_b200._lib import ResetError
    for args in [(0, 10, 1.5, 1, 4), (1 << 21, 10, 1.5, 1, 4), (10, 3, 1.5, 1, 4),
                 (10, 10, 1.5, 5, 4), (10, 10, 1.5, 1, 20000)]:
        with pytest.raises(ResetError):
            R.gen_token_sets(*args)


@pytest.mark.parametrize("n,ulog,lo,hi,num,den,dup", [
    (400, 7, 2, 30, 1, 2, 0.0), (1500, 9, 4, 40, 7, 10, 0.0), (1200, 8, 1, 12, 3, 4, 0.0),
    (900, 10, 10, 60, 9, 10, 0.0), (60, 4, 1, 16, 1, 1, 0.0), (1500, 20, 8, 80, 7, 10, 0.3)])
def test_prefix_candidates_match_oracle(R, oracle_mod, n, ulog, lo, hi, num, den, dup):
    off, tok = R.gen_token_sets(n, ulog, 1.3, lo, hi, seed=0x5EED1000 + n, dup_frac=dup)
    pa, pb = R.prefix_candidates(off, tok, ulog, num, den)
    a, b = host(pa), host(pb)
    assert np.all(a < b)
    k = a.astype(np.int64) << 32 | b
    assert np.all(np.diff(k) > 0)               # distinct, sorted by (a, b)
    oa, ob = oracle_mod.prefix_candidates(host(off), host(tok), num, den)
    assert np.array_equal(a, oa) and np.array_equal(b, ob)
    ja, jb = oracle_mod.jaccard_join(host(off), host(tok), num, den)
    assert _pairs(ja, jb) <= _pairs(a, b)        # no qualifying pair is lost


@pytest.mark.parametrize("hier,ulog,dup", [(True, 9, 0.0), (False, 9, 0.0), (True, 22, 0.3)])
def test_self_join_pipeline_equals_brute_force(R, oracle_mod, cuda, hier, ulog, dup):
    torch = cuda
    n, num, den = 1500, 7, 10
    off, tok = R.gen_token_sets(n, ulog, 1.3, 4, 40, seed=0x5EED2000, dup_frac=dup)
    t = R.Table(off, tok, hierarchical=hier)
    pa, pb = R.prefix_candidates(off, tok, ulog, num, den)
    batch = R.Batch(t, tok, capacity=max(1, pa.numel()), num=num, den=den)
    flags, inter = batch(pa, pb)
    torch.cuda.synchronize()
    keep = host(flags).astype(bool)
    got = _pairs(host(pa)[keep], host(pb)[keep])
    ja, jb = oracle_mod.jaccard_join(host(off), host(tok), num, den)
    assert got == _pairs(ja, jb)
    assert len(got) > 0
    batch.close()


@pytest.mark.parametrize("owner_grouped", [False, True])
def test_batch_equals_sss_across_replays(R, oracle_mod, cuda, owner_grouped):
    """Replays of different pair counts (including 0 and 1) equal the plain
    call and the oracle, for the persistent pair kernel and for the
    owner-grouped replay (pairs grouped by the larger set, its table staged
    in shared memory)."""
    torch = cuda
    off, cols = R.gen_rmat(12, 16, 0x5EED3000, oriented=False)
    t = R.Table(off, cols, hierarchical=True)
    n = off.numel() - 1
    g = torch.Generator(device="cuda").manual_seed(5)
    cap = 200_000
    batch = R.Batch(t, cols, capacity=cap, num=1, den=4, owner_grouped=owner_grouped)
    ot = oracle_mod.Table(host(off), host(cols), hier=1)
    for P in [cap, 1, 0, 77_777, 31, 32, 33, 150_000]:
        pa = torch.randint(0, n, (P,), device="cuda", dtype=torch.int32, generator=g)
        pb = torch.randint(0, n, (P,), device="cuda", dtype=torch.int32, generator=g)
        f, i = batch(pa, pb)
        f2, i2 = R.sss(t, off, cols, pa, pb, num=1, den=4)
        assert torch.equal(f, f2) and torch.equal(i, i2)
        if 0 < P <= 100_000:
            of, oi = oracle_mod.sss(ot, host(pa), host(pb), mode=1, num=1, den=4)
            assert np.array_equal(host(f), of.astype(np.uint8))
            assert np.array_equal(host(i), oi)
    t.check()
    batch.close()


@pytest.mark.parametrize("num,den", [(7, 10), (1, 4), (0, 1), (1, 1), (9, 10)])
def test_decisions_only_equal_full_decisions(R, oracle_mod, cuda, num, den):
    """Early exit (no intersection sizes wanted) decides exactly as the full
    probe: plain call without d_inter, and a decisions-only batch."""
    torch = cuda
    off, tok = R.gen_token_sets(30000, 16, 1.2, 8, 600, seed=0x5EED4000, dup_frac=0.4,
                                keep_min=0.6)
    t = R.Table(off, tok, hierarchical=True)
    pa, pb = R.prefix_candidates(off, tok, 16, 7, 10)
    g = torch.Generator(device="cuda").manual_seed(9)
    n = off.numel() - 1
    ra = torch.randint(0, n, (50000,), device="cuda", dtype=torch.int32, generator=g)
    rb = torch.randint(0, n, (50000,), device="cuda", dtype=torch.int32, generator=g)
    pa, pb = torch.cat([pa, ra, pa]), torch.cat([pb, rb, pa])   # similar, random, self pairs
    full, _ = R.sss(t, off, tok, pa, pb, num, den)
    dec, none = R.sss(t, off, tok, pa, pb, num, den, with_inter=False)
    assert none is None and torch.equal(full, dec)
    assert int(full.sum()) > 0
    b = R.Batch(t, tok, capacity=pa.numel(), num=num, den=den, decisions_only=True)
    f, _ = b(pa, pb)
    assert torch.equal(f, full)
    b.close()
    if num == 7:
        sub = slice(0, 40000)
        of, _ = oracle_mod.sss(oracle_mod.Table(host(off), host(tok), hier=1),
                               host(pa[sub]), host(pb[sub]), mode=1, num=num, den=den)
        assert np.array_equal(host(dec[sub]), of.astype(np.uint8))


def test_batch_replays_queue_without_host_sync(R, cuda):
    """Back-to-back runs of different sizes on one stream, read at the end:
    each replay sees its own pair count."""
    torch = cuda
    off, cols = R.gen_rmat(10, 16, 0x5EED3001, oriented=False)
    t = R.Table(off, cols)
    n = off.numel() - 1
    pa = torch.randint(0, n, (5000,), device="cuda", dtype=torch.int32)
    pb = torch.randint(0, n, (5000,), device="cuda", dtype=torch.int32)
    want, _ = R.sss(t, off, cols, pa, pb, num=1, den=3)
    batch = R.Batch(t, cols, capacity=5000, num=1, den=3)
    batch.pair_a.copy_(pa)
    batch.pair_b.copy_(pb)
    outs = []
    for P in [10, 5000, 2500, 4999]:
        batch.flags.fill_(2)
        batch.run(P)
        outs.append(batch.flags.clone())
    torch.cuda.synchronize()
    for P, f in zip([10, 5000, 2500, 4999], outs):
        assert torch.equal(f[:P], want[:P])
        assert bool((f[P:] == 2).all())
    batch.close()


def test_batch_rejects_bad_sizes(R, libreset, cuda):
    off, cols = R.gen_rmat(8, 8, 1, oriented=False)
    t = R.Table(off, cols)
    h = C.c_void_p()
    assert libreset.reset_batch_create(t.handle, C.c_void_p(cols.data_ptr()), 0, 7, 10,
                                       C.byref(h), None) == 3
    assert libreset.reset_batch_create(t.handle, C.c_void_p(cols.data_ptr()), 1 << 31, 7, 10,
                                       C.byref(h), None) == 3
    batch = R.Batch(t, cols, capacity=100)
    assert libreset.reset_batch_run(batch._h, 101, None) == 3
    assert libreset.reset_batch_run(batch._h, -1, None) == 3
    batch.close()

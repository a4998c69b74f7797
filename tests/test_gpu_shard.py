"""Element-modulo sharding on the GPU (reset_csr_shard, reset_tc_count_shard,
reset_sss_decide; multi-GPU/*/main.cu run as G passes on one device):
shards equal a numpy filter, partial triangle counts sum to the oracle's
count, summed partial intersections equal the unsharded sizes and decide
exactly like reset_sss."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def S(cuda, libreset):
    from reset_b200 import shard
    return shard


def test_shard_csr_matches_filter(S, cuda, oracle_mod):
    torch = cuda
    off, cols = oracle_mod.rmat_graph(11, 16, 0x5EED0211, oriented=False)
    d_off, d_cols = torch.from_numpy(off).cuda(), torch.from_numpy(cols).cuda()
    src = np.repeat(np.arange(off.size - 1), np.diff(off))
    for G in (1, 2, 3, 7):
        tot = 0
        for g in range(G):
            o, c = S.shard_csr(d_off, d_cols, G, g)
            o, c = o.cpu().numpy(), c.cpu().numpy()
            keep = cols % G == g
            want_off = np.concatenate([[0], np.cumsum(np.bincount(src[keep],
                                                                  minlength=off.size - 1))])
            assert np.array_equal(o, want_off) and np.array_equal(c, cols[keep])
            tot += c.size
        assert tot == cols.size


@pytest.mark.parametrize("scale", [10, 13])
@pytest.mark.parametrize("hier", [True, False])
def test_sharded_tc_sums_to_full_count(S, cuda, oracle_mod, scale, hier):
    torch = cuda
    off, cols = oracle_mod.rmat_graph(scale, 16, 0x5EED0300 + scale, oriented=True)
    want = oracle_mod.tc_merge(off, cols)
    d_off, d_cols = torch.from_numpy(off).cuda(), torch.from_numpy(cols).cuda()
    for G in (1, 2, 4, 5):
        assert S.tc_count_sharded(d_off, d_cols, G, hierarchical=hier) == want, G
    assert S.tc_count_sharded(d_off, d_cols, 3, alpha=0.5, bucket=1, hierarchical=hier) == want


def test_sharded_sss_equals_unsharded(S, cuda, oracle_mod):
    torch = cuda
    from reset_b200 import api
    off, cols = oracle_mod.rmat_graph(11, 16, 0x5EED0411, oriented=False)
    n = off.size - 1
    d_off, d_cols = torch.from_numpy(off).cuda(), torch.from_numpy(cols).cuda()
    pa = torch.from_numpy(np.repeat(np.arange(n, dtype=np.int32), np.diff(off))).cuda()
    t = api.Table(d_off, d_cols)
    for num, den in [(7, 10), (1, 4)]:
        f_full, i_full = api.sss(t, d_off, d_cols, pa, d_cols, num=num, den=den)
        for G in (2, 3):
            f, i = S.sss_sharded(d_off, d_cols, pa, d_cols, G, num=num, den=den)
            assert torch.equal(i, i_full) and torch.equal(f, f_full)
    of, _ = oracle_mod.sss(oracle_mod.Table(off, cols, hier=1), pa.cpu().numpy(), cols,
                           mode=1, num=1, den=4)
    assert np.array_equal(f.cpu().numpy(), of.astype(np.uint8))


def test_sss_decide_rejects_bad_ids(S, cuda):
    torch = cuda
    off = torch.tensor([0, 2, 4], dtype=torch.int32, device="cuda")
    el = torch.tensor([1, 2, 2, 3], dtype=torch.int32, device="cuda")
    pa = torch.tensor([0, 5], dtype=torch.int32, device="cuda")
    pb = torch.tensor([1, 0], dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError):
        S.sss_sharded(off, el, pa, pb, 1,
                      partial=lambda *a: torch.zeros(2, dtype=torch.int32, device="cuda"))

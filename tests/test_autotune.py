"""Autotuner: its cost model, the measured choice, and the JSON cache (CPU;
the measurement callback is a stand-in here, a GPU timing in bench.py)."""
import numpy as np

from reset_b200 import autotune as A


def test_calc_len_matches_oracle(oracle_mod):
    for a, b in [(0.2, 5), (0.5, 3), (1.0, 1), (0.15, 9)]:
        d = np.array([0, 1, 2, 7, 8, 9, 15, 16, 100, 1000, 1024, 12345, 1 << 20])
        assert list(A.calc_len(d, a, b)) == [oracle_mod.calc_len(int(x), a, b) for x in d]
        assert A.calc_len(77, a, b) == oracle_mod.calc_len(77, a, b)


def test_model_prefers_lower_load():
    degs = np.arange(1, 3000)
    r = [A.slot_reads(a, 5, degs) for a in (0.1, 0.2, 0.5, 1.0)]
    assert all(x < y for x, y in zip(r, r[1:]))
    assert 1.0 <= r[0] < 2.0
    assert A.table_bytes(0.1, 5, degs) > A.table_bytes(0.5, 5, degs)


def test_solve_picks_the_fastest_measurement_and_caches(tmp_path):
    degs = np.random.default_rng(1).integers(1, 500, 2000)
    seen = []

    def fake_ms(hp):
        seen.append((hp.alpha, hp.b, hp.probe_rounds, hp.warp_pair_min))
        return abs(hp.alpha - 0.2) + abs(hp.b - 5) + (0 if hp.warp_pair_min == 128 else 0.5)

    cache = str(tmp_path / "tune.json")
    hp = A.solve("sss", degs, measure=fake_ms, measure_top=3, cache=cache)
    assert (hp.alpha, hp.b, hp.warp_pair_min) == (0.2, 5, 128)
    assert (0.2, 5) in {(a, b) for a, b, _, _ in seen}   # the reference default is measured
    n = len(seen)
    hp2 = A.solve("sss", degs, measure=fake_ms, cache=cache)
    assert len(seen) == n and hp2 == hp      # served from the cache
    hp3 = A.solve("ir", degs, measure=None, cache=cache)
    assert (hp3.alpha, hp3.b) == (A.model_rank(degs)[0].alpha, A.model_rank(degs)[0].b)

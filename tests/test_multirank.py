"""The N>1 host logic of bench.py on CPU: world_size-2 gloo ranks reduce
their timings to the max over ranks and report weak-scaling throughput; the
reference arm under torch.distributed.run prints one line (rank 0) and the
other rank exits 0 without work."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    got = bench.max_over_ranks([10.0 + rank, 5.0 - rank, 7.0], world, device="cpu")
    v = bench.weak_value(1000, world, got[0])
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got, v))


def test_max_over_ranks_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, v in out:
        assert got == [11.0, 5.0, 7.0]           # max over ranks, same on every rank
        assert abs(v - 2 * 1000 / 0.011) < 1e-6  # both replicas' units / slowest time


def test_reference_arm_under_torchrun_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           "bench.py", "--impl", "reference", "--gpus", "2", "--scale", "10",
           "--steps", "1", "--warmup", "0", "--cpu-seconds", "0.5"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1                        # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["cpu_baseline"]["kind"] == "port" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def _shard_rank(rank, world, port, q):
    """Element-modulo sharding over two gloo ranks with CPU stand-ins for the
    per-shard GPU work: every rank takes shards rank, rank + 2, ...; the
    partial triangle counts and per-pair partial intersections are summed by
    the all-reduce and equal the unsharded values."""
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from reset_b200 import shard
    rng = np.random.default_rng(4)
    n = 60
    rows = [np.unique(rng.integers(0, n, size=rng.integers(0, 12))) for _ in range(n)]
    rows = [r[r > u] for u, r in enumerate(rows)]          # oriented, no repeats
    off = torch.tensor(np.concatenate([[0], np.cumsum([len(r) for r in rows])]), dtype=torch.int32)
    cols = torch.tensor(np.concatenate(rows), dtype=torch.int32)
    seen = []

    def tc_part(o, c, G, g):
        seen.append(g)
        return sum(int(np.sum((rows[u][:, None] == rows[v][None, :]) &
                              (rows[u][:, None] % G == g)))
                   for u in range(n) for v in rows[u])

    tri = shard.tc_count_sharded(off, cols, 5, group=dist.group.WORLD, partial=tc_part)
    pa = torch.tensor(rng.integers(0, n, 40), dtype=torch.int32)
    pb = torch.tensor(rng.integers(0, n, 40), dtype=torch.int32)

    def sss_part(o, e, a, b, G, g):
        return torch.tensor([int(np.sum(np.isin(rows[x][rows[x] % G == g], rows[y])))
                             for x, y in zip(a.tolist(), b.tolist())], dtype=torch.int32)

    def decide(o, a, b, inter, num, den):
        return inter
    _, inter = shard.sss_sharded(off, cols, pa, pb, 3, group=dist.group.WORLD,
                                 partial=sss_part, decide=decide)
    dist.barrier()
    dist.destroy_process_group()
    want_tri = sum(len(np.intersect1d(rows[u], rows[v])) for u in range(n) for v in rows[u])
    want_inter = [len(np.intersect1d(rows[x], rows[y])) for x, y in zip(pa.tolist(), pb.tolist())]
    q.put((rank, tri == want_tri, inter.tolist() == want_inter, sorted(seen)))


def test_element_sharding_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=180) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1:] == (True, True, [0, 2, 4])   # rank 0: shards 0, 2, 4 of 5
    assert out[1][1:] == (True, True, [1, 3])      # rank 1: shards 1, 3

"""Element-modulo sharding of the intersection path (the reference's
multi-GPU/ programs).

Shard g of G keeps, in every row, the elements x with x % G == g.  An
intersection splits exactly over the shards (|A ∩ B| = sum_g |A_g ∩ B_g| for
rows without repeated entries), so each device builds the tables of its
shards and probes the full pair or edge list:

* triangle counting (multi-GPU/tc-multi-GPU/main.cu:113-137): partial counts
  of all shards summed -- one u64 all-reduce across devices;
* set similarity (multi-GPU/sss-multi-GPU/main.cu:120-160): per-pair partial
  intersection sizes summed (an int32[P] all-reduce), then decided with the
  full set sizes (reset_sss_decide).

Without a process group every shard runs on this device, one after another,
as the reference's programs do; with one (torch.distributed, NCCL between
GPUs), rank r takes the shards r, r + W, r + 2W, ...  Each rank calls these
functions with the same arguments in the same order.  The per-shard work
functions can be replaced (the `partial` arguments), which is how the
multi-rank logic is tested on CPU.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional, Tuple

import torch

from ._lib import check, load
from . import api


def _ptr(t):
    return C.c_void_p(0 if t is None else t.data_ptr())


def shard_csr(off: torch.Tensor, cols: torch.Tensor, shards: int, shard: int,
              stream=None) -> Tuple[torch.Tensor, torch.Tensor]:
    """Rows of shard `shard` of `shards` (elements x with x % shards == shard)."""
    n = off.numel() - 1
    off_g = torch.empty_like(off)
    cols_g = torch.empty_like(cols)
    m_g = torch.zeros(1, dtype=torch.int64, device=off.device)
    check(load().reset_csr_shard(_ptr(off), _ptr(cols), n, cols.numel(), shards, shard,
                                 _ptr(off_g), _ptr(cols_g), _ptr(m_g), api._stream(stream)))
    mg = int(m_g.item())
    return off_g, (cols_g[:mg].clone() if mg < cols.numel() else cols_g)


def _my_shards(shards: int, group) -> range:
    if group is None:
        return range(shards)
    import torch.distributed as dist
    return range(dist.get_rank(group), shards, dist.get_world_size(group))


def _all_reduce(x: torch.Tensor, group):
    if group is not None:
        import torch.distributed as dist
        dist.all_reduce(x, op=dist.ReduceOp.SUM, group=group)
    return x


def _reduce_device(group, fallback: torch.device) -> torch.device:
    if group is None:
        return fallback
    import torch.distributed as dist
    return torch.device("cpu") if dist.get_backend(group) == "gloo" else fallback


# ------------------------------------------------------------- counting --

def tc_partial(off: torch.Tensor, cols: torch.Tensor, shards: int, shard: int,
               alpha: float = 0.2, bucket: int = 5, hierarchical: bool = True) -> int:
    """Partial triangle count of one shard on this device (reset_tc_count_shard)."""
    off_g, cols_g = shard_csr(off, cols, shards, shard)
    t = api.Table(off_g, cols_g, alpha=alpha, bucket=bucket, hierarchical=hierarchical)
    out = torch.empty(1, dtype=torch.int64, device=off.device)
    check(load().reset_tc_count_shard(t.handle, _ptr(off_g), _ptr(cols_g), cols_g.numel(),
                                      _ptr(off), _ptr(cols), cols.numel(), _ptr(out),
                                      api._stream(None)))
    c = int(out.item())
    t.check()
    t.free()
    return c


def tc_count_sharded(off: torch.Tensor, cols: torch.Tensor, shards: int,
                     alpha: float = 0.2, bucket: int = 5, hierarchical: bool = True,
                     group=None,
                     partial: Optional[Callable[[torch.Tensor, torch.Tensor, int, int], int]] = None
                     ) -> int:
    """Triangle count of an oriented graph over `shards` element shards."""
    if shards < 1:
        raise ValueError("shards must be >= 1")
    fn = partial or (lambda o, c, G, g: tc_partial(o, c, G, g, alpha, bucket, hierarchical))
    local = sum(fn(off, cols, shards, g) for g in _my_shards(shards, group))
    total = torch.tensor([local], dtype=torch.int64, device=_reduce_device(group, off.device))
    return int(_all_reduce(total, group).item())


def sss_partial(off: torch.Tensor, elems: torch.Tensor, pa: torch.Tensor, pb: torch.Tensor,
                shards: int, shard: int, alpha: float = 0.2, bucket: int = 5,
                hierarchical: bool = True) -> torch.Tensor:
    """|A_g ∩ B_g| of every pair for shard g on this device (int32[P])."""
    off_g, el_g = shard_csr(off, elems, shards, shard)
    t = api.Table(off_g, el_g, alpha=alpha, bucket=bucket, hierarchical=hierarchical)
    _, inter = api.sss(t, off_g, el_g, pa, pb, num=0, den=1)
    t.check()
    t.free()
    return inter


def sss_sharded(off: torch.Tensor, elems: torch.Tensor, pa: torch.Tensor, pb: torch.Tensor,
                shards: int, num: int = 7, den: int = 10, alpha: float = 0.2,
                bucket: int = 5, hierarchical: bool = True, group=None,
                partial: Optional[Callable[..., torch.Tensor]] = None,
                decide: Optional[Callable[..., torch.Tensor]] = None
                ) -> Tuple[torch.Tensor, torch.Tensor]:
    """Set-similarity decisions for the pairs (pa[p], pb[p]) over `shards`
    element shards -> (flags uint8[P], intersection sizes int32[P])."""
    if shards < 1:
        raise ValueError("shards must be >= 1")
    fn = partial or (lambda o, e, a, b, G, g: sss_partial(o, e, a, b, G, g, alpha, bucket,
                                                          hierarchical))
    inter = torch.zeros(pa.numel(), dtype=torch.int32, device=pa.device)
    for g in _my_shards(shards, group):
        inter += fn(off, elems, pa, pb, shards, g)
    _all_reduce(inter, group)
    if decide is not None:
        return decide(off, pa, pb, inter, num, den), inter
    flags = torch.empty(pa.numel(), dtype=torch.uint8, device=pa.device)
    status = torch.zeros(1, dtype=torch.int32, device=pa.device)
    check(load().reset_sss_decide(_ptr(off), off.numel() - 1, _ptr(pa), _ptr(pb), pa.numel(),
                                  _ptr(inter), num, den, _ptr(flags), _ptr(status),
                                  api._stream(None)))
    if int(status.item()):
        raise ValueError("a pair id was outside [0, n)")
    return flags, inter

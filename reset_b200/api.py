"""Python host API over the C ABI (include/reset.h).

Device buffers are torch CUDA tensors (plumbing only); every computation
runs in libreset.so.  Functions take and return int32/int64 tensors on the
current CUDA device and run on the current torch stream unless `stream` is
given.
"""
from __future__ import annotations

import ctypes as C
from typing import NamedTuple, Optional, Tuple

import torch

from ._lib import Params, Pattern, TableView, Tuning, check, load


def _lib():
    return load()


def _ptr(t: Optional[torch.Tensor]):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _need(t: torch.Tensor, dtype, name: str):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t


class _CudaArray:
    """Zero-copy view of a device pointer (__cuda_array_interface__ v3)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {
            "shape": (int(n),), "typestr": typestr, "data": (int(ptr or 0), False),
            "version": 3, "strides": None}


def _view(ptr, n, dtype) -> torch.Tensor:
    typestr = {torch.int32: "<i4", torch.int64: "<i8"}[dtype]
    if n == 0:
        return torch.empty(0, dtype=dtype, device="cuda")
    return torch.as_tensor(_CudaArray(ptr, n, typestr), device="cuda")


def params(alpha: float = 0.2, bucket: int = 5) -> Params:
    p = Params()
    _lib().reset_params_default(C.byref(p))
    p.alpha = alpha
    p.bucket = bucket
    return p


class Table:
    """A device-resident table over the sets (rows) of a CSR.

    Mirrors one half of HashTableBuilder (baseline/common/hash_table.cuh:12-95):
    build with (load factor, bucket size, hash function), read back len /
    offsets / slots, free.  With hash_order=True the rows read back in bucket
    order are produced in the same pass (``self.hash_order``).
    """

    def __init__(self, off: torch.Tensor, elems: torch.Tensor, alpha: float = 0.2,
                 bucket: int = 5, hierarchical: bool = True, hash_order: bool = False,
                 stream=None):
        self.off = _need(off, torch.int32, "off")
        self.elems = _need(elems, torch.int32, "elems")
        self.n = off.numel() - 1
        self.m = elems.numel()
        self.hash_order = torch.empty_like(elems) if hash_order else None
        h = C.c_void_p()
        p = params(alpha, bucket)
        check(_lib().reset_table_build(_ptr(off), _ptr(elems), self.n, self.m,
                                       C.byref(p), int(bool(hierarchical)),
                                       _ptr(self.hash_order), C.byref(h),
                                       _stream(stream)))
        self._h = h
        v = TableView()
        check(_lib().reset_table_info(h, C.byref(v)))
        self.bucket = v.bucket
        self.max_len = v.max_len
        self.hierarchical = bool(v.hierarchical)
        self.bucket_num = v.bucket_num
        self.alpha = v.alpha
        self._v = v

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("table already freed")
        return self._h

    def tensors(self) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """Zero-copy (slots, len, off) views; valid while the table lives."""
        v = self._v
        return (_view(v.d_table, self.bucket * self.bucket_num, torch.int32),
                _view(v.d_len, self.n, torch.int32),
                _view(v.d_off, self.n + 1, torch.int64))

    def check(self, stream=None):
        check(_lib().reset_table_check(self.handle, _stream(stream)))

    def csr_hash_order(self, off: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        off = self.off if off is None else _need(off, torch.int32, "off")
        out = torch.empty(self.m, dtype=torch.int32, device=self.off.device)
        check(_lib().reset_csr_hash_order(self.handle, _ptr(off), _ptr(out), _stream(stream)))
        return out

    def free(self):
        if self._h is not None:
            check(_lib().reset_table_free(self._h))
            self._h = None

    def free_async(self, stream=None):
        """Stream-ordered free (reset_table_free_async): every use of the
        table must be ordered before this point of `stream`."""
        if self._h is not None:
            check(_lib().reset_table_free_async(self._h, _stream(stream)))
            self._h = None

    def __del__(self):
        try:
            if getattr(self, "_h", None) is not None:
                _lib().reset_table_free(self._h)
                self._h = None
        except Exception:
            pass


# reset_tc_count_ex methods: 0 default (owner-grouped when the columns are
# 16-byte aligned, else edge-flattened), 1 edge-flattened, 2 vertex-staged,
# 3 owner-grouped (probed tables staged in shared memory)
TC_DEFAULT, TC_EDGE, TC_STAGED, TC_OWNER = 0, 1, 2, 3


def tc_count_async(t: Table, off: torch.Tensor, cols: torch.Tensor,
                   out: Optional[torch.Tensor] = None, method: int = TC_DEFAULT,
                   stream=None) -> torch.Tensor:
    """Triangle count into a device u64 (as int64 tensor), asynchronously."""
    if out is None:
        out = torch.empty(1, dtype=torch.int64, device=cols.device)
    check(_lib().reset_tc_count_ex(t.handle, _ptr(off), _ptr(cols), cols.numel(),
                                   method, _ptr(out), _stream(stream)))
    return out


def tc_count(t: Table, off: torch.Tensor, cols: torch.Tensor, method: int = TC_DEFAULT,
             stream=None) -> int:
    out = tc_count_async(t, off, cols, method=method, stream=stream)
    return int(out.item()) & ((1 << 64) - 1)


def clique4_count(t: Table, off: torch.Tensor, cols: torch.Tensor, stream=None) -> int:
    """4-cliques of the oriented graph the table was built on."""
    out = torch.zeros(1, dtype=torch.int64, device=cols.device)
    check(_lib().reset_clique4_count(t.handle, _ptr(off), _ptr(cols), cols.numel(), _ptr(out),
                                     _stream(stream)))
    return int(out.item()) & ((1 << 64) - 1)


def tc_count_batch(t: Table, off: torch.Tensor, cols: torch.Tensor, graph_off: torch.Tensor,
                   out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
    """Per-graph triangle counts of disjoint graphs in one block-diagonal
    CSR (graph g owns vertices graph_off[g] .. graph_off[g+1]-1) -> int64
    tensor of len(graph_off) - 1 counts, asynchronously."""
    g = graph_off.numel() - 1
    _need(graph_off, torch.int32, "graph_off")
    if out is None:
        out = torch.empty(g, dtype=torch.int64, device=cols.device)
    check(_lib().reset_tc_count_batch(t.handle, _ptr(off), _ptr(cols), cols.numel(),
                                      _ptr(graph_off), g, _ptr(out), _stream(stream)))
    return out


def clique_count(t: Table, off: torch.Tensor, cols: torch.Tensor, k: int, stream=None) -> int:
    """k-cliques (3 <= k <= 16) of the oriented graph the table was built on."""
    out = torch.zeros(1, dtype=torch.int64, device=cols.device)
    check(_lib().reset_clique_count(t.handle, _ptr(off), _ptr(cols), cols.numel(), k,
                                    _ptr(out), _stream(stream)))
    return int(out.item()) & ((1 << 64) - 1)


PATTERN_RESTRICT = 1  # withRestriction: m_l < m_restriction[l]
PATTERN_DISTINCT = 2  # withDuplicate: levels without a restriction take new vertices


class PatternSpec(NamedTuple):
    """A query pattern in SMOG's encoding (reset_pattern in reset.h):
    backward[offsets[l-1]:offsets[l]] are the earlier vertices adjacent to
    vertex l, -1 standing for those a reused level's set covers."""
    k: int
    offsets: Tuple[int, ...]
    backward: Tuple[int, ...]
    restriction: Optional[Tuple[int, ...]] = None
    reuse: Optional[Tuple[int, ...]] = None
    flags: int = 0
    graph: str = "symmetric"  # the CSR the pattern is counted on


_RD = PATTERN_RESTRICT | PATTERN_DISTINCT
# SMOG's query patterns (SMOG/SMOG_hie/script_hie.py:85-152), each with the
# graph the reference counts it on (SMOG/SMOG_hie/common_hie.cu:72-85: the
# oriented files for Q0, Q3, Q5 and Q7 -- triangles and 4-, 5-, 6-cliques --
# the symmetric ones for the rest).
PATTERNS = {
    "Q0": PatternSpec(3, (0, 1, 3), (0, 0, 1), graph="oriented"),
    "Q1": PatternSpec(4, (0, 1, 2, 4), (0, 0, 1, 2), (-1, 0, 1, 0), None, PATTERN_RESTRICT),
    "Q2": PatternSpec(4, (0, 1, 3, 5), (0, 0, 1, 1, 2), (-1, -1, 1, 0), None, PATTERN_RESTRICT),
    "Q3": PatternSpec(4, (0, 1, 3, 5), (0, 0, 1, -1, 2), None, (-1, -1, -1, 2),
                      graph="oriented"),
    "Q4": PatternSpec(5, (0, 1, 3, 5, 6), (0, 0, 1, -1, 2, -1), (-1, 0, -1, 2, -1),
                      (-1, -1, -1, 2, 2), _RD),
    "Q5": PatternSpec(5, (0, 1, 3, 5, 7), (0, 0, 1, -1, 2, -1, 3), None, (-1, -1, -1, 2, 3),
                      graph="oriented"),
    "Q6": PatternSpec(5, (0, 1, 3, 4, 6), (0, 0, 1, -1, 2, 3), (-1, 0, -1, 2, -1),
                      (-1, -1, -1, 2, -1), _RD),
    "Q7": PatternSpec(6, (0, 1, 3, 5, 7, 9), (0, 0, 1, -1, 2, -1, 3, -1, 4), None,
                      (-1, -1, -1, 2, 3, 4), graph="oriented"),
    "Q8": PatternSpec(5, (0, 1, 3, 5, 6), (0, 0, 1, -1, 2, -1), (-1, 0, -1, -1, 3),
                      (-1, -1, -1, 2, 3), PATTERN_RESTRICT),
}


def pattern_struct(p: PatternSpec):
    """-> (reset_pattern, the int32 arrays it points to); checks the array
    lengths the C side cannot."""
    k = p.k
    if len(p.offsets) != k:
        raise ValueError("offsets needs k entries")
    if len(p.backward) < p.offsets[-1]:
        raise ValueError("backward needs offsets[k-1] entries")
    for a in (p.restriction, p.reuse):
        if a is not None and len(a) != k:
            raise ValueError("restriction and reuse need k entries")
    arrs = [None if a is None else (C.c_int32 * max(len(a), 1))(*a)
            for a in (p.offsets, p.backward, p.restriction, p.reuse)]
    ptrs = [C.cast(a, C.POINTER(C.c_int32)) if a is not None else None for a in arrs]
    return Pattern(k, p.flags, *ptrs), arrs


def pattern_count(t: Table, off: torch.Tensor, cols: torch.Tensor, pattern, stream=None) -> int:
    """Embeddings of `pattern` (a PatternSpec or a PATTERNS name) in the
    graph the table was built on (SMOG's subgraph matching)."""
    p = PATTERNS[pattern] if isinstance(pattern, str) else pattern
    ps, _keep = pattern_struct(p)
    out = torch.zeros(1, dtype=torch.int64, device=cols.device)
    check(_lib().reset_pattern_count(t.handle, _ptr(off), _ptr(cols), cols.numel(), C.byref(ps),
                                     _ptr(out), _stream(stream)))
    return int(out.item()) & ((1 << 64) - 1)


def sss(t: Table, off, elems, pa, pb, num: int = 7, den: int = 10,
        with_inter: bool = True, stream=None):
    """Integer-rule set-similarity decisions -> (flags uint8, inter int32)."""
    P = pa.numel()
    flags = torch.empty(P, dtype=torch.uint8, device=pa.device)
    inter = torch.empty(P, dtype=torch.int32, device=pa.device) if with_inter else None
    check(_lib().reset_sss(t.handle, _ptr(off), _ptr(elems), _ptr(pa), _ptr(pb), P,
                           num, den, _ptr(flags), _ptr(inter), _stream(stream)))
    return flags, inter


def sss_float(t: Table, off, elems, pa, pb, thr: float, with_inter: bool = True,
              stream=None):
    """Reference float-rule decisions (sss.cu:139-141) -> (flags, inter)."""
    P = pa.numel()
    flags = torch.empty(P, dtype=torch.uint8, device=pa.device)
    inter = torch.empty(P, dtype=torch.int32, device=pa.device) if with_inter else None
    check(_lib().reset_sss_float(t.handle, _ptr(off), _ptr(elems), _ptr(pa), _ptr(pb),
                                 P, C.c_float(thr), _ptr(flags), _ptr(inter),
                                 _stream(stream)))
    return flags, inter


def ir_result_offsets(toff: torch.Tensor, query: torch.Tensor, qoff: torch.Tensor) -> torch.Tensor:
    """res_off[q+1] = res_off[q] + df(first term of q) (ir.cu:324-330); 0 for
    empty queries.  Plain tensor arithmetic (input plumbing)."""
    Q = qoff.numel() - 1
    ql = qoff[1:] - qoff[:-1]
    first = query[qoff[:-1].clamp(max=max(query.numel() - 1, 0)).long()] if query.numel() else \
        torch.zeros(Q, dtype=torch.int32, device=qoff.device)
    df = (toff[first.long() + 1] - toff[first.long()]).to(torch.int64)
    df = torch.where(ql > 0, df, torch.zeros_like(df))
    roff = torch.zeros(Q + 1, dtype=torch.int64, device=qoff.device)
    roff[1:] = torch.cumsum(df, 0)
    return roff


def ir(t: Table, toff, docs, query, qoff, res_off=None, stream=None):
    """Conjunctive retrieval -> (res_off int64[Q+1], res int32, cnt int32[Q])."""
    Q = qoff.numel() - 1
    if res_off is None:
        res_off = ir_result_offsets(toff, query, qoff)
    total = int(res_off[-1].item()) if Q > 0 else 0
    res = torch.full((max(total, 1),), -1, dtype=torch.int32, device=docs.device)
    cnt = torch.zeros(max(Q, 1), dtype=torch.int32, device=docs.device)
    check(_lib().reset_ir(t.handle, _ptr(toff), _ptr(docs), _ptr(query), _ptr(qoff), Q,
                          _ptr(res_off), _ptr(res), _ptr(cnt), _stream(stream)))
    return res_off, res[:total], cnt[:Q]


def intersect_count(a: torch.Tensor, b: torch.Tensor, alpha: float = 0.2,
                    bucket: int = 5, stream=None) -> int:
    out = torch.zeros(1, dtype=torch.int64, device=a.device)
    p = params(alpha, bucket)
    check(_lib().reset_intersect_count(_ptr(a), a.numel(), _ptr(b), b.numel(),
                                       C.byref(p), _ptr(out), _stream(stream)))
    return int(out.item())


def gen_rmat(scale: int, edge_factor: int = 16, seed: int = 0x5EED0016,
             a: float = 0.57, b: float = 0.19, c: float = 0.19,
             oriented: bool = True, relabel: bool = True, stream=None):
    """Seeded R-MAT CSR generated on the device -> (off int32, cols int32)."""
    L = _lib()
    po, pc, m = C.c_void_p(), C.c_void_p(), C.c_int64()
    opts = (0 if oriented else 1) | (0 if relabel else 2)
    check(L.reset_gen_rmat(scale, edge_factor, seed, a, b, c, opts,
                           C.byref(po), C.byref(pc), C.byref(m), _stream(stream)))
    try:
        n = 1 << scale
        off = _view(po.value, n + 1, torch.int32).clone()
        cols = _view(pc.value, m.value, torch.int32).clone()
        torch.cuda.current_stream().synchronize()
    finally:
        L.reset_free(po)
        L.reset_free(pc)
    return off, cols


def get_tuning() -> dict:
    t = Tuning()
    check(_lib().reset_get_tuning(C.byref(t)))
    return {"probe_rounds": t.probe_rounds, "warp_pair_min": t.warp_pair_min,
            "probe_variant": t.probe_variant, "pair_method": t.pair_method}


# reset_tuning.pair_method values
PAIR_DEFAULT, PAIR_FLAT, PAIR_OWNER = 0, 1, 2


def set_tuning(probe_rounds: Optional[int] = None, warp_pair_min: Optional[int] = None,
               probe_variant: Optional[int] = None, pair_method: Optional[int] = None):
    t = Tuning()
    check(_lib().reset_get_tuning(C.byref(t)))
    if probe_rounds is not None:
        t.probe_rounds = probe_rounds
    if warp_pair_min is not None:
        t.warp_pair_min = warp_pair_min
    if probe_variant is not None:
        t.probe_variant = probe_variant
    if pair_method is not None:
        t.pair_method = pair_method
    check(_lib().reset_set_tuning(C.byref(t)))


class Batch:
    """Batched set-similarity decisions over one table (reset_batch_*): a
    captured CUDA graph of the persistent pair kernel with device pair
    buffers for up to `capacity` pairs.  Fill `pair_a` / `pair_b` (views of
    the batch's own buffers), call run(npairs), read `flags` / `inter`
    (`inter` is not written when decisions_only)."""

    def __init__(self, t: Table, elems: torch.Tensor, capacity: int, num: int = 7,
                 den: int = 10, decisions_only: bool = False, owner_grouped: bool = False,
                 stream=None):
        """owner_grouped: the replay groups the pairs by the larger set and
        stages its table in shared memory (full sizes; faster when many
        pairs share a large set)."""
        _need(elems, torch.int32, "elems")
        self._table = t          # the batch reads the table's device arrays
        self._elems = elems
        self.capacity = int(capacity)
        self.decisions_only = bool(decisions_only)
        h = C.c_void_p()
        opts = (1 if decisions_only else 0) | (2 if owner_grouped else 0)
        check(_lib().reset_batch_create_ex(t.handle, _ptr(elems), self.capacity, num, den,
                                           opts, C.byref(h), _stream(stream)))
        self._h = h
        pa, pb, fl, it = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(_lib().reset_batch_buffers(h, C.byref(pa), C.byref(pb), C.byref(fl),
                                         C.byref(it)))
        self.pair_a = _view(pa.value, self.capacity, torch.int32)
        self.pair_b = _view(pb.value, self.capacity, torch.int32)
        self.inter = _view(it.value, self.capacity, torch.int32)
        self.flags = torch.as_tensor(_CudaArray(fl.value, self.capacity, "|u1"),
                                     device="cuda")

    def run(self, npairs: int, stream=None):
        check(_lib().reset_batch_run(self._h, int(npairs), _stream(stream)))

    def __call__(self, pa: torch.Tensor, pb: torch.Tensor, stream=None):
        """Copy pairs in, run, and return (flags, inter) views of length P."""
        P = pa.numel()
        if P > self.capacity:
            raise ValueError(f"{P} pairs exceed the batch capacity {self.capacity}")
        s = stream if stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(s):
            self.pair_a[:P].copy_(pa, non_blocking=True)
            self.pair_b[:P].copy_(pb, non_blocking=True)
        self.run(P, s)
        return self.flags[:P], self.inter[:P]

    def close(self):
        if getattr(self, "_h", None):
            check(_lib().reset_batch_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gen_token_sets(n: int, universe_log2: int = 20, size_s: float = 1.6,
                   size_lo: int = 8, size_hi: int = 512, seed: int = 0x5EED0033,
                   dup_frac: float = 0.0, keep_min: float = 0.8, stream=None):
    """Seeded token sets on the device -> (off int32[n+1], tokens int32);
    dup_frac of them planted near-duplicates (see reset_gen_token_sets)."""
    L = _lib()
    po, pt, m = C.c_void_p(), C.c_void_p(), C.c_int64()
    check(L.reset_gen_token_sets(n, universe_log2, size_s, size_lo, size_hi, dup_frac,
                                 keep_min, seed,
                                 C.byref(po), C.byref(pt), C.byref(m), _stream(stream)))
    try:
        off = _view(po.value, n + 1, torch.int32).clone()
        tok = _view(pt.value, m.value, torch.int32).clone()
        torch.cuda.current_stream().synchronize()
    finally:
        L.reset_free(po)
        L.reset_free(pt)
    return off, tok


def gen_inverted_index(nterms: int, ndocs: int, zipf_s: float = 1.1,
                       df_max: Optional[int] = None, seed: int = 0x5EED0044, stream=None):
    """Seeded inverted index on the device -> (toff int32[nterms+1], docs int32)."""
    L = _lib()
    df_max = ndocs // 2 if df_max is None else df_max
    po, pd, m = C.c_void_p(), C.c_void_p(), C.c_int64()
    check(L.reset_gen_inverted_index(nterms, ndocs, zipf_s, df_max, seed, C.byref(po),
                                     C.byref(pd), C.byref(m), _stream(stream)))
    try:
        toff = _view(po.value, nterms + 1, torch.int32).clone()
        docs = _view(pd.value, m.value, torch.int32).clone()
        torch.cuda.current_stream().synchronize()
    finally:
        L.reset_free(po)
        L.reset_free(pd)
    return toff, docs


def prefix_candidates(off: torch.Tensor, tokens: torch.Tensor, universe_log2: int,
                      num: int = 7, den: int = 10, stream=None):
    """Prefix-filter candidate pairs (a < b, sorted) -> (pa, pb) int32."""
    _need(off, torch.int32, "off")
    _need(tokens, torch.int32, "tokens")
    L = _lib()
    pa, pb, npr = C.c_void_p(), C.c_void_p(), C.c_int64()
    check(L.reset_prefix_candidates(_ptr(off), _ptr(tokens), off.numel() - 1,
                                    tokens.numel(), universe_log2, num, den,
                                    C.byref(pa), C.byref(pb), C.byref(npr),
                                    _stream(stream)))
    try:
        a = _view(pa.value, npr.value, torch.int32).clone()
        b = _view(pb.value, npr.value, torch.int32).clone()
        torch.cuda.current_stream().synchronize()
    finally:
        L.reset_free(pa)
        L.reset_free(pb)
    return a, b

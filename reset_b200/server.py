"""Served form over the C ABI (reset_server_* in include/reset.h).

    srv = Server(streams=4)
    ix = srv.add_index(table)            # a reset_b200.api.Table, kept alive
    t = srv.submit_ir(ix, [17, 4, 99])   # -> ticket, returns at once
    r = srv.wait(t)                      # Result: docs / values / flags / latency

Requests are queued as they arrive and run in continuous batches on the
GPU; see reset_server_create for the admission rule.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from ._lib import Request, Result, ServerConfig, ServerCounters, check, load

IR, PAIRS, TRIPLES, TC_VERTEX, RAW = 1, 2, 3, 4, 5


@dataclass
class ServedResult:
    status: int
    kind: int
    count: int
    docs: Optional[np.ndarray]
    values: Optional[np.ndarray]
    flags: Optional[np.ndarray]
    queue_us: float
    service_us: float
    latency_us: float
    batch_id: int
    batch_size: int


def now_ns() -> int:
    return int(load().reset_now_ns())


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())


class Server:
    def __init__(self, streams: int = 4, max_batch_requests: int = 1024,
                 mem_budget_bytes: int = 0, max_batch_cost: Optional[int] = None,
                 pinned_result_bytes: Optional[int] = None):
        L = load()
        cfg = ServerConfig()
        L.reset_server_config_default(C.byref(cfg))
        cfg.streams = streams
        cfg.max_batch_requests = max_batch_requests
        cfg.mem_budget_bytes = mem_budget_bytes
        if max_batch_cost is not None:   # estimated probes per batch; 0 = no limit
            cfg.max_batch_cost = max_batch_cost
        if pinned_result_bytes is not None:   # host arena for IR results
            cfg.pinned_result_bytes = pinned_result_bytes
        h = C.c_void_p()
        check(L.reset_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._keep: List[object] = []   # tables and arrays the indexes read

    def add_index(self, table) -> int:
        """Registers a reset_b200.api.Table (built on its own off/elems)."""
        out = C.c_int32()
        check(load().reset_server_add_index(self._h, table.handle,
                                            C.c_void_p(table.off.data_ptr()),
                                            C.c_void_p(table.elems.data_ptr()),
                                            C.byref(out)))
        self._keep.append(table)
        return out.value

    def submit(self, kind: int, index: int = 0, args: Sequence[int] = (),
               args2: Sequence[int] = (), num: int = 7, den: int = 10,
               arrival_ns: int = 0) -> int:
        a = _i32(args)
        b = _i32(args2)
        q = Request()
        q.kind = kind
        q.index = index
        q.args = a.ctypes.data_as(C.POINTER(C.c_int32))
        q.nargs = a.size
        q.args2 = b.ctypes.data_as(C.POINTER(C.c_int32))
        q.nargs2 = b.size
        q.num = num
        q.den = den
        q.arrival_ns = arrival_ns
        t = C.c_uint64()
        check(load().reset_server_submit(self._h, C.byref(q), C.byref(t)))
        return t.value

    def submit_ir(self, index: int, terms, arrival_ns: int = 0) -> int:
        return self.submit(IR, index, terms, arrival_ns=arrival_ns)

    def submit_pairs(self, index: int, pa, pb, num: int = 7, den: int = 10,
                     arrival_ns: int = 0) -> int:
        ab = np.empty(2 * len(pa), np.int32)
        ab[0::2] = pa
        ab[1::2] = pb
        return self.submit(PAIRS, index, ab, num=num, den=den, arrival_ns=arrival_ns)

    def submit_triples(self, index: int, triples, arrival_ns: int = 0) -> int:
        return self.submit(TRIPLES, index, np.asarray(triples, np.int32).ravel(),
                           arrival_ns=arrival_ns)

    def submit_tc_vertices(self, index: int, vertices, arrival_ns: int = 0) -> int:
        return self.submit(TC_VERTEX, index, vertices, arrival_ns=arrival_ns)

    def submit_raw(self, a, b, arrival_ns: int = 0) -> int:
        return self.submit(RAW, 0, a, b, arrival_ns=arrival_ns)

    def wait(self, ticket: int, timeout_ms: int = -1, release: bool = True,
             copy_out: bool = True) -> ServedResult:
        """Blocks until the request is done.  copy_out=False skips copying
        the result arrays (docs, values and flags are then None; the count
        and timings are kept)."""
        r = Result()
        check(load().reset_server_wait(self._h, ticket, timeout_ms, C.byref(r)))
        docs = vals = flags = None
        if copy_out:
            docs = np.ctypeslib.as_array(r.docs, shape=(r.ndocs,)).copy() if r.ndocs else None
            vals = (np.ctypeslib.as_array(r.values, shape=(r.nvalues,)).copy()
                    if r.nvalues else None)
            flags = (np.ctypeslib.as_array(r.flags, shape=(r.nvalues,)).copy()
                     if r.nvalues and r.flags else None)
        out = ServedResult(r.status, r.kind, r.count, docs, vals, flags, r.queue_us,
                           r.service_us, r.latency_us, r.batch_id, r.batch_size)
        if release:
            check(load().reset_server_release(self._h, ticket))
        return out

    def stats(self) -> dict:
        c = ServerCounters()
        check(load().reset_server_stats(self._h, C.byref(c)))
        return {k: getattr(c, k) for k, _ in ServerCounters._fields_ if k != "reserved"}

    def close(self):
        if getattr(self, "_h", None):
            check(load().reset_server_destroy(self._h))
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

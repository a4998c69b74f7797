"""CPU oracle for the RESET set-intersection path -- TEST INFRASTRUCTURE ONLY.

numpy/ctypes front end of ``oracle.c``, the plain-C restatement of the
reference algorithms (table layout and build, probe rule, hash-order
extraction, triangle counting, set-similarity search, conjunctive IR, raw
pair intersection, and the seeded R-MAT generator).  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may use
it, and only as the checker.  The product (``reset_b200``) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


class _Csr(C.Structure):
    _fields_ = [("n", C.c_int32), ("m", C.c_int64),
                ("off", C.POINTER(C.c_int32)), ("cols", C.POINTER(C.c_int32))]


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (gcc, no GPU)."""
    src = os.path.join(HERE, "oracle.c")
    if force or not os.path.exists(LIB_PATH) or \
            os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(build())
        L.ro_calc_len.argtypes = [C.c_int32, C.c_float, C.c_int32]
        L.ro_calc_len.restype = C.c_int32
        L.ro_hash_normal.argtypes = [C.c_int32, C.c_int32]
        L.ro_hash_normal.restype = C.c_int32
        L.ro_hash_hier.argtypes = [C.c_int32, C.c_int32, C.c_int32]
        L.ro_hash_hier.restype = C.c_int32
        L.ro_table_meta.argtypes = [C.c_int32, _i32p, C.c_float, C.c_int32,
                                    _i32p, _i64p, C.POINTER(C.c_int32)]
        L.ro_table_meta.restype = C.c_int64
        L.ro_table_build.argtypes = [C.c_int32, _i32p, _i32p, C.c_int32, _i32p,
                                     _i64p, C.c_int64, C.c_int32, C.c_int32,
                                     _i32p]
        L.ro_table_build.restype = C.c_int32
        L.ro_hash_order.argtypes = [C.c_int32, _i32p, _i64p, _i32p, C.c_int64,
                                    C.c_int32, _i32p]
        L.ro_hash_order.restype = None
        L.ro_tc_merge.argtypes = [C.c_int32, _i32p, _i32p, C.c_int32]
        L.ro_tc_merge.restype = C.c_uint64
        L.ro_tc_merge_range.argtypes = [C.c_int32, _i32p, _i32p, C.c_int32,
                                        C.c_int32, C.c_int32]
        L.ro_tc_merge_range.restype = C.c_uint64
        L.ro_tc_hash.argtypes = [C.c_int32, _i32p, _i32p, _i32p, _i64p, _i32p,
                                 C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                 C.c_int32]
        L.ro_tc_hash.restype = C.c_uint64
        L.ro_sss.argtypes = [C.c_int32, _i32p, _i32p, _i32p, _i32p, C.c_int64,
                             _i32p, _i64p, _i32p, C.c_int64, C.c_int32,
                             C.c_int32, C.c_int32, C.c_int32, C.c_float,
                             C.c_int32, C.c_int32, _u8p, _i32p]
        L.ro_sss.restype = None
        L.ro_ir.argtypes = [C.c_int32, _i32p, _i32p, _i32p, _i32p, C.c_int32,
                            _i64p, _i32p, _i64p, _i32p, C.c_int64, C.c_int32,
                            C.c_int32, C.c_int32, _i32p, _i32p]
        L.ro_ir.restype = None
        L.ro_pair_count.argtypes = [_i32p, C.c_int64, _i32p, C.c_int64]
        L.ro_pair_count.restype = C.c_int64
        L.ro_jaccard_join.argtypes = [C.c_int32, _i32p, _i32p, C.c_int32,
                                      C.c_int32, _i32p, _i32p, C.c_int64]
        L.ro_jaccard_join.restype = C.c_int64
        L.ro_clique4.argtypes = [C.c_int32, _i32p, _i32p]
        L.ro_clique4.restype = C.c_uint64
        L.ro_clique_k.argtypes = [C.c_int32, _i32p, _i32p, C.c_int32]
        L.ro_clique_k.restype = C.c_uint64
        L.ro_pattern_count.argtypes = [C.c_int32, _i32p, _i32p, C.c_int32, C.c_int32,
                                       _i32p, _i32p, C.c_void_p, C.c_void_p, C.c_int32]
        L.ro_pattern_count.restype = C.c_uint64
        L.ro_relabel.argtypes = [C.c_uint64, C.c_int32, C.c_uint32]
        L.ro_relabel.restype = C.c_uint32
        L.ro_mix64.argtypes = [C.c_uint64]
        L.ro_mix64.restype = C.c_uint64
        L.ro_rmat_graph.argtypes = [C.c_int32, C.c_int32, C.c_uint64,
                                    C.c_double, C.c_double, C.c_double,
                                    C.c_int32]
        L.ro_rmat_graph.restype = C.POINTER(_Csr)
        L.ro_csr_free.argtypes = [C.POINTER(_Csr)]
        L.ro_csr_free.restype = None
        _lib = L
    return _lib


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ---------------------------------------------------------------- layout ----

def calc_len(degree: int, alpha: float = 0.2, bucket: int = 5) -> int:
    return int(lib().ro_calc_len(degree, alpha, bucket))


def table_meta(off, alpha=0.2, bucket=5):
    """-> (len int32[n], off64 int64[n+1], bucket_num, max_len)."""
    off = _c(off, np.int32)
    n = off.size - 1
    ln = np.zeros(max(n, 1), np.int32)
    o64 = np.zeros(n + 1, np.int64)
    mx = C.c_int32(0)
    bn = lib().ro_table_meta(n, off, alpha, bucket, ln, o64, C.byref(mx))
    return ln[:n], o64, int(bn), int(mx.value)


class Table:
    """A per-set bucketed table in the reference layout (slot-major)."""

    def __init__(self, off, elems, alpha=0.2, bucket=5, hier=True):
        self.off = _c(off, np.int32)
        self.elems = _c(elems, np.int32)
        self.n = self.off.size - 1
        self.bucket = bucket
        self.hier = int(bool(hier))
        self.len, self.off64, self.bucket_num, self.max_len = table_meta(
            self.off, alpha, bucket)
        self.table = np.empty(max(bucket * self.bucket_num, 1), np.int32)
        st = lib().ro_table_build(self.n, self.off, self.elems, bucket,
                                  _c(self.len, np.int32) if self.n else np.zeros(1, np.int32),
                                  self.off64, self.bucket_num, self.max_len,
                                  self.hier, self.table)
        if st != 0:
            raise RuntimeError("oracle table overflow")
        self.table = self.table[:bucket * self.bucket_num]

    def _lenp(self):
        return self.len if self.n else np.zeros(1, np.int32)

    def hash_order(self):
        out = self.elems.copy()
        lib().ro_hash_order(self.n, self.off, self.off64,
                            self.table if self.table.size else np.zeros(1, np.int32),
                            self.bucket_num, self.bucket, out)
        return out


# ----------------------------------------------------------- applications ---

def tc_merge(off, cols, nthreads: int = 0) -> int:
    off = _c(off, np.int32)
    return int(lib().ro_tc_merge(off.size - 1, off, _c(cols, np.int32), nthreads))


def tc_merge_range(off, cols, v0, v1, nthreads: int = 0) -> int:
    off = _c(off, np.int32)
    return int(lib().ro_tc_merge_range(off.size - 1, off, _c(cols, np.int32),
                                       v0, v1, nthreads))


def tc_hash(t: Table, cols=None, nthreads: int = 0) -> int:
    cols = t.elems if cols is None else _c(cols, np.int32)
    return int(lib().ro_tc_hash(t.n, t.off, cols, t._lenp(), t.off64, t.table,
                                t.bucket_num, t.max_len, t.bucket, t.hier,
                                nthreads))


def sss(t: Table, pa, pb, mode=1, thr=0.7, num=7, den=10, elems=None):
    """-> (flags uint8[P], inter int32[P])."""
    pa = _c(pa, np.int32)
    pb = _c(pb, np.int32)
    P = pa.size
    flags = np.zeros(max(P, 1), np.uint8)
    inter = np.zeros(max(P, 1), np.int32)
    el = t.elems if elems is None else _c(elems, np.int32)
    lib().ro_sss(t.n, t.off, el if el.size else np.zeros(1, np.int32),
                 pa if P else np.zeros(1, np.int32),
                 pb if P else np.zeros(1, np.int32), P, t._lenp(), t.off64,
                 t.table, t.bucket_num, t.max_len, t.bucket, t.hier, mode, thr,
                 num, den, flags, inter)
    return flags[:P], inter[:P]


def ir(t: Table, query, qoff, docs=None):
    """-> (res_off int64[Q+1], result int32[...], count int32[Q])."""
    query = _c(query, np.int32)
    qoff = _c(qoff, np.int32)
    Q = qoff.size - 1
    docs = t.elems if docs is None else _c(docs, np.int32)
    df = np.diff(t.off)
    roff = np.zeros(Q + 1, np.int64)
    for q in range(Q):
        roff[q + 1] = roff[q] + (df[query[qoff[q]]] if qoff[q + 1] > qoff[q] else 0)
    res = np.full(max(int(roff[-1]), 1), -1, np.int32)
    cnt = np.zeros(max(Q, 1), np.int32)
    lib().ro_ir(t.n, t.off, docs if docs.size else np.zeros(1, np.int32),
                query if query.size else np.zeros(1, np.int32), qoff, Q, roff,
                t._lenp(), t.off64, t.table, t.bucket_num, t.max_len, t.bucket,
                t.hier, res, cnt)
    return roff, res[:int(roff[-1])], cnt[:Q]


def pair_count(a, b) -> int:
    a = _c(a, np.int32)
    b = _c(b, np.int32)
    return int(lib().ro_pair_count(a if a.size else np.zeros(1, np.int32), a.size,
                                   b if b.size else np.zeros(1, np.int32), b.size))


def clique4(off, cols) -> int:
    """4-cliques of an oriented graph with sorted rows."""
    off = _c(off, np.int32)
    cols = _c(cols, np.int32)
    return int(lib().ro_clique4(off.size - 1, off, cols if cols.size else np.zeros(1, np.int32)))


def clique_k(off, cols, k: int) -> int:
    """k-cliques (k >= 3) of an oriented graph with sorted rows (ro_clique_k)."""
    off = _c(off, np.int32)
    cols = _c(cols, np.int32)
    return int(lib().ro_clique_k(off.size - 1, off, cols if cols.size else np.zeros(1, np.int32),
                                 k))


def pattern_count(off, cols, k, flags, offsets, backward, restriction=None, reuse=None,
                  nthreads=0) -> int:
    """Embeddings of a pattern in SMOG's encoding (ro_pattern_count); rows
    must be sorted."""
    off = _c(off, np.int32)
    cols = _c(cols, np.int32)
    offsets = _c(offsets, np.int32)
    backward = _c(backward, np.int32)
    keep = [_c(a, np.int32) if a is not None else None for a in (restriction, reuse)]
    ptrs = [a.ctypes.data_as(C.c_void_p) if a is not None else None for a in keep]
    return int(lib().ro_pattern_count(off.size - 1, off, cols if cols.size else np.zeros(1, np.int32),
                                      k, flags, offsets, backward, ptrs[0], ptrs[1], nthreads))


def jaccard_join(off, tok, num=7, den=10):
    """All pairs a < b with den*I >= num*U, U > 0 (brute force; small n)."""
    off = _c(off, np.int32)
    tok = _c(tok, np.int32)
    n = off.size - 1
    cap = n * (n - 1) // 2 + 1
    pa = np.zeros(cap, np.int32)
    pb = np.zeros(cap, np.int32)
    k = int(lib().ro_jaccard_join(n, off, tok if tok.size else np.zeros(1, np.int32),
                                  num, den, pa, pb, cap))
    return pa[:k], pb[:k]


def prefix_candidates(off, tok, num=7, den=10):
    """Restated prefix filter: tokens ranked by (min(freq, 2^19-1), id);
    prefix of x = first |x| - ceil(num|x|/den) + 1 tokens in that order;
    candidates = pairs a < b sharing a prefix token with
    den*min(|a|,|b|) >= num*max(|a|,|b|).  Returns (pa, pb) sorted."""
    off = np.asarray(off, np.int64)
    tok = np.asarray(tok, np.int64)
    n = off.size - 1
    sz = np.diff(off)
    freq = np.bincount(tok, minlength=int(tok.max()) + 1 if tok.size else 1)
    freq = np.minimum(freq, (1 << 19) - 1)
    by_token = {}
    for x in range(n):
        row = tok[off[x]:off[x + 1]]
        order = row[np.lexsort((row, freq[row]))]
        p = int(sz[x] - (num * sz[x] + den - 1) // den + 1) if sz[x] > 0 else 0
        for t in order[:p].tolist():
            by_token.setdefault(t, []).append(x)
    out = set()
    for sets in by_token.values():
        for i in range(len(sets)):
            for j in range(i + 1, len(sets)):
                a, b = sets[i], sets[j]
                lo, hi = min(sz[a], sz[b]), max(sz[a], sz[b])
                if den * lo >= num * hi:
                    out.add((min(a, b), max(a, b)))
    if not out:
        return np.zeros(0, np.int32), np.zeros(0, np.int32)
    arr = np.array(sorted(out), np.int32)
    return arr[:, 0].copy(), arr[:, 1].copy()


# ------------------------------------------------------------- generators ---

def rmat_graph(scale, edge_factor=16, seed=0x5EED0016, a=0.57, b=0.19, c=0.19,
               oriented=True, relabel=True):
    """-> (off int32[n+1], cols int32[m]) (see ro_rmat_graph)."""
    mode = (0 if oriented else 1) | (0 if relabel else 2)
    g = lib().ro_rmat_graph(scale, edge_factor, seed, a, b, c, mode)
    try:
        n, m = g.contents.n, g.contents.m
        off = np.ctypeslib.as_array(g.contents.off, shape=(n + 1,)).copy()
        cols = np.ctypeslib.as_array(g.contents.cols, shape=(max(m, 1),))[:m].copy()
    finally:
        lib().ro_csr_free(g)
    return off, cols


def mix64(z: int) -> int:
    return int(lib().ro_mix64(z))

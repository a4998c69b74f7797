"""reset_tc_count_noalloc: the triangle count for callers that cannot
allocate device memory while they run (its scratch is a fixed device array
inside libreset.so).  Checked through the C ABI against the allocating entry
point, reset_tc_count, on two calls in a row -- the second call reuses the
scratch the first one left behind.  Collected last on purpose, and written to
pass alone in a fresh process as well as after the other tests."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _noalloc(lib, torch, table, off, cols):
    out = torch.full((1,), -7, dtype=torch.int64, device="cuda")
    st = lib.reset_tc_count_noalloc(table.handle, _ptr(off), _ptr(cols), cols.numel(),
                                    _ptr(out), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, lib.reset_last_error_string()
    torch.cuda.synchronize()
    return int(out.item())


@pytest.mark.parametrize("hier", [True, False])
def test_noalloc_equals_allocating_entry_point(cuda, libreset, hier):
    torch = cuda
    from reset_b200 import api
    off, cols = api.gen_rmat(15, 16, 0x5EED0015, oriented=True)
    t = api.Table(off, cols, hierarchical=hier, hash_order=True)
    want = api.tc_count(t, off, t.hash_order)          # reset_tc_count (allocates)
    assert want > 0
    for _ in range(2):                                  # two calls in a row
        assert _noalloc(libreset, torch, t, off, t.hash_order) == want
    t.check()


def test_noalloc_second_table_and_shapes(cuda, libreset):
    """A second, differently shaped table after the first one: rows long
    enough for the CTA work units, so the shared unit list is refilled."""
    torch = cuda
    from reset_b200 import api
    rng = np.random.default_rng(2)
    n = 6000
    sizes = rng.integers(0, 60, size=n)
    sizes[:8] = [300, 700, 1500, 257, 256, 4096, 5000, 33]
    rows = [np.sort(rng.choice(n, size=s, replace=False)) for s in sizes]
    off = np.zeros(n + 1, np.int32)
    off[1:] = np.cumsum(sizes)
    cols = np.concatenate(rows).astype(np.int32)
    d_off = torch.from_numpy(off).cuda()
    d_cols = torch.from_numpy(cols).cuda()
    t = api.Table(d_off, d_cols, hierarchical=True)
    want = api.tc_count(t, d_off, d_cols)
    for _ in range(2):
        assert _noalloc(libreset, torch, t, d_off, d_cols) == want


def test_noalloc_rejects_what_it_cannot_hold(cuda, libreset):
    torch = cuda
    from reset_b200 import api
    off, cols = api.gen_rmat(8, 8, 1, oriented=True)
    t = api.Table(off, cols)
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # more edges than the fixed scratch can schedule: refused on the host
    st = libreset.reset_tc_count_noalloc(t.handle, _ptr(off), _ptr(cols), 200_000_000,
                                         _ptr(out), s)
    assert st == 3 and b"at most" in libreset.reset_last_error_string()
    # offsets other than the build's would need a fresh descriptor array
    st = libreset.reset_tc_count_noalloc(t.handle, _ptr(off.clone()), _ptr(cols),
                                         cols.numel(), _ptr(out), s)
    assert st == 3
    # a column count other than the table's: rows are walked through the
    # build-time descriptors, so a shorter array would be read past its end
    st = libreset.reset_tc_count_noalloc(t.handle, _ptr(off), _ptr(cols),
                                         cols.numel() - 1, _ptr(out), s)
    assert st == 3 and b"edge count" in libreset.reset_last_error_string()


@pytest.mark.parametrize("name", ["tc_s10", "tc_s11_a05_b3"])
def test_noalloc_equals_reference_golden_count(cuda, libreset, name):
    """Against the triangle counts the reference's own kernel produced on the
    same graphs (golden fixtures), both hashes, on the fixture's alpha and
    bucket size."""
    import os
    torch = cuda
    from reset_b200 import api
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    _, _, c_norm, c_hier = (int(x) for x in g["ref_meta"])
    off = torch.from_numpy(g["off"]).cuda()
    cols = torch.from_numpy(g["cols"]).cuda()
    for hier, want in ((False, c_norm), (True, c_hier)):
        t = api.Table(off, cols, alpha=float(g["alpha"]), bucket=int(g["bucket"]),
                      hierarchical=hier)
        for _ in range(2):
            assert _noalloc(libreset, torch, t, off, cols) == want
        t.check()

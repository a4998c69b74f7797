"""C-ABI boundary checks that need no GPU: the library loads, and exports
every entry point include/reset.h declares, with bindings for each."""
import ctypes
import os
import re

import pytest
from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "reset.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(reset_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["reset_table_build", "reset_tc_count", "reset_sss", "reset_ir",
                 "reset_intersect_count", "reset_csr_hash_order", "reset_table_free"]:
        assert must in names


def test_library_exports_every_declared_symbol(libreset):
    for name in declared_functions():
        assert hasattr(libreset, name), f"libreset.so does not export {name}"


def test_python_binding_covers_header(libreset):
    from reset_b200 import _lib
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_status_strings_and_version(libreset):
    assert libreset.reset_abi_version() == 1
    assert libreset.reset_status_string(0) == b"RESET_OK"
    assert libreset.reset_status_string(4) == b"RESET_ERR_TABLE_FULL"


def test_params_default(libreset):
    from reset_b200 import _lib
    p = _lib.Params()
    libreset.reset_params_default(ctypes.byref(p))
    assert abs(p.alpha - 0.2) < 1e-7 and p.bucket == 5


def test_build_rejects_bad_arguments_without_touching_the_gpu(libreset):
    # Argument validation happens on the host before any CUDA call.
    from reset_b200 import _lib
    p = _lib.Params()
    libreset.reset_params_default(ctypes.byref(p))
    out = ctypes.c_void_p()
    st = libreset.reset_table_build(None, None, 4, 0, ctypes.byref(p), 1, None,
                                    ctypes.byref(out), None)
    assert st == 3  # RESET_ERR_ARG: NULL offsets
    p.alpha = 1.5
    st = libreset.reset_table_build(ctypes.c_void_p(16), None, 0, 0, ctypes.byref(p), 1,
                                    None, ctypes.byref(out), None)
    assert st == 3 and b"alpha" in libreset.reset_last_error_string()
    p.alpha = 0.2
    p.bucket = 0
    st = libreset.reset_table_build(ctypes.c_void_p(16), None, 0, 0, ctypes.byref(p), 1,
                                    None, ctypes.byref(out), None)
    assert st == 3


def test_no_oracle_in_product():
    """The product package never imports or links the oracle."""
    pkg = os.path.join(ROOT, "reset_b200")
    for dp, _, fs in os.walk(pkg):
        for f in fs:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                txt = open(os.path.join(dp, f)).read()
                assert "import oracle" not in txt and "liboracle" not in txt, f


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors have the C layout: sizes and every field offset,
    printed by a C program compiled against include/reset.h."""
    import subprocess
    from reset_b200 import _lib
    structs = {"reset_params": _lib.Params, "reset_tuning": _lib.Tuning,
               "reset_table_view": _lib.TableView, "reset_server_config": _lib.ServerConfig,
               "reset_request": _lib.Request, "reset_result": _lib.Result,
               "reset_server_counters": _lib.ServerCounters, "reset_pattern": _lib.Pattern}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "reset.h"',
             'int main(void) {']
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append('  return 0; }')
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    got = {}
    for line in out.splitlines():
        cname, key, val = line.split()
        got[(cname, key)] = int(val)
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_new_entry_points_validate_on_the_host(libreset):
    """Argument checks of the batched, served and generator entry points run
    on the host before any CUDA call."""
    from reset_b200 import _lib
    out = ctypes.c_void_p()
    cfg = _lib.ServerConfig()
    libreset.reset_server_config_default(ctypes.byref(cfg))
    assert cfg.streams == 4 and cfg.max_batch_requests == 1024
    cfg.streams = 0
    assert libreset.reset_server_create(ctypes.byref(cfg), ctypes.byref(out)) == 3
    cfg.streams, cfg.max_batch_requests = 4, 0
    assert libreset.reset_server_create(ctypes.byref(cfg), ctypes.byref(out)) == 3
    libreset.reset_server_config_default(ctypes.byref(cfg))
    assert cfg.pinned_result_bytes == 256 << 20 and cfg.max_batch_cost == 1 << 22
    for field in ("pinned_result_bytes", "max_batch_cost", "mem_budget_bytes"):
        libreset.reset_server_config_default(ctypes.byref(cfg))
        setattr(cfg, field, -1)
        assert libreset.reset_server_create(ctypes.byref(cfg), ctypes.byref(out)) == 3, field
    # unknown batch option; NULL table
    assert libreset.reset_batch_create_ex(ctypes.c_void_p(8), ctypes.c_void_p(8), 10, 7, 10,
                                          1 << 5, ctypes.byref(out), None) == 3
    assert libreset.reset_batch_create_ex(None, None, 10, 7, 10, 0, ctypes.byref(out),
                                          None) == 3
    po, pt, m = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_int64()
    assert libreset.reset_gen_token_sets(0, 10, 1.2, 8, 64, 0.0, 0.8, 1, ctypes.byref(po),
                                         ctypes.byref(pt), ctypes.byref(m), None) == 3
    assert libreset.reset_gen_token_sets(10, 10, 1.2, 8, 64, 1.5, 0.8, 1, ctypes.byref(po),
                                         ctypes.byref(pt), ctypes.byref(m), None) == 3
    assert libreset.reset_gen_inverted_index(0, 10, 1.1, 5, 1, ctypes.byref(po),
                                             ctypes.byref(pt), ctypes.byref(m), None) == 3
    assert libreset.reset_server_wait(None, 1, 0, None) == 3
    t = _lib.Tuning()
    libreset.reset_get_tuning(ctypes.byref(t))
    bad = _lib.Tuning(t.probe_rounds, t.warp_pair_min, 7)
    assert libreset.reset_set_tuning(ctypes.byref(bad)) == 3


def test_pattern_count_validates_on_the_host(libreset):
    """reset_pattern_count rejects malformed patterns before any CUDA call
    (a NULL table is checked first, so a dummy handle stands in)."""
    from reset_b200 import api
    fake = ctypes.c_void_p(8)
    cnt = ctypes.c_void_p(8)

    def status(spec):
        ps, _keep = api.pattern_struct(spec)
        return libreset.reset_pattern_count(fake, None, None, 0, ctypes.byref(ps), cnt, None)

    P = api.PatternSpec
    bad = [
        P(2, (0, 1), (0,)),                                  # k < 3
        P(9, tuple(range(9)), (0,) * 8),                     # k > RESET_PATTERN_MAX
        P(3, (0, 1, 3), (1, 0, 1)),                          # level 1 must be [0]
        P(3, (0, 1, 3), (0, 0, 2)),                          # backward not earlier
        P(3, (0, 1, 3), (0, 0, -1)),                         # -1 without reuse
        P(4, (0, 1, 3, 4), (0, 0, 1, 2), None, (-1, -1, -1, 2)),  # reuse without -1
        P(4, (0, 1, 3, 5), (0, 0, 1, -1, 2), None, (-1, -1, -1, 3)),  # reuse not earlier
        P(4, (0, 1, 3, 3), (0, 0, 1)),                       # empty level, no reuse
        P(3, (0, 1, 3), (0, 0, 1), (0, -1, -1), None, 1),    # restriction[0]
        P(3, (0, 1, 3), (0, 0, 1), (-1, 0, 2), None, 1),     # restriction not earlier
        P(3, (0, 1, 3), (0, 0, 1), None, None, 4),           # unknown flag
    ]
    for spec in bad:
        assert status(spec) == 3, spec
    assert libreset.reset_pattern_count(fake, None, None, 0, None, cnt, None) == 3
    ps, _keep = api.pattern_struct(api.PATTERNS["Q4"])
    assert libreset.reset_pattern_count(None, None, None, 0, ctypes.byref(ps), cnt, None) == 3
    with pytest.raises(ValueError):
        api.pattern_struct(P(4, (0, 1, 3), (0, 0, 1)))
    with pytest.raises(ValueError):
        api.pattern_struct(P(3, (0, 1, 3), (0, 0, 1), (-1, 0)))


def test_named_patterns_match_the_python_table(libreset):
    """reset_pattern_named (the C copy of SMOG's Q0..Q8 table) holds the
    same arrays, flags and graph choice as api.PATTERNS."""
    from reset_b200 import _lib, api
    for name, spec in api.PATTERNS.items():
        ps, ori = _lib.Pattern(), ctypes.c_int32(-1)
        assert libreset.reset_pattern_named(name.encode(), ctypes.byref(ps), ctypes.byref(ori)) == 0
        assert (ps.k, ps.flags) == (spec.k, spec.flags), name
        assert ori.value == (1 if spec.graph == "oriented" else 0), name
        assert [ps.offsets[i] for i in range(ps.k)] == list(spec.offsets), name
        nb = spec.offsets[-1]
        assert [ps.backward[i] for i in range(nb)] == list(spec.backward[:nb]), name
        for field in ("restriction", "reuse"):
            want, ptr = getattr(spec, field), getattr(ps, field)
            if want is None:
                assert not ptr, (name, field)
            else:
                assert [ptr[i] for i in range(ps.k)] == list(want), (name, field)
    assert libreset.reset_pattern_named(b"Q9", ctypes.byref(_lib.Pattern()), None) == 3
    assert libreset.reset_pattern_named(None, ctypes.byref(_lib.Pattern()), None) == 3


def test_smog_cli_rejects_bad_input_before_any_gpu_work(libreset, tmp_path):
    """reset_smog checks the pattern name and its graph files on the host."""
    import subprocess
    exe = os.path.join(ROOT, "reset_b200", "bin", "reset_smog")
    if not os.path.exists(exe):
        from reset_b200 import build
        build.build_host_tools()
    r = subprocess.run([exe, str(tmp_path), "Q9"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "unknown pattern" in r.stderr
    r = subprocess.run([exe, str(tmp_path / "missing"), "Q1"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 1 and "cannot open file" in r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "Usage" in r.stderr

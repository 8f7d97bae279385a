"""CPU tests of the C-ABI library: it loads, exports every symbol include/*.h declares,
and rejects bad arguments before touching a device (no compute calls here)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared_symbols() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        for m in re.finditer(r"^CS_API\s+[\w\s\*]+?\b(\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_header_declares_the_entry_points():
    names = _declared_symbols()
    for must in ("compressstore", "compressstore_ex", "cs_popc_chunks", "cs_chunk_prefix_sum", "cs_writeout",
                 "compressstore_workspace_size", "cs_workspace_init"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from gpu_compressstore2_b200 import _lib

    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in sorted(_declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding declares a signature for each
    assert _declared_symbols() <= set(_lib.SIGNATURES)


def test_cub_comparator_exports():
    from gpu_compressstore2_b200 import _lib

    c = _lib.cub()
    assert hasattr(c, "cs_cub_flagged") and hasattr(c, "cs_cub_flagged_temp_bytes")


def test_info_calls():
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    assert L.cs_version() == 0x000100
    assert [cs.tile_elems(w) for w in (1, 2, 4, 8)] == [32768, 16384, 8192, 4096]
    assert cs.tile_elems(3) == 0
    assert L.cs_status_string(-5) == b"bounded device wait timed out"
    assert L.cs_status_string(0) == b"success"


def test_argument_validation_without_device():
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    # bad element width, null count, oversize n: rejected before any CUDA call
    assert L.compressstore(1 << 12, 1 << 12, 1 << 12, 10, 3, 1 << 12, None) == cs._lib.ERR_INVALID_VALUE
    assert L.compressstore(1 << 12, 1 << 12, 1 << 12, 10, 4, None, None) == cs._lib.ERR_INVALID_VALUE
    assert L.compressstore(1 << 12, 1 << 12, 1 << 12, 1 << 41, 4, 1 << 12, None) == cs._lib.ERR_NOT_SUPPORTED
    # misaligned element pointer
    assert L.compressstore((1 << 12) + 2, 1 << 12, 1 << 12, 10, 4, 1 << 12, None) == cs._lib.ERR_MISALIGNED
    # null payload with n > 0
    assert L.compressstore(None, 1 << 12, 1 << 12, 10, 4, 1 << 12, None) == cs._lib.ERR_INVALID_VALUE
    # bad chunk lengths for the pass entry points
    assert L.cs_popc_chunks(1 << 12, 100, 48, 1 << 12, None) == cs._lib.ERR_INVALID_VALUE
    assert L.cs_popc_chunks(1 << 12, 100, 16, 1 << 12, None) == cs._lib.ERR_INVALID_VALUE
    assert L.cs_writeout(1 << 12, 1 << 12, 1 << 12, 100, 4, 1 << 12, None, 1024, 1, None) == cs._lib.ERR_INVALID_VALUE
    # bernoulli probability outside [0, 1]
    assert L.cs_gen_mask_bernoulli(1 << 12, 10, 1.5, 0, None) == cs._lib.ERR_INVALID_VALUE
    # pattern compaction: period outside 1..32, null count
    assert L.compressstore_pattern(1 << 12, 1 << 12, 100, 4, 1, 0, 1 << 12, None) == cs._lib.ERR_INVALID_VALUE
    assert L.compressstore_pattern(1 << 12, 1 << 12, 100, 4, 1, 33, 1 << 12, None) == cs._lib.ERR_INVALID_VALUE
    assert L.compressstore_pattern(1 << 12, 1 << 12, 100, 4, 1, 8, None, None) == cs._lib.ERR_INVALID_VALUE
    assert L.cs_gen_mask_pattern(1 << 12, 100, 1, 0, None) == cs._lib.ERR_INVALID_VALUE
    # serving: bad mode, null handles
    h = ctypes.c_void_p()
    cfg = cs._lib.CsServerConfig(0, 0, 0, 0, 7, 0, 0)
    assert L.cs_server_create(ctypes.byref(h), ctypes.byref(cfg)) == cs._lib.ERR_INVALID_VALUE
    assert L.cs_server_create(None, None) == cs._lib.ERR_INVALID_VALUE
    assert L.cs_server_submit(None, None, None) == cs._lib.ERR_INVALID_VALUE
    assert L.cs_server_release(None, 1) == cs._lib.ERR_INVALID_VALUE
    assert L.cs_server_destroy(None) == cs._lib.SUCCESS
    assert L.cs_status_string(1) == b"pending"


def test_server_create_needs_a_device():
    import torch
    import gpu_compressstore2_b200 as cs

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    h = ctypes.c_void_p()
    assert cs.lib().cs_server_create(ctypes.byref(h), None) == cs._lib.ERR_NO_DEVICE


def test_workspace_sizes():
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    c1024 = cs.make_config(cs.ALGO_3PASS, 1024)
    s1 = L.compressstore_workspace_size(1 << 28, 4, ctypes.byref(c1024))
    assert s1 > 0 and s1 % 256 == 0
    assert L.compressstore_workspace_size(1 << 28, 4, None) > 0  # AUTO: whatever the table picks
    # tiles*8 + chunks*(4+8) plus header, for 2^28 u32 with chunk length 1024
    tiles = (1 << 28) // (4 * 8192)  # one look-back status per 4-tile unit
    chunks = (1 << 28) // 1024
    assert s1 >= 256 + 8 * tiles + 12 * chunks
    blocks = (1 << 28) >> 18  # block prefixes of the reduce-then-scan pass
    items = (1 << 28) >> 14   # sparse-item flags of the hybrid writeout
    assert s1 < 256 + 8 * tiles + 12 * chunks + 8 * (chunks // 64 + 1) + 8 * blocks + 4 * items + 7 * 256 + 4 * 2048
    cfg = cs.make_config(cs.ALGO_3PASS, 32)
    assert L.compressstore_workspace_size(1 << 20, 4, ctypes.byref(cfg)) > s1 // 256
    bad = cs.make_config(cs.ALGO_3PASS, 100)
    assert L.compressstore_workspace_size(1 << 20, 4, ctypes.byref(bad)) == 0
    assert L.cs_scan_workspace_size(4096) == 512
    assert L.cs_scan_workspace_size(4097) == 512


def test_tuning_table_roundtrip():
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    algo = ctypes.c_int32()
    chunk = ctypes.c_uint32()
    b = L.cs_tune_size_bucket(1 << 20)
    assert b == 10
    assert L.cs_tune_set(4, b, cs.ALGO_3PASS, 2048) == 0
    assert L.cs_tune_get(4, 1 << 20, ctypes.byref(algo), ctypes.byref(chunk)) == 0
    assert (algo.value, chunk.value) == (cs.ALGO_3PASS, 2048)
    assert L.cs_tune_set(4, b, cs.ALGO_AUTO, 1024) == 0  # clear
    assert L.cs_tune_get(4, 1 << 20, ctypes.byref(algo), ctypes.byref(chunk)) == 0
    assert algo.value == cs.ALGO_3PASS
    assert L.cs_tune_set(4, 99, cs.ALGO_3PASS, 1024) == cs._lib.ERR_INVALID_VALUE
    assert L.cs_tune_set(4, 3, cs.ALGO_3PASS, 1000) == cs._lib.ERR_INVALID_VALUE


def test_tuning_table_files(tmp_path):
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    algo = ctypes.c_int32()
    chunk = ctypes.c_uint32()
    good = tmp_path / "t.txt"
    good.write_text("# comment\n\n8 12 1 1024  # trailing comment\n2 3 2 4096\n")
    assert L.cs_tune_load(str(good).encode()) == 0
    assert L.cs_tune_get(8, 1 << 24, ctypes.byref(algo), ctypes.byref(chunk)) == 0
    assert (algo.value, chunk.value) == (cs.ALGO_1PASS, 1024)
    assert L.cs_tune_get(2, 1 << 6, ctypes.byref(algo), ctypes.byref(chunk)) == 0
    assert (algo.value, chunk.value) == (cs.ALGO_3PASS, 4096)
    out = tmp_path / "saved.txt"
    assert L.cs_tune_save(str(out).encode()) == 0
    lines = [ln for ln in out.read_text().splitlines() if ln and not ln.startswith("#")]
    assert "8 12 1 1024" in lines and "2 3 2 4096" in lines
    # a bad line rejects the whole file and installs nothing
    bad = tmp_path / "bad.txt"
    bad.write_text("4 5 2 1024\n4 6 2 1000\n")
    assert L.cs_tune_load(str(bad).encode()) == cs._lib.ERR_INVALID_VALUE
    assert L.cs_tune_get(4, 1 << 10, ctypes.byref(algo), ctypes.byref(chunk)) == 0
    assert L.cs_tune_load(str(tmp_path / "missing.txt").encode()) == cs._lib.ERR_INVALID_VALUE
    for w, b in ((8, 12), (2, 3)):  # clear
        assert L.cs_tune_set(w, b, cs.ALGO_AUTO, 1024) == 0


def test_batch_table(tmp_path):
    """The batched form's (width, size, selectivity) table: buckets, set/get, and the
    "batch ..." lines of table files (validated with the plain entries, saved back)."""
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    ps = (0.0, 0.049, 0.05, 0.29, 0.3, 0.5, 0.7, 0.71, 0.95, 0.951, 1.0)
    assert [L.cs_tune_sel_bucket(p) for p in ps] == [0, 0, 1, 1, 2, 2, 2, 3, 3, 4, 4]
    algo = ctypes.c_int32()
    n = 1 << 28  # a bucket the packaged table leaves unset (3-pass)
    b = L.cs_tune_size_bucket(n)
    assert L.cs_tune_batch_get(4, n, 0.99, ctypes.byref(algo)) == 0 and algo.value == cs.ALGO_3PASS
    assert L.cs_tune_batch_set(4, b, 4, cs.ALGO_1PASS) == 0
    assert L.cs_tune_batch_get(4, n, 0.99, ctypes.byref(algo)) == 0 and algo.value == cs.ALGO_1PASS
    assert L.cs_tune_batch_get(4, n, 0.9, ctypes.byref(algo)) == 0 and algo.value == cs.ALGO_3PASS
    assert L.cs_tune_batch_get(4, n, 0.5, ctypes.byref(algo)) == 0 and algo.value == cs.ALGO_3PASS
    assert L.cs_tune_batch_set(4, b, 5, cs.ALGO_1PASS) == cs._lib.ERR_INVALID_VALUE
    assert L.cs_tune_batch_set(4, b, 1, cs.ALGO_NAIVE) == cs._lib.ERR_INVALID_VALUE
    out = tmp_path / "t.txt"
    assert L.cs_tune_save(str(out).encode()) == 0
    assert f"batch 4 {b} 4 1" in out.read_text().splitlines()
    assert L.cs_tune_batch_set(4, b, 4, cs.ALGO_AUTO) == 0  # clear
    assert L.cs_tune_batch_get(4, n, 0.99, ctypes.byref(algo)) == 0 and algo.value == cs.ALGO_3PASS
    f = tmp_path / "b.txt"
    f.write_text("8 3 2 4096\nbatch 8 3 0 1  # sparse columns of this size take the 1-pass form\n")
    assert L.cs_tune_load(str(f).encode()) == 0
    assert L.cs_tune_batch_get(8, 1 << 6, 0.01, ctypes.byref(algo)) == 0 and algo.value == cs.ALGO_1PASS
    # the packaged B200 table holds batch entries: 1-pass for u32 columns of 2^21 at p = 0.5
    assert L.cs_tune_batch_get(4, 1 << 21, 0.5, ctypes.byref(algo)) == 0 and algo.value == cs.ALGO_1PASS
    for bad in ("batch 8 3 5 1\n", "batch 8 3 0 3\n", "batch 8 3 0\n", "nonsense\n"):
        f.write_text(bad)
        assert L.cs_tune_load(str(f).encode()) == cs._lib.ERR_INVALID_VALUE, bad
    assert L.cs_tune_batch_set(8, 3, 0, cs.ALGO_AUTO) == 0
    assert L.cs_tune_set(8, 3, cs.ALGO_AUTO, 1024) == 0


def test_selectivity_table(tmp_path):
    """The plain call's entries for a stated selectivity: set/get, fallback to the (width,
    size) entry where a bucket has none, the "sel ..." lines of table files, and the
    cs_config field that carries the caller's fraction."""
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    algo, chunk = ctypes.c_int32(), ctypes.c_uint32()
    n = 1 << 36  # a size bucket the packaged table leaves unset
    b = L.cs_tune_size_bucket(n)
    assert L.cs_tune_set(4, b, cs.ALGO_3PASS, 4096) == 0
    try:
        for p in (0.0, 0.01, 0.5, 0.99):  # no selectivity entries yet: the (width, size) entry
            assert L.cs_tune_sel_get(4, n, p, ctypes.byref(algo), ctypes.byref(chunk)) == 0
            assert (algo.value, chunk.value) == (cs.ALGO_3PASS, 4096)
        assert L.cs_tune_sel_set(4, b, 4, cs.ALGO_1PASS, 1024) == 0
        assert L.cs_tune_sel_get(4, n, 0.99, ctypes.byref(algo), ctypes.byref(chunk)) == 0
        assert (algo.value, chunk.value) == (cs.ALGO_1PASS, 1024)
        for p in (0.0, 0.5, 0.9):  # unknown, or another bucket: unchanged
            assert L.cs_tune_sel_get(4, n, p, ctypes.byref(algo), ctypes.byref(chunk)) == 0
            assert (algo.value, chunk.value) == (cs.ALGO_3PASS, 4096)
        assert L.cs_tune_get(4, n, ctypes.byref(algo), ctypes.byref(chunk)) == 0 and algo.value == cs.ALGO_3PASS
        for bad in ((4, b, 5, cs.ALGO_1PASS, 1024), (4, b, 0, cs.ALGO_3PASS, 1000), (3, b, 0, cs.ALGO_3PASS, 1024),
                    (4, 21, 0, cs.ALGO_3PASS, 1024)):
            assert L.cs_tune_sel_set(*bad) == cs._lib.ERR_INVALID_VALUE, bad
        for bad_p in (-0.1, 1.5, float("nan")):
            assert L.cs_tune_sel_get(4, n, bad_p, ctypes.byref(algo), ctypes.byref(chunk)) == cs._lib.ERR_INVALID_VALUE
        out = tmp_path / "t.txt"
        assert L.cs_tune_save(str(out).encode()) == 0
        assert f"sel 4 {b} 4 1 1024" in out.read_text().splitlines()
        assert L.cs_tune_sel_set(4, b, 4, cs.ALGO_AUTO, 0) == 0  # clear
        f = tmp_path / "s.txt"
        f.write_text(f"sel 4 {b} 0 2 2048  # sparse columns of this size: 3-pass at L = 2048\n")
        assert L.cs_tune_load(str(f).encode()) == 0
        assert L.cs_tune_sel_get(4, n, 0.01, ctypes.byref(algo), ctypes.byref(chunk)) == 0
        assert (algo.value, chunk.value) == (cs.ALGO_3PASS, 2048)
        for bad in ("sel 4 3 0 2\n", "sel 4 3 5 2 1024\n", "sel 4 3 0 2 1000\n", "sel 4 3 0 2 1024 9\n"):
            f.write_text(bad)
            assert L.cs_tune_load(str(f).encode()) == cs._lib.ERR_INVALID_VALUE, bad
        # the config field sits after timeout_ns, as in include/compressstore.h
        assert cs.CsConfig.selectivity.offset == 24 and ctypes.sizeof(cs.CsConfig) == 32
        assert cs.make_config(selectivity=0.25).selectivity == 0.25
    finally:
        for sb in range(5):
            L.cs_tune_sel_set(4, b, sb, cs.ALGO_AUTO, 0)
        L.cs_tune_set(4, b, cs.ALGO_AUTO, 1024)


@pytest.mark.parametrize("w", [1, 2, 4, 8])
def test_shared_memory_budget(w):
    """The TMA kernel's own shared-memory layout (Layout<...>::TOTAL, read from the library)
    fits the 227 KB a CTA may opt into, with room for its static variables and the 1 KB
    the hardware reserves per CTA."""
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    for algo in (cs.ALGO_1PASS, cs.ALGO_3PASS):
        b = L.cs_compact_smem_bytes(w, algo)
        assert b > 4 * 32768, (w, algo, b)  # at least the payload ring
        assert b + 1024 + 64 <= 227 * 1024, (w, algo, b)
    assert L.cs_compact_smem_bytes(3, cs.ALGO_1PASS) == 0
    assert L.cs_compact_smem_bytes(4, cs.ALGO_NAIVE) == 0


def _header_define(name: str) -> int:
    text = (ROOT / "include" / "compressstore.h").read_text()
    m = re.search(rf"#define {name} \((\d+)(u|ull) << (\d+)\)", text)
    assert m, name
    return int(m.group(1)) << int(m.group(3))


@pytest.mark.parametrize("w", [1, 2, 4, 8])
def test_noalloc_scratch_bound(w):
    """compressstore_noalloc runs with its chunk length fixed at 4096: the workspace that
    needs, at the largest n it accepts, fits the fixed scratch array for every width."""
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    max_n = _header_define("CS_NOALLOC_MAX_N")
    scratch = _header_define("CS_NOALLOC_SCRATCH_BYTES")
    assert (max_n, scratch) == (1 << 30, 4 << 20)
    cfg = cs.make_config(cs.ALGO_AUTO, 4096)
    need = L.compressstore_workspace_size(max_n, w, ctypes.byref(cfg))
    assert 0 < need <= scratch, (w, need)
    # the bound is not loose by chance: the default chunk length would not fit
    assert L.compressstore_workspace_size(max_n, w, ctypes.byref(cs.make_config(cs.ALGO_3PASS, 1024))) > scratch
    # argument errors come before any device work
    assert L.compressstore_noalloc(1 << 12, 1 << 12, 1 << 12, max_n + 1, w, 1 << 12, None) == cs._lib.ERR_NOT_SUPPORTED
    assert L.compressstore_noalloc(1 << 12, 1 << 12, 1 << 12, 100, 3, 1 << 12, None) == cs._lib.ERR_INVALID_VALUE

"""CPU tests: pin the oracle restatement against the reference's own CPU code and the
committed golden vectors (the reference's known answers included)."""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _golden():
    meta = json.loads((GOLDEN / "golden.json").read_text())
    arrays = np.load(GOLDEN / "golden_small.npz")
    return meta, arrays


def test_kat_reference_uniform_mask_seed42(oracle):
    # generate_mask_uniform(buf, 0, 8, 0.5) with seed 42 (src/data_generator.cuh:14-31)
    b, ones = oracle.ref_mask_uniform_msb(8, 0.5, 42)
    assert b.tobytes().hex() == "09f7bb9f36fcb434"
    assert ones == 38
    meta, _ = _golden()
    kat = meta["kat"]["ref_mask_uniform_seed42_p50_64B"]
    b64, ones64 = oracle.ref_mask_uniform_msb(64, 0.5, 42)
    assert b64.tobytes().hex() == kat["bytes"] and ones64 == kat["ones"]


def test_kat_sixteen_elements(oracle):
    # mask bytes {0x81, 0x40} (MSB-first) over data[i] = 100 + i selects {100, 107, 109}
    msb = np.array([0x81, 0x40, 0, 0], dtype=np.uint8)
    words = oracle.rev8(msb).view(np.uint32)
    data = (100 + np.arange(16)).astype(np.uint32)
    out = oracle.compact(data, words, 16)
    assert out.tolist() == [100, 107, 109]


def test_rev8_roundtrip(oracle):
    rng = np.random.default_rng(0)
    b = rng.integers(0, 256, 4096, dtype=np.uint8)
    assert np.array_equal(oracle.rev8(oracle.rev8(b)), b)
    assert oracle.rev8(np.array([1], np.uint8))[0] == 0x80


@pytest.mark.parametrize("case", range(13))
def test_golden_small(oracle, case):
    meta, arrays = _golden()
    rec = meta["small"][case]
    name, n, w = rec["name"], rec["n"], rec["elem_bytes"]
    payload = arrays[f"{name}__payload"]
    mask = arrays[f"{name}__mask"]
    out = oracle.compact(payload, mask, n)
    assert len(out) == rec["count"]
    assert np.array_equal(out, arrays[f"{name}__out"])
    assert hashlib.sha256(out.tobytes()).hexdigest() == rec["sha256"]


def _regen(oracle, rec):
    n, w, kind, param = rec["n"], rec["elem_bytes"], rec["kind"], rec["param"]
    payload = oracle.payload(n, w, rec["payload_seed"], float_unit=(kind == "bernoulli_f32"))
    if kind in ("bernoulli", "bernoulli_f32"):
        mask = oracle.mask_bernoulli(n, param, rec["mask_seed"])
    elif kind == "runs":
        mask = oracle.mask_runs(n, param, rec["mask_seed"])
    else:
        mask = oracle.mask_dense_prefix(n, param)
    return payload, mask


@pytest.mark.parametrize("case", range(4))
def test_golden_large(oracle, case):
    meta, _ = _golden()
    rec = meta["large"][case]
    payload, mask = _regen(oracle, rec)
    out = oracle.compact(payload, mask, rec["n"])
    assert len(out) == rec["count"]
    assert hashlib.sha256(out.tobytes()).hexdigest() == rec["sha256"]
    out_mt = oracle.compact(payload, mask, rec["n"], threads=4)
    assert np.array_equal(out, out_mt)


def test_golden_regenerated_inputs_match(oracle):
    # the stored small-case inputs are exactly what the seeded generators produce
    meta, arrays = _golden()
    for rec in meta["small"]:
        if rec["kind"] == "explicit":
            continue
        payload, mask = _regen(oracle, rec)
        assert np.array_equal(payload, arrays[rec["name"] + "__payload"])
        assert np.array_equal(mask, arrays[rec["name"] + "__mask"])


@pytest.mark.parametrize("w", [1, 2, 4, 8])
@pytest.mark.parametrize("p", [0.0, 0.01, 0.5, 0.97, 1.0])
def test_oracle_vs_reference_cpu(oracle, reference, w, p):
    n = 8 * 1237
    payload = oracle.payload(n, w, 7 + w)
    mask = oracle.mask_bernoulli(n, p, 99)
    msb = oracle.rev8(mask.view(np.uint8))[: n // 8]
    ref = reference.generate_validation(payload, msb, n)
    ours = oracle.compact(payload, mask, n)
    assert np.array_equal(ref, ours)


def test_reference_uniform_and_clustering_match_restatement(oracle, reference):
    b, ones = reference.generate_mask_uniform(256, 0.3)
    b2, ones2 = oracle.ref_mask_uniform_msb(256, 0.3, 42)
    assert np.array_equal(b, b2) and ones == ones2
    for n in (1024, 4096, 8 * 999):
        c, cones = reference.generate_mask_clustering(0.1, 1, n)
        words = oracle.mask_dense_prefix(n, 0.1)
        lsb = oracle.rev8(c)
        assert np.array_equal(lsb, words.view(np.uint8)[: n // 8])
        assert cones == oracle.count(words, n)


def test_partial_tail_is_honoured(oracle):
    # n not a multiple of 8: the reference drops the partial last byte, the oracle keeps it
    n = 13
    data = np.arange(n, dtype=np.uint16)
    mask = np.array([0xFFFFFFFF], dtype=np.uint32)
    out = oracle.compact(data, mask, n)
    assert out.tolist() == list(range(13))  # bits >= n ignored


def test_popc_and_scan(oracle):
    n = 100_003
    mask = oracle.mask_bernoulli(n, 0.3, 5)
    for L in (32, 64, 1024, 65536):
        counts = oracle.popc_chunks(mask, n, L)
        assert counts.sum() == oracle.count(mask, n)
        offs, total = oracle.exclusive_scan(counts)
        assert total == counts.sum()
        assert offs[0] == 0 and np.array_equal(np.diff(offs), counts[:-1])


def test_runs_generator_statistics(oracle):
    n = 1 << 20
    for mean in (8.0, 64.0):
        words = oracle.mask_runs(n, mean, 3)
        bits = np.unpackbits(words.view(np.uint8), bitorder="little")[:n]
        p = bits.mean()
        assert 0.45 < p < 0.55
        changes = np.count_nonzero(np.diff(bits.astype(np.int8)))
        mean_run = n / (changes + 1)
        assert 0.9 * mean < mean_run < 1.1 * mean


def test_bernoulli_generator_statistics(oracle):
    n = 1 << 18
    for p in (0.001, 0.1, 0.5, 0.9):
        c = oracle.count(oracle.mask_bernoulli(n, p, 1), n)
        assert abs(c / n - p) < 4 * np.sqrt(p * (1 - p) / n) + 1e-4


def test_mix64_known_value(oracle):
    # SplitMix64 with state 0 -> first output 0xe220a8397b1dcdaf (published test value)
    assert oracle.mix64(0, 0) == 0xE220A8397B1DCDAF


def rev32(x: int) -> int:
    return int(f"{x:032b}"[::-1], 2)


@pytest.mark.parametrize("length", [1, 2, 3, 7, 8, 13, 31, 32])
def test_pattern_mask_matches_reference(oracle, reference, length):
    """The LSB-first periodic mask equals the reference's generate_mask_pattern (pattern read
    from the MSB) fed the bit-reversed pattern."""
    top = ((1 << length) - 1) << (32 - length)
    for msb in (0x80000000, 0xA5A5A5A5, 0xFFFFFFFF, 0x12345678, 0x00000000):
        p = msb & top
        n = 8 * 131
        ref_bytes, ref_ones = reference.generate_mask_pattern(n // 8, p, length)
        words = oracle.mask_pattern(n, rev32(p), length)
        assert np.array_equal(oracle.rev8(words.view(np.uint8))[: n // 8], ref_bytes), (length, hex(p))
        assert oracle.count(words, n) == ref_ones


def test_pattern_count_formula(oracle):
    import gpu_compressstore2_b200 as cs

    rng = np.random.default_rng(5)
    for _ in range(200):
        length = int(rng.integers(1, 33))
        pattern = int(rng.integers(0, 2**32))
        n = int(rng.integers(0, 5000))
        assert cs.pattern_count(n, pattern, length) == oracle.count(oracle.mask_pattern(n, pattern, length), n)

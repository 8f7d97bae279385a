"""GPU parity at the configurations' stated sizes, against digests of the reference's own
CPU compaction (generate_validation, src/data_generator.cuh:171-188) computed from the same
seeded inputs by tests/golden/make_golden.py --sized.

* n = 2^28 float32 uniform in [0, 1), iid masks p in {0.001, 0.01, 0.1, 0.5, 0.9, 0.99}:
  AUTO, 1-pass, 3-pass and the CUB Flagged comparator.
* n = 2^29 at widths 1, 2, 4 and 8 on alternating-runs masks (mean run 8, 64, 4096) and the
  single dense block of the first 10%: AUTO, 1-pass and 3-pass. The 8-byte column is 4 GiB,
  so its output byte offsets pass 2^31 and 2^32.

Inputs are generated on the device (the device generators reproduce the oracle's bit for
bit; each record also pins the digest of its mask words). The first algorithm's output is
hashed and compared with the reference digest; every other algorithm must produce the same
count and the same bytes, compared on the device, and must leave the bytes past the count
untouched. Needs a B200 with about 13 GB free.
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import pytest

SIZED = json.loads((Path(__file__).resolve().parent / "golden" / "golden_sized.json").read_text())["sized"]
GUARD = 4096  # elements past the count that must keep their fill
FILL = 0x5A


def _algos():
    import gpu_compressstore2_b200 as cs

    return [("auto", cs.ALGO_AUTO), ("1pass", cs.ALGO_1PASS), ("3pass", cs.ALGO_3PASS)]


def _sha(t) -> str:
    return hashlib.sha256(t.cpu().numpy().tobytes()).hexdigest()


def _gen_mask(cs, d_mask, rec):
    n, kind, par = rec["n"], rec["kind"], rec["param"]
    if kind.startswith("bernoulli"):
        cs.gen_mask_bernoulli(d_mask, n, par, rec["mask_seed"])
    elif kind == "runs":
        cs.gen_mask_runs(d_mask, n, par, rec["mask_seed"])
    elif kind == "dense":
        cs.gen_mask_dense_prefix(d_mask, n, par)
    else:
        raise ValueError(kind)


def _run_sweep(records, extra=None):
    """All records share n and width: one payload, one mask buffer, two output buffers."""
    import torch
    import gpu_compressstore2_b200 as cs

    n, w = records[0]["n"], records[0]["elem_bytes"]
    dt = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[w]
    d_in = torch.empty(n, dtype=dt, device="cuda")
    cs.gen_payload(d_in, n, records[0]["payload_seed"], float_unit=records[0]["kind"] == "bernoulli_f32")
    d_mask = torch.empty((n + 31) // 32, dtype=torch.int32, device="cuda")
    first = torch.empty(n, dtype=dt, device="cuda")
    other = torch.empty(n, dtype=dt, device="cuda")
    d_count = torch.zeros(1, dtype=torch.int64, device="cuda")
    runs = _algos() + (extra or [])
    try:
        for rec in records:
            _gen_mask(cs, d_mask, rec)
            torch.cuda.synchronize()
            assert _sha(d_mask) == rec["mask_sha256"], rec["name"]
            k = rec["count"]
            for i, (name, algo) in enumerate(runs):
                dst = first if i == 0 else other
                dst.view(torch.uint8).fill_(FILL)
                d_count.fill_(-3)
                if callable(algo):
                    algo(d_in, d_mask, dst, n, d_count)
                else:
                    cs.compressstore(d_in, d_mask, dst, n, d_count, algo=algo)
                torch.cuda.synchronize()
                assert int(d_count.item()) == k, (rec["name"], name, int(d_count.item()), k)
                if i == 0:
                    assert _sha(first[:k]) == rec["sha256"], (rec["name"], name)
                else:
                    assert torch.equal(other[:k], first[:k]), (rec["name"], name)
                tail = dst[k:k + GUARD].view(torch.uint8)
                assert bool((tail == FILL).all()), f"{rec['name']} {name}: wrote past the count"
        cs.compressstore_check()
    finally:
        del d_in, d_mask, first, other
        torch.cuda.empty_cache()


@pytest.mark.gpu
def test_config2_selectivity_sweep_2p28_f32(cuda):
    import gpu_compressstore2_b200 as cs

    recs = [r for r in SIZED if r["name"].startswith("cfg2_")]
    assert [r["param"] for r in recs] == [0.001, 0.01, 0.1, 0.5, 0.9, 0.99]
    flagged = cs.CubFlagged(recs[0]["n"], 4)
    _run_sweep(recs, extra=[("cub_flagged", flagged)])


@pytest.mark.gpu
@pytest.mark.parametrize("w", [1, 2, 4, 8])
def test_config3_width_and_mask_structure_2p29(cuda, w):
    recs = [r for r in SIZED if r["name"].startswith("cfg3_") and r["elem_bytes"] == w]
    assert len(recs) == 4
    _run_sweep(recs)


def test_sized_records_cover_the_configurations():
    """CPU check of the fixture itself: every stated selectivity, width and mask structure."""
    c2 = [r for r in SIZED if r["name"].startswith("cfg2_")]
    c3 = [r for r in SIZED if r["name"].startswith("cfg3_")]
    assert {r["param"] for r in c2} == {0.001, 0.01, 0.1, 0.5, 0.9, 0.99}
    assert all(r["n"] == 1 << 28 and r["elem_bytes"] == 4 for r in c2)
    assert {(r["elem_bytes"], r["kind"], r["param"]) for r in c3} == {
        (w, k, p) for w in (1, 2, 4, 8) for k, p in (("runs", 8.0), ("runs", 64.0), ("runs", 4096.0), ("dense", 0.1))}
    assert all(r["n"] == 1 << 29 for r in c3)
    for r in SIZED:  # selectivities land where the configurations say
        frac = r["count"] / r["n"]
        if r["kind"] == "dense":
            assert frac == pytest.approx(0.1, abs=1e-6)
        elif r["kind"] == "runs":
            assert frac == pytest.approx(0.5, abs=0.02)
        else:
            assert frac == pytest.approx(r["param"], rel=0.02)

"""Generate the golden fixtures in this directory from the reference's OWN CPU code.

Inputs come from the seeded counter-based generators (oracle restatement, reproduced bit
for bit by the device generators). Outputs come from the reference's generate_validation
(src/data_generator.cuh:171-188), compiled from its sources into oracle/_ref/libcsref.so
by oracle/Makefile, fed the per-byte bit-reversed (MSB-first) copy of each mask.

Run in a container that has the reference tree:  python tests/golden/make_golden.py
The digests at the configurations' full sizes (golden_sized.json; about 10 GiB of host
memory and a few minutes):                           python tests/golden/make_golden.py --sized
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import Oracle, Reference, build  # noqa: E402

DT = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}

# (name, n, elem_bytes, mask kind, mask param, payload seed, mask seed); n a multiple of 8
# because the reference ignores a partial last mask byte.
SMALL_CASES = [
    ("kat16_u32", 16, 4, "explicit", None, 0, 0),
    ("u8_p50_n8", 8, 1, "bernoulli", 0.5, 11, 12),
    ("u8_p10_n4096", 4096, 1, "bernoulli", 0.1, 13, 14),
    ("u16_p50_n1000", 1000, 2, "bernoulli", 0.5, 15, 16),
    ("u16_p99_n4096", 4096, 2, "bernoulli", 0.99, 17, 18),
    ("u32_p01_n4096", 4096, 4, "bernoulli", 0.01, 19, 20),
    ("u32_p50_n2040", 2040, 4, "bernoulli", 0.5, 21, 22),
    ("u32_runs8_n4096", 4096, 4, "runs", 8.0, 23, 24),
    ("u64_p50_n4096", 4096, 8, "bernoulli", 0.5, 25, 26),
    ("u64_runs64_n4096", 4096, 8, "runs", 64.0, 27, 28),
    ("u32_all0_n256", 256, 4, "bernoulli", 0.0, 29, 30),
    ("u32_all1_n256", 256, 4, "bernoulli", 1.0, 31, 32),
    ("u32_dense10_n4096", 4096, 4, "dense", 0.1, 33, 0),
]

# Large cases: only seeds, count and a digest of the reference output are stored.
LARGE_CASES = [
    # configuration 1: n=2^20 uint32, iid Bernoulli(0.5), chunk length 1024
    ("config1_u32_p50_n1M", 1 << 20, 4, "bernoulli", 0.5, 1001, 1002),
    ("f32_p001_n1M", 1 << 20, 4, "bernoulli_f32", 0.001, 1003, 1004),
    ("u8_runs4096_n1M", 1 << 20, 1, "runs", 4096.0, 1005, 1006),
    ("u64_p90_n256K", 1 << 18, 8, "bernoulli", 0.9, 1007, 1008),
]


def make_inputs(o: Oracle, n, w, kind, param, pseed, mseed, payload=None):
    if kind == "explicit":
        payload = (100 + np.arange(n)).astype(DT[w])
        msb = np.array([0x81, 0x40], dtype=np.uint8)
        words = o.rev8(msb)
        words = np.concatenate([words, np.zeros(4 - len(words) % 4, np.uint8)]).view(np.uint32)
        return payload, words
    if payload is None:
        payload = o.payload(n, w, pseed, float_unit=(kind == "bernoulli_f32"))
    if kind in ("bernoulli", "bernoulli_f32"):
        words = o.mask_bernoulli(n, param, mseed)
    elif kind == "runs":
        words = o.mask_runs(n, param, mseed)
    elif kind == "dense":
        words = o.mask_dense_prefix(n, param)
    else:
        raise ValueError(kind)
    return payload, words


# Cases at the configurations' stated sizes (golden_sized.json): the selectivity sweep of
# 2^28 float32 (uniform in [0, 1)) with iid masks, and the width x mask-structure sweep of 2^29
# elements (alternating runs of geometric mean length 8 / 64 / 4096, and the single dense block
# of the first 10%). Only seeds, the count and digests are stored: the inputs are regenerated
# on the device by the seeded generators (the device generators reproduce the oracle's bit for
# bit), so each record also keeps the digest of its mask words.
SIZED_F32_P = [0.001, 0.01, 0.1, 0.5, 0.9, 0.99]
SIZED_MASKS = [("runs", 8.0), ("runs", 64.0), ("runs", 4096.0), ("dense", 0.1)]


def sized_cases():
    cases = []
    for i, p in enumerate(SIZED_F32_P):
        cases.append((f"cfg2_f32_p{p:g}_n2^28", 1 << 28, 4, "bernoulli_f32", p, 2001, 2100 + i))
    for w in (1, 2, 4, 8):
        for j, (kind, param) in enumerate(SIZED_MASKS):
            tag = f"runs{int(param)}" if kind == "runs" else "dense10"
            cases.append((f"cfg3_u{8 * w}_{tag}_n2^29", 1 << 29, w, kind, param, 3000 + w, 3100 + j))
    return cases


def make_sized(o: Oracle, ref: Reference) -> None:
    recs = []
    payloads: dict[tuple, np.ndarray] = {}
    for name, n, w, kind, param, pseed, mseed in sized_cases():
        key = (n, w, pseed, kind == "bernoulli_f32")
        if key not in payloads:
            payloads.clear()  # one payload at a time (up to 4 GiB)
            payloads[key] = o.payload(n, w, pseed, float_unit=key[3])
        payload = payloads[key]
        _, words = make_inputs(o, n, w, kind, param, pseed, mseed, payload=payload)
        msb = o.rev8(words.view(np.uint8))[: n // 8]
        out = ref.generate_validation(payload, msb, n)
        recs.append(dict(name=name, n=n, elem_bytes=w, kind=kind, param=param, payload_seed=pseed, mask_seed=mseed,
                         count=int(len(out)), sha256=hashlib.sha256(out.tobytes()).hexdigest(),
                         mask_sha256=hashlib.sha256(words.tobytes()).hexdigest()))
        print(name, recs[-1]["count"], flush=True)
        del out, msb, words
    (HERE / "golden_sized.json").write_text(json.dumps({"sized": recs}, indent=1, sort_keys=True) + "\n")
    print(f"wrote {len(recs)} sized cases")


def main() -> None:
    build()
    o = Oracle.instance()
    ref = Reference()
    if "--sized" in sys.argv:
        make_sized(o, ref)
        return
    arrays = {}
    meta = {"small": [], "large": [], "kat": {}}
    for name, n, w, kind, param, pseed, mseed in SMALL_CASES + LARGE_CASES:
        payload, words = make_inputs(o, n, w, kind, param, pseed, mseed)
        msb = o.rev8(words.view(np.uint8))[: n // 8]
        out = ref.generate_validation(payload, msb, n)
        rec = dict(name=name, n=n, elem_bytes=w, kind=kind, param=param, payload_seed=pseed, mask_seed=mseed,
                   count=int(len(out)), sha256=hashlib.sha256(out.tobytes()).hexdigest())
        if (name, n, w, kind, param, pseed, mseed) in SMALL_CASES:
            arrays[f"{name}__payload"] = payload
            arrays[f"{name}__mask"] = words
            arrays[f"{name}__out"] = out
            meta["small"].append(rec)
        else:
            meta["large"].append(rec)
    u, ones = ref.generate_mask_uniform(64, 0.5)
    meta["kat"]["ref_mask_uniform_seed42_p50_64B"] = {"bytes": u.tobytes().hex(), "ones": ones}
    c, cones = ref.generate_mask_clustering(0.1, 1, 4096)
    meta["kat"]["ref_mask_clustering_p10_c1_n4096"] = {"bytes_sha256": hashlib.sha256(c.tobytes()).hexdigest(),
                                                       "ones": cones}
    np.savez_compressed(HERE / "golden_small.npz", **arrays)
    (HERE / "golden.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    print(f"wrote {len(meta['small'])} small and {len(meta['large'])} large cases")


if __name__ == "__main__":
    main()

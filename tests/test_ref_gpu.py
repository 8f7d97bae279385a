"""The reference's own GPU compositions (bench10, bench7, bench8), run by the comparator
baseline/_ref/ref_gpu_bench (built from the reference's sources by baseline/Makefile), give
the oracle's output on the library's seeded inputs. This pins the comparator the bench
times: its outputs are the reference CPU compaction's, so the GB/s it reports are for the
same work. Skipped where the comparator was not built (no reference sources)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "baseline" / "_ref" / "ref_gpu_bench"


@pytest.mark.gpu
@pytest.mark.parametrize("w,p", [(4, 0.5), (8, 0.02)])
def test_reference_gpu_compositions_match_the_oracle(cuda, oracle, tmp_path, w, p):
    import json

    if not BIN.exists():
        pytest.skip("baseline/_ref/ref_gpu_bench not built")
    n, pseed, mseed = 1 << 20, 71, 72
    dump = tmp_path / "out"
    r = subprocess.run([str(BIN), str(n), str(w), str(p), str(pseed), str(mseed), "2", "1024,4096", "256", "1024",
                        "bench10,bench7,bench8", str(dump)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert {x["bench"] for x in d["results"]} == {"bench10", "bench7", "bench8"}
    assert all(x["ok"] for x in d["results"]), d["results"]  # every swept point == the library's output
    payload = oracle.payload(n, w, pseed, float_unit=(w == 4))
    mask = oracle.mask_bernoulli(n, p, mseed)
    exp = oracle.compact(payload, mask, n)
    assert d["count"] == len(exp)
    for bench in ("bench10", "bench7", "bench8"):
        got = np.fromfile(f"{dump}_{bench}.bin", dtype=exp.dtype)
        assert np.array_equal(got, exp), bench

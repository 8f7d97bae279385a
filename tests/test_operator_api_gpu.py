"""GPU tests of the Python mirror of the reference's operator API: IntermediateData (the
counterpart of intermediate_data, src/benchmarks.cuh:53-151) and the bench_* compositions
(the counterparts of bench7/bench10, src/benchmarks.cuh:360-440), with their per-phase
Timings (src/benchmarks.cuh:10-47): outputs against the oracle, phases filled as the
reference fills them, and the scratch reused across calls of different sizes."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import dev_empty, from_dev, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w", [1, 4, 8])
def test_compositions_against_the_oracle(cuda, oracle, w):
    import torch
    import gpu_compressstore2_b200 as cs

    nmax = 700_001
    ident = cs.IntermediateData(nmax, 256, w)
    for n, p, L in ((nmax, 0.5, 1024), (123_457, 0.03, 256), (40_000, 0.97, 4096)):
        payload = oracle.payload(n, w, 10 + n)
        mask = oracle.mask_bernoulli(n, p, 20 + n)
        exp = oracle.compact(payload, mask, n)
        d_in, d_mask = to_dev(payload), to_dev(mask)
        for fn in (cs.bench_1pass, cs.bench_auto, cs.bench_3pass, cs.bench_naive):
            d_out = dev_empty(n, w, fill=0)
            t = fn(ident, d_in, d_mask, d_out, n, L)
            torch.cuda.synchronize()
            k = int(ident.d_count.item())
            assert k == len(exp), (fn.__name__, n)
            assert np.array_equal(from_dev(d_out, w)[:k], exp), (fn.__name__, n)
            assert t.total > 0
            if fn in (cs.bench_3pass, cs.bench_naive):  # three timed phases, like bench7/bench10
                assert min(t.popc, t.pss1, t.proc) >= 0 and t.pss2 == -1
                assert t.total >= max(t.popc, t.pss1, t.proc)
            elif fn is cs.bench_1pass:
                assert t.popc == -1 and t.pss1 == -1 and t.proc == t.total
            else:
                assert t.popc == -1 and t.proc == -1


def test_sizes_beyond_the_intermediate_data_are_rejected(cuda):
    import gpu_compressstore2_b200 as cs

    ident = cs.IntermediateData(1000, 1024, 4)
    d = dev_empty(2048, 4, fill=0)
    with pytest.raises(cs.CsError):
        cs.bench_3pass(ident, d, d, d, 2000, 1024)
    with pytest.raises(cs.CsError):
        cs.bench_3pass(ident, d, d, d, 500, 512)  # chunk shorter than the one it was sized for

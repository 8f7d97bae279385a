"""GPU tests of the batched form (cs_batch_*): many uneven columns of mixed width in one
plan, direct and graph-replayed, against the CPU oracle and against the plain call."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import dev_empty, from_dev, to_dev

pytestmark = pytest.mark.gpu

GUARD = 32


def _columns(oracle, specs):
    import torch

    cols, host = [], []
    counts = torch.full((len(specs),), -5, dtype=torch.int64, device="cuda")
    for i, (n, w, kind, par) in enumerate(specs):
        payload = oracle.payload(n, w, 500 + i)
        if kind == "b":
            mask = oracle.mask_bernoulli(n, par, 900 + i)
        else:
            mask = oracle.mask_runs(n, par, 900 + i)
        d_in = to_dev(payload) if n else dev_empty(4, w)
        d_mask = to_dev(mask) if n else dev_empty(4, 4)
        d_out = dev_empty(n + GUARD, w, fill=0xAB)
        cols.append((d_in, d_mask, d_out, n, counts[i:i + 1]))
        host.append((payload, mask, n, w))
    return cols, host, counts


def _check(oracle, cols, host, counts):
    import torch

    torch.cuda.synchronize()
    got = counts.cpu().numpy()
    for (d_in, d_mask, d_out, n, _), (payload, mask, _, w), k in zip(cols, host, got):
        exp = oracle.compact(payload, mask, n) if n else payload[:0]
        assert k == len(exp), (n, w, k, len(exp))
        out = from_dev(d_out, w)
        assert np.array_equal(out[:k], exp), (n, w)
        assert np.all(out[k:].view(np.uint8) == 0xAB), (n, w)


SPECS = [
    (0, 4, "b", 0.5), (1, 1, "b", 1.0), (31, 2, "b", 0.5), (33, 8, "b", 0.7), (1000, 4, "b", 0.01),
    (4096, 1, "b", 0.5), (8193, 8, "b", 0.99), (32769, 4, "b", 0.001), (131072, 1, "r", 8.0),
    (131073, 2, "b", 0.02), (200_000, 4, "b", 0.5), (262_144, 8, "r", 4096.0), (300_001, 4, "b", 0.0),
    (500_000, 1, "b", 0.3), (524_288, 2, "b", 0.03), (1_048_577, 4, "b", 0.5), (777_777, 8, "b", 0.02),
    (2_000_000, 4, "r", 64.0), (5, 4, "b", 0.5), (65_536, 8, "b", 1.0),
]


def test_batch_direct_and_graph(cuda, oracle):
    import torch
    import gpu_compressstore2_b200 as cs

    cols, host, counts = _columns(oracle, SPECS)
    b = cs.Batch(cols)
    b.run()
    _check(oracle, cols, host, counts)
    for (_, _, d_out, _, _) in cols:  # reset outputs; runs must rewrite them identically
        d_out.view(torch.uint8).fill_(0xAB)
    counts.fill_(-5)
    b.run()
    b.check()
    _check(oracle, cols, host, counts)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b.capture_graph(stream=s)
        for _ in range(2):
            for (_, _, d_out, _, _) in cols:
                d_out.view(torch.uint8).fill_(0xAB)
            counts.fill_(-5)
            b.run(stream=s)
            b.check(stream=s)
            _check(oracle, cols, host, counts)
    assert b.launches_per_run == 1
    b.close()


def test_batch_matches_plain_calls(cuda):
    """A config-4-shaped batch (uneven lengths log-uniform, widths 4 and 8, p uniform in
    [0.01, 0.99]): every column equals the plain call's output."""
    import torch
    import gpu_compressstore2_b200 as cs

    rng = np.random.default_rng(4)
    ncols = 96
    lens = np.exp(rng.uniform(np.log(2 ** 10), np.log(2 ** 21), ncols)).astype(np.int64)
    widths = rng.choice([4, 8], ncols)
    ps = rng.uniform(0.01, 0.99, ncols)
    cols = []
    counts = torch.zeros(ncols, dtype=torch.int64, device="cuda")
    for i in range(ncols):
        n, w = int(lens[i]), int(widths[i])
        d_in = dev_empty(n, w)
        cs.gen_payload(d_in, n, 100 + i)
        d_mask = dev_empty((n + 31) // 32, 4)
        cs.gen_mask_bernoulli(d_mask, n, float(ps[i]), 200 + i)
        cols.append((d_in, d_mask, dev_empty(n, w), n, counts[i:i + 1]))
    b = cs.Batch(cols)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b.capture_graph(stream=s)
        b.run(stream=s)
        b.check(stream=s)
    torch.cuda.synchronize()
    ref_count = torch.zeros(1, dtype=torch.int64, device="cuda")
    for i, (d_in, d_mask, d_out, n, _) in enumerate(cols):
        ref = torch.empty_like(d_out)
        cs.compressstore(d_in, d_mask, ref, n, ref_count)
        torch.cuda.synchronize()
        k = int(ref_count.item())
        assert int(counts[i].item()) == k
        assert torch.equal(d_out[:k], ref[:k]), i
    b.close()


def test_batch_rejects_bad_columns(cuda):
    import torch
    import gpu_compressstore2_b200 as cs

    d = torch.zeros(1024, dtype=torch.int32, device="cuda")
    c = torch.zeros(1, dtype=torch.int64, device="cuda")
    with pytest.raises(cs.CsError) as ei:
        cs.Batch([(d[1:], d, d, 100, c)])  # payload not 16-byte aligned
    assert ei.value.status == cs._lib.ERR_MISALIGNED

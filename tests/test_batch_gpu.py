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


@pytest.mark.parametrize("algo", ["auto", "1pass", "3pass"])
def test_batch_forms_against_the_oracle(cuda, oracle, algo):
    """Every column of a mixed-width plan forced to one form (or AUTO) equals the oracle,
    direct and graph-replayed."""
    import torch
    import gpu_compressstore2_b200 as cs

    a = {"auto": cs.ALGO_AUTO, "1pass": cs.ALGO_1PASS, "3pass": cs.ALGO_3PASS}[algo]
    cols, host, counts = _columns(oracle, SPECS)
    b = cs.Batch(cols, algo=a)
    nonempty = sum(1 for n, *_ in SPECS if n)
    assert b.one_pass_columns == (nonempty if algo == "1pass" else 0 if algo == "3pass" else b.one_pass_columns)
    b.run()
    b.check()
    _check(oracle, cols, host, counts)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b.capture_graph(stream=s)
        for _ in range(3):  # replays advance the epoch; statuses of earlier runs must not leak
            for (_, _, d_out, _, _) in cols:
                d_out.view(torch.uint8).fill_(0xAB)
            counts.fill_(-5)
            b.run(stream=s)
            b.check(stream=s)
            _check(oracle, cols, host, counts)
    b.close()


def test_batch_table_picks_the_form_per_column(cuda, oracle):
    """With batch-table entries, AUTO gives each column the form of its (width, size,
    selectivity) bucket: the selectivity is measured at plan time, and a mixed plan of 1-pass
    and 3-pass columns still equals the oracle column by column. The 3-pass columns keep
    their form only while they hold at least 256 MB of payload (here a sparse 2^28-element u8
    column); with less, the plan gives every column the 1-pass form."""
    import torch
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    big = (1 << 28) + 12345  # u8, p = 0.01: 268 MB of 3-pass payload
    specs = [(300_000, 4, "b", 0.5), (300_000, 4, "b", 0.99), (300_000, 4, "b", 0.01), (70_001, 8, "b", 0.5),
             (70_001, 8, "b", 0.95), (1_000_000, 1, "b", 0.5), (5000, 2, "r", 8.0), (0, 4, "b", 0.5),
             (big, 1, "b", 0.01)]
    b4 = L.cs_tune_size_bucket(300_000)
    b8 = L.cs_tune_size_bucket(70_001)
    b1 = L.cs_tune_size_bucket(1_000_000)
    b2 = L.cs_tune_size_bucket(5000)
    bb = L.cs_tune_size_bucket(big)
    entries = [(4, b4, 4), (8, b8, 2), (1, b1, 2)]  # (width, size bucket, selectivity bucket) -> 1-pass
    try:
        # start from a table whose buckets of these columns are all unset (3-pass) ...
        for w, sb in ((4, b4), (8, b8), (1, b1), (2, b2), (1, bb)):
            for sel in range(5):
                assert L.cs_tune_batch_set(w, sb, sel, cs.ALGO_AUTO) == 0
        # ... then name the 1-pass form for three of the columns' buckets
        for w, sb, sel in entries:
            assert L.cs_tune_batch_set(w, sb, sel, cs.ALGO_1PASS) == 0
        small_cols, _, _ = _columns(oracle, specs[:-1])
        b = cs.Batch(small_cols)
        assert b.one_pass_columns == 7  # every non-empty column: 3-pass payload under 256 MB
        b.close()
        del small_cols
        cols, host, counts = _columns(oracle, specs)
        b = cs.Batch(cols)
        assert b.one_pass_columns == 3  # p=0.99 u32, p=0.5 u64, p=0.5 u8
        for _ in range(2):
            b.run()
            b.check()
            _check(oracle, cols, host, counts)
            for (_, _, d_out, _, _) in cols:
                d_out.view(torch.uint8).fill_(0xAB)
        b.close()
    finally:  # the packaged table again (it holds entries for every bucket touched here)
        assert L.cs_tune_load(str(cs._lib.TUNE_TABLE).encode()) == 0


def test_batch_matches_plain_calls(cuda):
    """A config-4-shaped batch (uneven lengths log-uniform up to the configuration's 2^24,
    widths 4 and 8, p uniform in [0.01, 0.99]): every column equals the plain call's output,
    for the plan and for its per-call loop."""
    import torch
    import gpu_compressstore2_b200 as cs

    rng = np.random.default_rng(4)
    ncols = 96
    lens = np.exp(rng.uniform(np.log(2 ** 10), np.log(2 ** 24), ncols)).astype(np.int64)
    lens[:2] = [1 << 24, (1 << 24) - 3]  # the configuration's longest columns
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
    # the per-call loop of the same plan writes the same outputs
    saved = [(c[2].clone(), int(counts[i].item())) for i, c in enumerate(cols)]
    for c in cols:
        c[2].fill_(0)
    counts.fill_(-1)
    b.run_per_call()
    torch.cuda.synchronize()
    for i, c in enumerate(cols):
        k = saved[i][1]
        assert int(counts[i].item()) == k
        assert torch.equal(c[2][:k], saved[i][0][:k]), i
    b.close()


def test_batch_rejects_bad_columns(cuda):
    import torch
    import gpu_compressstore2_b200 as cs

    d = torch.zeros(1024, dtype=torch.int32, device="cuda")
    c = torch.zeros(1, dtype=torch.int64, device="cuda")
    with pytest.raises(cs.CsError) as ei:
        cs.Batch([(d[1:], d, d, 100, c)])  # payload not 16-byte aligned
    assert ei.value.status == cs._lib.ERR_MISALIGNED


def test_batch_streaming_pass(cuda, oracle):
    """3-pass columns whose mask blocks together number more than 4 per SM (the streaming form
    of the plan's pass 1 + 2), each column ending in a partial block, widths 1 and 2: every
    column against the oracle."""
    import torch
    import gpu_compressstore2_b200 as cs

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    ncols = (4 * sms) // 7 + 12
    specs = [(6 * (1 << 18) + 1000 + 37 * i, 1 + (i & 1), "b", (0.3, 0.001, 0.9)[i % 3]) for i in range(ncols)]
    cols, host, counts = _columns(oracle, specs)
    b = cs.Batch(cols, algo=cs.ALGO_3PASS)
    b.run()
    b.check()
    _check(oracle, cols, host, counts)
    b.close()


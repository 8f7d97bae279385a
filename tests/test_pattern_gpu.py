"""GPU tests of pattern compaction (compressstore_pattern): the selection is a period of
1..32 elements instead of a mask in memory. Outputs must equal the oracle's compaction by
the same periodic mask, bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import dev_empty, from_dev, to_dev

pytestmark = pytest.mark.gpu

GUARD = 40


def run_pattern(oracle, n, w, pattern, length, seed=3, misalign_out=0):
    import torch
    import gpu_compressstore2_b200 as cs

    payload = oracle.payload(max(n, 1), w, seed)[:n]
    mask = oracle.mask_pattern(n, pattern, length)
    exp = oracle.compact(payload, mask, n) if n else payload[:0]
    d_in = to_dev(payload) if n else dev_empty(4, w)
    out = dev_empty(n + GUARD + misalign_out, w, fill=0xEE)
    d_out = out[misalign_out:]
    d_count = torch.full((1,), -7, dtype=torch.int64, device="cuda")
    cs.compressstore_pattern(d_in, d_out, n, pattern, length, d_count)
    torch.cuda.synchronize()
    k = int(d_count.item())
    assert k == len(exp) == cs.pattern_count(n, pattern, length), (n, w, hex(pattern), length, k, len(exp))
    got = from_dev(d_out, w)
    assert np.array_equal(got[:k], exp), (n, w, hex(pattern), length)
    assert np.all(got[k:].view(np.uint8) == 0xEE), "wrote past the count"


@pytest.mark.parametrize("w", [1, 2, 4, 8])
@pytest.mark.parametrize("length", [1, 2, 3, 5, 8, 13, 16, 31, 32])
def test_pattern_lengths(cuda, oracle, w, length):
    rng = np.random.default_rng(length * 10 + w)
    for _ in range(3):
        pattern = int(rng.integers(1, 2**32)) & ((1 << length) - 1) or 1
        for n in (1, 31, length, 1000, 65_536 + 7, 300_001):
            run_pattern(oracle, n, w, pattern, length)


@pytest.mark.parametrize("w", [1, 4, 8])
def test_pattern_edges(cuda, oracle, w):
    run_pattern(oracle, 0, w, 0b1, 1)                    # empty column
    run_pattern(oracle, 100_000, w, 0, 8)                # zero pattern: count 0, nothing written
    run_pattern(oracle, 100_000, w, 0xFFFFFFFF, 32)      # every element: a copy
    run_pattern(oracle, 100_000, w, 0xFF, 8)             # every element, short period
    run_pattern(oracle, 100_000, w, 0xFFFFFF00, 8)       # bits past the length are ignored: count 0
    run_pattern(oracle, 5, w, 0b10011, 7)                # n < length
    run_pattern(oracle, 77_777, w, 0x80000000, 32)       # one element per period
    if w < 8:
        run_pattern(oracle, 50_001, w, 0b1011, 4, misalign_out=1)  # element-aligned output


def test_pattern_full_size(cuda):
    """n = 2^28 float32, period 8 with 4 selected: equals masked_select over the pattern."""
    import torch
    import gpu_compressstore2_b200 as cs

    n = 1 << 28
    d_in = torch.empty(n, dtype=torch.int32, device="cuda")
    cs.gen_payload(d_in, n, 9, float_unit=True)
    d_out = torch.empty(n, dtype=torch.int32, device="cuda")
    d_count = torch.zeros(1, dtype=torch.int64, device="cuda")
    pattern, length = 0b10110010, 8
    cs.compressstore_pattern(d_in, d_out, n, pattern, length, d_count)
    torch.cuda.synchronize()
    k = int(d_count.item())
    assert k == cs.pattern_count(n, pattern, length) == n // 2
    bits = torch.tensor([(pattern >> b) & 1 for b in range(length)], dtype=torch.bool, device="cuda")
    ref = torch.masked_select(d_in.view(-1, length), bits.view(1, -1))
    assert torch.equal(d_out[:k], ref)


def test_pattern_argument_errors(cuda):
    import torch
    import gpu_compressstore2_b200 as cs

    x = torch.zeros(64, dtype=torch.int32, device="cuda")
    c = torch.zeros(1, dtype=torch.int64, device="cuda")
    for length in (0, 33):
        with pytest.raises(cs.CsError):
            cs.compressstore_pattern(x, x, 64, 1, length, c)


@pytest.mark.parametrize("length", [1, 3, 8, 13, 32])
def test_gen_mask_pattern_matches_oracle(cuda, oracle, length):
    import torch
    import gpu_compressstore2_b200 as cs

    pattern = 0x9E3779B9 & ((1 << length) - 1) | 1
    for n in (1, 33, 1000, 100_003):
        d_mask = torch.full(((n + 31) // 32,), -1, dtype=torch.int32, device="cuda")
        cs.gen_mask_pattern(d_mask, n, pattern, length)
        torch.cuda.synchronize()
        assert np.array_equal(from_dev(d_mask, 4), oracle.mask_pattern(n, pattern, length)), (n, length)

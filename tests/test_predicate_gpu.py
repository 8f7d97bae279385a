"""GPU tests of predicate compaction (compressstore_if): the selection is a comparison
evaluated on the payload on the device. Expected results: numpy evaluates the predicate
(IEEE comparisons: false with a NaN, != true), the oracle compacts by the resulting mask."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import UNSIGNED, dev_empty, from_dev, to_dev

pytestmark = pytest.mark.gpu

GUARD = 24
NP = {0: np.uint8, 1: np.uint16, 2: np.uint32, 3: np.uint64, 4: np.int8, 5: np.int16, 6: np.int32, 7: np.int64,
      8: np.float32, 9: np.float64}
OPS = {
    "<": lambda x, a, b: x < a, "<=": lambda x, a, b: x <= a, ">": lambda x, a, b: x > a,
    ">=": lambda x, a, b: x >= a, "==": lambda x, a, b: x == a, "!=": lambda x, a, b: x != a,
    "between": lambda x, a, b: (a <= x) & (x <= b),
}


def sample(rng, dt, n):
    if np.issubdtype(dt, np.floating):
        x = rng.normal(0.0, 100.0, n).astype(dt)
        k = max(n // 50, 1)
        for v in (np.nan, np.inf, -np.inf, -0.0, 0.0, 7.5):
            x[rng.integers(0, n, k)] = v
        return x
    info = np.iinfo(dt)
    x = rng.integers(info.min, info.max, n, dtype=dt, endpoint=True)
    k = max(n // 50, 1)
    for v in (info.min, info.max, 0, 7):
        x[rng.integers(0, n, k)] = v
    return x


def pack(bits):
    b = np.packbits(bits.astype(np.uint8), bitorder="little")
    b = np.concatenate([b, np.zeros((-len(b)) % 4, dtype=np.uint8)])
    return b.view(np.uint32)


def run_pred(oracle, x, op, a, b=None, with_mask=True):
    import torch
    import gpu_compressstore2_b200 as cs

    n = len(x)
    code = [k for k, v in NP.items() if v == x.dtype.type][0]
    w = x.dtype.itemsize
    bits = OPS[op](x, x.dtype.type(a), x.dtype.type(b) if b is not None else None) if n else np.zeros(0, bool)
    words = pack(bits) if n else np.zeros(0, np.uint32)
    raw = x.view(UNSIGNED[w])
    exp = oracle.compact(raw, words, n) if n else raw[:0]
    d_in = to_dev(raw) if n else dev_empty(16, w)
    d_out = dev_empty(n + GUARD, w, fill=0xA5)
    d_mask = torch.full((max((n + 31) // 32, 1) + 4,), -1, dtype=torch.int32, device="cuda") if with_mask else None
    d_count = torch.full((1,), -3, dtype=torch.int64, device="cuda")
    pred = cs.predicate(op, a, b, elem_type=code)
    cs.compressstore_if(d_in, d_out, n, pred, d_count, d_mask_out=d_mask)
    torch.cuda.synchronize()
    k = int(d_count.item())
    assert k == len(exp), (x.dtype, op, a, b, n, k, len(exp))
    got = from_dev(d_out, w)
    assert np.array_equal(got[:k], exp), (x.dtype, op, a, b, n)
    assert np.all(got[k:].view(np.uint8) == 0xA5), "wrote past the count"
    if with_mask and n:
        mw = from_dev(d_mask, 4)[: (n + 31) // 32]
        assert np.array_equal(mw, words), (x.dtype, op, n)
    cs.compressstore_check()


@pytest.mark.parametrize("code", list(NP))
@pytest.mark.parametrize("op", list(OPS))
def test_predicate_types_and_ops(cuda, oracle, code, op):
    dt = NP[code]
    rng = np.random.default_rng(code * 31 + len(op))
    for n in (1, 77, 4096, 4097, 300_001):
        x = sample(rng, dt, n)
        a = x[len(x) // 2] if not (np.issubdtype(dt, np.floating) and np.isnan(x[len(x) // 2])) else dt(1.5)
        b = None
        if op == "between":
            a, b = (dt(-20), dt(60)) if np.issubdtype(dt, np.floating) or np.iinfo(dt).min < 0 else (dt(10), dt(200))
        run_pred(oracle, x, op, a, b, with_mask=(n % 2 == 1))


@pytest.mark.parametrize("n", [0, 31, 32, 33, (1 << 18) - 1, 1 << 18, (1 << 18) + 1, 3 * (1 << 18) + 12345])
def test_predicate_sizes(cuda, oracle, n):
    rng = np.random.default_rng(n)
    x = rng.normal(0, 300, max(n, 1)).astype(np.float32)[:n]
    run_pred(oracle, x, ">", np.float32(200.0))  # the reference's predicate_function: x > threshold


def test_predicate_extremes(cuda, oracle):
    x = np.array([np.nan, -np.inf, np.inf, -0.0, 0.0] * 999, dtype=np.float64)
    for op in OPS:
        run_pred(oracle, x, op, 0.0, 1.0 if op == "between" else None)
    run_pred(oracle, x, "==", np.inf)
    run_pred(oracle, x, "<", -np.inf)  # selects nothing
    y = np.array([0, 255, 128, 1] * 3001, dtype=np.uint8)
    run_pred(oracle, y, ">", 254)
    run_pred(oracle, y, "<=", 255)     # selects everything
    z = np.array([np.iinfo(np.int64).min, -1, 0, np.iinfo(np.int64).max] * 2049, dtype=np.int64)
    run_pred(oracle, z, ">=", np.iinfo(np.int64).min)
    run_pred(oracle, z, "between", -1, 0)


def test_predicate_full_size(cuda):
    """n = 2^28 float32 uniform [0, 1), x > 0.5: equals masked_select of the comparison."""
    import torch
    import gpu_compressstore2_b200 as cs

    n = 1 << 28
    d_in = torch.empty(n, dtype=torch.int32, device="cuda")
    cs.gen_payload(d_in, n, 4, float_unit=True)
    f = d_in.view(torch.float32)
    d_out = torch.empty(n, dtype=torch.int32, device="cuda")
    d_count = torch.zeros(1, dtype=torch.int64, device="cuda")
    cs.compressstore_if(d_in, d_out, n, cs.predicate(">", 0.5, dtype=torch.float32), d_count)
    torch.cuda.synchronize()
    sel = f > 0.5
    k = int(d_count.item())
    assert k == int(sel.sum().item())
    assert torch.equal(d_out[:k], torch.masked_select(d_in, sel))


@pytest.mark.parametrize("code", [0, 1, 3, 6, 9])
def test_predicate_long_columns_every_width(cuda, oracle, code):
    """Columns long enough that most of the mask pass runs its bounds-free path for complete
    iterations and the rest its checked path (the last, partial iteration), at every element
    width: output, count and mask words against numpy + the oracle."""
    rng = np.random.default_rng(100 + code)
    dt = NP[code]
    n = ((1 << 24) + 12345) // dt().itemsize
    x = sample(rng, dt, n)
    a = dt(0) if np.issubdtype(dt, np.floating) else x[n // 2]
    run_pred(oracle, x, ">", a)
    run_pred(oracle, x, "between", a, dt(np.iinfo(dt).max if np.issubdtype(dt, np.integer) else 50.0))

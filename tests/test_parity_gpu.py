"""GPU parity: every algorithm through the C ABI against the CPU oracle, bit for bit, plus
the reference-generated golden fixtures, edge cases, and the size-independent properties
at full size. Needs a B200."""
from __future__ import annotations

import ctypes
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from conftest import dev_empty, from_dev, to_dev

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
ALGOS = ["auto", "1pass", "3pass", "naive"]
GUARD = 64  # elements past the capacity the call may use; must stay untouched


def _algo(name):
    import gpu_compressstore2_b200 as cs

    return {"auto": cs.ALGO_AUTO, "1pass": cs.ALGO_1PASS, "3pass": cs.ALGO_3PASS, "naive": cs.ALGO_NAIVE}[name]


def run_cs(payload: np.ndarray, mask: np.ndarray, n: int, algo="auto", chunk_length=0, workspace=None, **kw):
    import torch
    import gpu_compressstore2_b200 as cs

    w = payload.dtype.itemsize
    d_in = to_dev(payload) if n else dev_empty(1, w)
    d_mask = to_dev(mask) if len(mask) else dev_empty(1, 4)
    d_out = dev_empty(n + GUARD, w, fill=0xAB)
    d_count = torch.full((1,), -7, dtype=torch.int64, device="cuda")
    cs.compressstore(d_in, d_mask, d_out, n, d_count, algo=_algo(algo), chunk_length=chunk_length,
                     workspace=workspace, **kw)
    torch.cuda.synchronize()
    count = int(d_count.item())
    out = from_dev(d_out, w)
    return out, count


def check_against_oracle(oracle, payload, mask, n, algo="auto", chunk_length=0, **kw):
    exp = oracle.compact(payload, mask, n)
    out, count = run_cs(payload, mask, n, algo, chunk_length, **kw)
    assert count == len(exp), (algo, n, count, len(exp))
    assert np.array_equal(out[:count], exp), (algo, n, chunk_length)
    guard = out[count:].view(np.uint8)
    assert np.all(guard == 0xAB), f"wrote past the count ({algo}, n={n})"


# ----------------------------------------------------------------------------- generators
@pytest.mark.parametrize("n", [1, 31, 32, 33, 1000, 65536 + 17])
def test_generators_match_oracle(cuda, oracle, n):
    import torch
    import gpu_compressstore2_b200 as cs

    for w in (1, 2, 4, 8):
        d = dev_empty(n, w)
        cs.gen_payload(d, n, seed=77 + w)
        torch.cuda.synchronize()
        assert np.array_equal(from_dev(d, w)[:n], oracle.payload(n, w, 77 + w))
    d = dev_empty(n, 4)
    cs.gen_payload(d, n, seed=5, float_unit=True)
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(d, 4)[:n], oracle.payload(n, 4, 5, float_unit=True))
    nw = (n + 31) // 32
    m = dev_empty(nw, 4)
    for p in (0.0, 0.001, 0.37, 1.0):
        cs.gen_mask_bernoulli(m, n, p, seed=9)
        torch.cuda.synchronize()
        assert np.array_equal(from_dev(m, 4)[:nw], oracle.mask_bernoulli(n, p, 9))
    for mean in (8.0, 64.0, 4096.0):
        cs.gen_mask_runs(m, n, mean, seed=10)
        torch.cuda.synchronize()
        assert np.array_equal(from_dev(m, 4)[:nw], oracle.mask_runs(n, mean, 10))
    cs.gen_mask_dense_prefix(m, n, 0.1)
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(m, 4)[:nw], oracle.mask_dense_prefix(n, 0.1))


# ----------------------------------------------------------------------------- golden
def test_golden_small_fixtures(cuda, oracle):
    meta = json.loads((GOLDEN / "golden.json").read_text())
    arrays = np.load(GOLDEN / "golden_small.npz")
    for rec in meta["small"]:
        name, n = rec["name"], rec["n"]
        for algo in ALGOS:
            out, count = run_cs(arrays[name + "__payload"], arrays[name + "__mask"], n, algo)
            assert count == rec["count"], (name, algo)
            assert np.array_equal(out[:count], arrays[name + "__out"]), (name, algo)


@pytest.mark.parametrize("algo", ALGOS)
def test_golden_large_fixtures_device_inputs(cuda, algo):
    """Inputs generated on the device from the fixture seeds; output digest must equal the
    reference CPU compaction's."""
    import torch
    import gpu_compressstore2_b200 as cs

    meta = json.loads((GOLDEN / "golden.json").read_text())
    for rec in meta["large"]:
        n, w, kind = rec["n"], rec["elem_bytes"], rec["kind"]
        d_in = dev_empty(n, w)
        cs.gen_payload(d_in, n, rec["payload_seed"], float_unit=(kind == "bernoulli_f32"))
        d_mask = dev_empty((n + 31) // 32, 4)
        if kind.startswith("bernoulli"):
            cs.gen_mask_bernoulli(d_mask, n, rec["param"], rec["mask_seed"])
        elif kind == "runs":
            cs.gen_mask_runs(d_mask, n, rec["param"], rec["mask_seed"])
        d_out = dev_empty(n, w)
        d_count = torch.zeros(1, dtype=torch.int64, device="cuda")
        cs.compressstore(d_in, d_mask, d_out, n, d_count, algo=_algo(algo))
        torch.cuda.synchronize()
        count = int(d_count.item())
        assert count == rec["count"], (rec["name"], algo)
        digest = hashlib.sha256(from_dev(d_out, w)[:count].tobytes()).hexdigest()
        assert digest == rec["sha256"], (rec["name"], algo)


# ----------------------------------------------------------------------------- sweeps
EDGE_SIZES = [0, 1, 7, 31, 32, 33, 255, 1000, 4095, 4096, 4097, 8191, 8192, 8193, 16384 + 5, 32768 - 1, 32768,
              32768 + 33, 3 * 32768 + 1234, 100_003, 131072 - 1, 131072, 131072 + 1, 4 * 131072 + 77]


@pytest.mark.parametrize("w", [1, 2, 4, 8])
@pytest.mark.parametrize("algo", ALGOS)
def test_edge_sizes(cuda, oracle, w, algo):
    for n in EDGE_SIZES:
        payload = oracle.payload(n, w, 1000 + n)
        for p in (0.5, 0.03):
            mask = oracle.mask_bernoulli(n, p, 2000 + n)
            check_against_oracle(oracle, payload, mask, n, algo)


@pytest.mark.parametrize("w", [1, 2, 4, 8])
@pytest.mark.parametrize("algo", ALGOS)
def test_mask_shapes(cuda, oracle, w, algo):
    n = 5 * 131072 + 999
    payload = oracle.payload(n, w, 31)
    nw = (n + 31) // 32
    masks = {
        "zeros": np.zeros(nw, np.uint32),
        "ones": np.full(nw, 0xFFFFFFFF, np.uint32),  # includes garbage bits past n
        "single_first": np.eye(1, nw, 0, dtype=np.uint32)[0],
        "single_last": np.zeros(nw, np.uint32),
        "runs8": oracle.mask_runs(n, 8.0, 3),
        "runs4096": oracle.mask_runs(n, 4096.0, 4),
        "dense10": oracle.mask_dense_prefix(n, 0.1),
        "p001": oracle.mask_bernoulli(n, 0.001, 5),
        "p99": oracle.mask_bernoulli(n, 0.99, 6),
        "garbage_tail": oracle.mask_bernoulli(n, 0.5, 7) | np.uint32(0),
    }
    masks["single_last"][(n - 1) // 32] = np.uint32(1 << ((n - 1) % 32))
    masks["garbage_tail"][-1] |= np.uint32(0xFFFFFFFF) << np.uint32(n % 32)
    for name, mask in masks.items():
        check_against_oracle(oracle, payload, mask, n, algo)


@pytest.mark.parametrize("chunk_length", [32, 64, 256, 1024, 4096, 8192, 65536])
@pytest.mark.parametrize("algo", ["3pass", "naive"])
def test_chunk_lengths(cuda, oracle, chunk_length, algo):
    for w in (1, 4, 8):
        n = 200_000 + w
        payload = oracle.payload(n, w, 3)
        mask = oracle.mask_bernoulli(n, 0.4, 4)
        check_against_oracle(oracle, payload, mask, n, algo, chunk_length)


def test_grid_sizes(cuda, oracle):
    n = 300_001
    payload = oracle.payload(n, 4, 8)
    mask = oracle.mask_bernoulli(n, 0.5, 9)
    for algo in ("1pass", "3pass"):
        for g in (1, 2, 7, 148, 1000):
            check_against_oracle(oracle, payload, mask, n, algo, grid_dim=g)


def test_skip_modes(cuda, oracle):
    n = 400_000
    payload = oracle.payload(n, 4, 8)
    for p in (0.001, 0.5):
        mask = oracle.mask_bernoulli(n, p, 9)
        for algo in ("1pass", "3pass"):
            for skip in (1, 2):
                check_against_oracle(oracle, payload, mask, n, algo, skip=skip)


def test_misaligned_pointers_route_to_naive(cuda, oracle):
    import torch
    import gpu_compressstore2_b200 as cs

    n = 10_000
    payload = oracle.payload(n + 1, 4, 1)
    mask = oracle.mask_bernoulli(n, 0.5, 2)
    exp = oracle.compact(payload[1:], mask, n)
    d_in = to_dev(payload)[1:]  # 4-byte aligned, not 16
    d_mask = to_dev(mask)
    d_out = dev_empty(n + 1, 4)[1:]
    d_count = torch.zeros(1, dtype=torch.int64, device="cuda")
    cs.compressstore(d_in, d_mask, d_out, n, d_count)  # AUTO routes around the TMA path
    torch.cuda.synchronize()
    k = int(d_count.item())
    assert k == len(exp)
    assert np.array_equal(from_dev(d_out, 4)[:k], exp)
    with pytest.raises(cs.CsError) as ei:
        cs.compressstore(d_in, d_mask, d_out, n, d_count, algo=cs.ALGO_1PASS)
    assert ei.value.status == cs._lib.ERR_MISALIGNED


def test_repeated_calls_one_workspace(cuda, oracle):
    """Epochs advance call after call on one workspace; sizes shrink and grow."""
    import gpu_compressstore2_b200 as cs

    ws = cs.Workspace.for_call(1 << 20, 1)
    rng = np.random.default_rng(0)
    for it in range(40):
        n = int(rng.integers(1, 1 << 18))
        w = int(rng.choice([1, 2, 4, 8]))
        payload = oracle.payload(n, w, it)
        mask = oracle.mask_bernoulli(n, float(rng.random()), it + 100)
        algo = ["1pass", "3pass", "naive"][it % 3]
        check_against_oracle(oracle, payload, mask, n, algo, workspace=ws)
    ws.check()


def test_pass_entry_points(cuda, oracle):
    import torch
    import gpu_compressstore2_b200 as cs

    n = 1_000_003
    w = 4
    payload = oracle.payload(n, w, 11)
    mask = oracle.mask_bernoulli(n, 0.3, 12)
    exp = oracle.compact(payload, mask, n)
    d_in, d_mask = to_dev(payload), to_dev(mask)
    for L in (32, 1024, 8192, 65536):
        c = (n + L - 1) // L
        d_counts = torch.zeros(c, dtype=torch.int32, device="cuda")
        cs.popc_chunks(d_mask, n, L, d_counts)
        torch.cuda.synchronize()
        counts = from_dev(d_counts, 4)
        assert np.array_equal(counts, oracle.popc_chunks(mask, n, L))
        d_offs = torch.zeros(c, dtype=torch.int64, device="cuda")
        d_total = torch.zeros(1, dtype=torch.int64, device="cuda")
        cs.chunk_prefix_sum(d_counts, c, d_offs, d_total)
        torch.cuda.synchronize()
        offs, total = oracle.exclusive_scan(counts)
        assert np.array_equal(from_dev(d_offs, 8), offs)
        assert int(d_total.item()) == total == len(exp)
        algos = [cs.ALGO_NAIVE] + ([cs.ALGO_3PASS] if L <= 4 * cs.tile_elems(w) else [])
        for algo in algos:
            d_out = dev_empty(n, w)
            cs.writeout(d_in, d_mask, d_out, n, d_offs, d_counts, L, algo)
            torch.cuda.synchronize()
            assert np.array_equal(from_dev(d_out, w)[:total], exp)


def test_scan_large_chunk_count(cuda, oracle):
    import torch
    import gpu_compressstore2_b200 as cs

    rng = np.random.default_rng(5)
    for c in (1, 4095, 4096, 4097, 1_000_000):
        counts = rng.integers(0, 1 << 16, c).astype(np.uint32)
        d_counts = to_dev(counts)
        d_offs = torch.zeros(c, dtype=torch.int64, device="cuda")
        d_total = torch.zeros(1, dtype=torch.int64, device="cuda")
        cs.chunk_prefix_sum(d_counts, c, d_offs, d_total)
        torch.cuda.synchronize()
        offs, total = oracle.exclusive_scan(counts)
        assert np.array_equal(from_dev(d_offs, 8), offs)
        assert int(d_total.item()) == total


@pytest.mark.parametrize("w", [1, 2, 4, 8])
def test_cub_flagged_comparator(cuda, oracle, w):
    import torch
    import gpu_compressstore2_b200 as cs

    n = 123_457
    payload = oracle.payload(n, w, 21)
    mask = oracle.mask_bernoulli(n, 0.5, 22)
    exp = oracle.compact(payload, mask, n)
    d_out = dev_empty(n, w)
    d_count = torch.zeros(1, dtype=torch.int64, device="cuda")
    cs.cub_flagged(to_dev(payload), to_dev(mask), d_out, n, d_count)
    torch.cuda.synchronize()
    k = int(d_count.item())
    assert k == len(exp)
    assert np.array_equal(from_dev(d_out, w)[:k], exp)


def test_auto_takes_the_entry_of_a_stated_selectivity(cuda, oracle):
    """With a stated selectivity (cs_config.selectivity), CS_ALGO_AUTO takes the table's
    entry for that selectivity bucket; an unknown fraction or a bucket without an entry keeps
    the (width, size) entry. The form that ran shows in the launch count (the 1-pass form is
    one launch, the 3-pass form more); every result equals the oracle's, and a fraction
    outside [0, 1] is rejected."""
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    n, w = 300_000, 4
    b = L.cs_tune_size_bucket(n)
    payload = oracle.payload(n, w, 61)
    masks = {p: oracle.mask_bernoulli(n, p, 62) for p in (0.5, 0.99)}
    assert L.cs_tune_set(w, b, cs.ALGO_3PASS, 4096) == 0
    for sb in (0, 1, 2, 3):  # no entry for these buckets: the (width, size) entry applies
        assert L.cs_tune_sel_set(w, b, sb, cs.ALGO_AUTO, 0) == 0
    assert L.cs_tune_sel_set(w, b, 4, cs.ALGO_1PASS, 1024) == 0  # selected fraction above 0.95
    try:
        for p, sel, one_pass in ((0.99, 0.99, True), (0.99, 0.0, False), (0.5, 0.5, False), (0.5, 0.96, True)):
            check_against_oracle(oracle, payload, masks[p], n, "auto", selectivity=sel)  # warm: scratch sized
            before = cs.launch_count()
            check_against_oracle(oracle, payload, masks[p], n, "auto", selectivity=sel)
            launches = cs.launch_count() - before
            assert (launches == 1) == one_pass, (p, sel, launches)
        with pytest.raises(cs.CsError):
            run_cs(payload, masks[0.5], n, "auto", selectivity=1.5)
    finally:
        for sb in range(5):
            L.cs_tune_sel_set(w, b, sb, cs.ALGO_AUTO, 0)
        L.cs_tune_set(w, b, cs.ALGO_AUTO, 1024)
        L.cs_tune_load(str(cs._lib.TUNE_TABLE).encode())


def test_lookback_timeout_reports_error(cuda, oracle):
    """A tile that nobody processes (the tile counter is advanced past it by hand) leaves
    its successors waiting: the bounded look-back gives up, records CS_ERR_TIMEOUT, writes
    the error count, writes nothing, and the workspace works again afterwards."""
    import torch
    import gpu_compressstore2_b200 as cs

    n = 64 * 8192
    payload = oracle.payload(n, 4, 1)
    mask = oracle.mask_bernoulli(n, 0.5, 2)
    cfg = cs.make_config(cs.ALGO_1PASS)
    ws = cs.Workspace.for_call(n, 4, cfg)
    torch.cuda.synchronize()
    off = ws.ptr - ws.buf.data_ptr()
    ws.buf[off + 16: off + 20].view(torch.int32).fill_(1)  # tile_counter = 1: tile 0 is never taken
    d_in, d_mask = to_dev(payload), to_dev(mask)
    d_out = dev_empty(n, 4, fill=0xCD)
    d_count = torch.zeros(1, dtype=torch.int64, device="cuda")
    cs.compressstore(d_in, d_mask, d_out, n, d_count, algo=cs.ALGO_1PASS, timeout_ns=20_000_000, workspace=ws)
    with pytest.raises(cs.CsError) as ei:
        ws.check()
    assert ei.value.status == cs._lib.ERR_TIMEOUT
    assert int(d_count.item()) == -1  # CS_COUNT_ERROR as int64
    assert np.all(from_dev(d_out, 4).view(np.uint8) == 0xCD)
    # the workspace recovers
    check_against_oracle(oracle, payload, mask, n, "1pass", workspace=ws)
    ws.check()


def test_scan_timeout_reports_error(cuda, oracle):
    import torch
    import gpu_compressstore2_b200 as cs

    n = 64 * 8192
    payload = oracle.payload(n, 4, 1)
    mask = oracle.mask_bernoulli(n, 0.5, 2)
    cfg = cs.make_config(cs.ALGO_3PASS, 32)
    ws = cs.Workspace.for_call(n, 4, cfg)
    torch.cuda.synchronize()
    off = ws.ptr - ws.buf.data_ptr()
    ws.buf[off + 24: off + 28].view(torch.int32).fill_(1)  # scan_tile_counter = 1
    d_out = dev_empty(n, 4, fill=0xCD)
    d_count = torch.zeros(1, dtype=torch.int64, device="cuda")
    cs.compressstore(to_dev(payload), to_dev(mask), d_out, n, d_count, algo=cs.ALGO_3PASS, chunk_length=32,
                     timeout_ns=20_000_000, workspace=ws)
    with pytest.raises(cs.CsError) as ei:
        ws.check()
    assert ei.value.status == cs._lib.ERR_TIMEOUT
    assert int(d_count.item()) == -1
    assert np.all(from_dev(d_out, 4).view(np.uint8) == 0xCD)
    check_against_oracle(oracle, payload, mask, n, "3pass", chunk_length=32, workspace=ws)


# ----------------------------------------------------------------------------- streaming pass 1 + 2
def _words(rng, k: int, density_log2: int) -> np.ndarray:
    """k mask words whose bits are set with probability 2^-density_log2 (AND of random words)."""
    m = np.full(k, 0xFFFFFFFF, dtype=np.uint32)
    for _ in range(density_log2):
        m &= rng.integers(0, 1 << 32, size=k, dtype=np.uint64).astype(np.uint32)
    return m


@pytest.mark.parametrize("chunk_length", [128, 1024, 4096])
def test_streaming_pass_ragged_column(cuda, oracle, chunk_length):
    """A u8 column of more than 4 mask blocks (2^18 elements) per SM, where passes 1 + 2 take
    the streaming form, whose last block is partial: a sparse first third (units the hybrid
    gathers), a dense rest, an empty stretch. The 3-pass output and count against the oracle,
    and nothing written past the count."""
    import torch

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    n = (4 * sms + 9) * (1 << 18) + 12345
    rng = np.random.default_rng(chunk_length)
    words = (n + 31) // 32
    third = words // 3
    mask = np.concatenate([_words(rng, third, 9), _words(rng, words - third, 1)])
    mask[third + 5000:third + 60000] = 0
    payload = rng.integers(0, 256, size=n, dtype=np.uint8)
    check_against_oracle(oracle, payload, mask, n, "3pass", chunk_length=chunk_length)
    check_against_oracle(oracle, payload, mask, n, "auto")


# ----------------------------------------------------------------------------- full size
@pytest.mark.parametrize("algo", ["1pass", "3pass"])
def test_full_size_f32_properties(cuda, algo):
    """n = 2^28 float32 at each selectivity: count equals the mask popcount and the output
    equals torch.masked_select over the unpacked mask (an independent device path)."""
    import torch
    import gpu_compressstore2_b200 as cs

    n = 1 << 28
    d_in = torch.empty(n, dtype=torch.int32, device="cuda")
    cs.gen_payload(d_in, n, 1, float_unit=True)
    d_mask = torch.empty(n // 32, dtype=torch.int32, device="cuda")
    d_out = torch.empty(n, dtype=torch.int32, device="cuda")
    d_count = torch.zeros(1, dtype=torch.int64, device="cuda")
    shifts = torch.arange(32, device="cuda", dtype=torch.int32)
    for p in (0.001, 0.5, 0.99):
        cs.gen_mask_bernoulli(d_mask, n, p, 2)
        cs.compressstore(d_in, d_mask, d_out, n, d_count, algo=_algo(algo))
        torch.cuda.synchronize()
        k = int(d_count.item())
        bits = ((d_mask.view(-1, 1) >> shifts) & 1).view(-1).bool()
        assert k == int(bits.sum().item())
        ref = torch.masked_select(d_in, bits)
        assert torch.equal(d_out[:k], ref)
        del bits, ref

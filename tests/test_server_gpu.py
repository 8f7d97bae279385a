"""GPU tests of the serving loop (cs_server_*): requests over device-resident columns,
admitted by an output-memory budget and batched as they arrive. Each result must be the
oracle's compaction and the same whether the request ran alone or inside a mixed batch."""
from __future__ import annotations

import time

import numpy as np
import pytest

from conftest import from_dev, to_dev

pytestmark = pytest.mark.gpu

MIB = 1 << 20


def _requests(oracle, specs, seed0=0):
    """specs: (n, w, kind, par). Returns device inputs and the oracle's outputs."""
    reqs = []
    for i, (n, w, kind, par) in enumerate(specs):
        payload = oracle.payload(max(n, 1), w, 700 + seed0 + i)[:n]
        if kind == "b":
            mask = oracle.mask_bernoulli(max(n, 1), par, 1300 + seed0 + i)
        else:
            mask = oracle.mask_runs(max(n, 1), par, 1300 + seed0 + i)
        exp = oracle.compact(payload, mask, n) if n else payload[:0]
        d_in = to_dev(payload if n else np.zeros(4, dtype=payload.dtype))
        d_mask = to_dev(mask)
        reqs.append((d_in, d_mask, n, w, exp))
    return reqs


def _out(server, ticket, res, w):
    t = server.output(ticket, res)
    return from_dev(t, w) if res.count else np.zeros(0, dtype={1: np.uint8, 2: np.uint16, 4: np.uint32,
                                                                8: np.uint64}[w])


SPECS = [
    (0, 4, "b", 0.5), (1, 4, "b", 1.0), (31, 1, "b", 0.5), (33, 8, "b", 0.7), (1000, 2, "b", 0.01),
    (4096, 4, "b", 0.5), (4097, 8, "b", 0.99), (32_769, 4, "b", 0.001), (131_072, 1, "r", 8.0),
    (131_073, 2, "b", 0.02), (200_000, 4, "b", 0.5), (262_144, 8, "r", 4096.0), (300_001, 4, "b", 0.0),
    (500_000, 1, "b", 0.3), (524_288, 4, "b", 0.03), (1_048_577, 4, "b", 0.5), (777_777, 8, "b", 0.02),
    (2_000_000, 4, "r", 64.0), (5, 4, "b", 0.5), (65_536, 8, "b", 1.0), (4_194_304, 4, "b", 0.9),
    (3_000_001, 4, "b", 0.2), (12_345, 4, "b", 0.6), (9_999, 8, "b", 0.4),
]


def _run_alone(server, reqs):
    outs = []
    for d_in, d_mask, n, w, _ in reqs:
        t = server.submit(d_in, d_mask, n, w)
        r = server.wait(t, timeout_s=30)
        assert r.status == 0, r
        assert r.batch_size in (0, 1)
        outs.append((r.count, _out(server, t, r, w).copy()))
        server.release(t)
    return outs


def test_server_mixed_equals_alone(cuda, oracle):
    import gpu_compressstore2_b200 as cs

    reqs = _requests(oracle, SPECS)
    with cs.Server(out_budget_bytes=256 * MIB, max_batch=16, slots=3) as srv:
        alone = _run_alone(srv, reqs)
        for (count, out), (_, _, n, w, exp) in zip(alone, reqs):
            assert count == len(exp), (n, w)
            assert np.array_equal(out, exp), (n, w)
        # the same requests arriving together: they are admitted, batched and overlapped
        tickets = [srv.submit(d_in, d_mask, n, w) for d_in, d_mask, n, w, _ in reqs]
        sizes = []
        for t, (count, out), (_, _, n, w, exp) in zip(tickets, alone, reqs):
            r = srv.wait(t, timeout_s=30)
            assert r.status == 0, r
            assert r.count == count, (n, w)
            got = _out(srv, t, r, w)
            assert np.array_equal(got, out), (n, w)
            assert np.array_equal(got, exp), (n, w)
            sizes.append(r.batch_size)
        for t in tickets:
            srv.release(t)
        st = srv.stats()
        assert max(sizes) > 1, sizes  # at least one real mix
        assert st["arena_used"] == 0
        assert st["completed"] == st["submitted"] == 2 * len(SPECS)
        assert st["batches"] < st["submitted"]


def test_server_mixed_repeated_interleaved(cuda, oracle):
    """Waves of requests submitted while earlier waves are still on the GPU."""
    import gpu_compressstore2_b200 as cs

    reqs = _requests(oracle, SPECS, seed0=50)
    with cs.Server(out_budget_bytes=512 * MIB, max_batch=8, slots=2) as srv:
        live = []
        for wave in range(4):
            for d_in, d_mask, n, w, exp in reqs[wave::2]:
                live.append((srv.submit(d_in, d_mask, n, w), w, exp))
            # drain half of what is outstanding while the rest keeps running
            keep = []
            for i, (t, w, exp) in enumerate(live):
                if i % 2 == 0:
                    r = srv.wait(t, timeout_s=30)
                    assert r.status == 0
                    assert np.array_equal(_out(srv, t, r, w), exp)
                    srv.release(t)
                else:
                    keep.append((t, w, exp))
            live = keep
        for t, w, exp in live:
            r = srv.wait(t, timeout_s=30)
            assert r.status == 0
            assert np.array_equal(_out(srv, t, r, w), exp)
            srv.release(t)
        assert srv.stats()["arena_used"] == 0


def test_server_per_call_mode(cuda, oracle):
    import gpu_compressstore2_b200 as cs

    reqs = _requests(oracle, SPECS[:16], seed0=100)
    with cs.Server(out_budget_bytes=128 * MIB, slots=1, mode=cs.SERVE_PER_CALL) as srv:
        tickets = [srv.submit(d_in, d_mask, n, w) for d_in, d_mask, n, w, _ in reqs]
        for t, (_, _, n, w, exp) in zip(tickets, reqs):
            r = srv.wait(t, timeout_s=30)
            assert r.status == 0
            assert r.batch_size in (0, 1)
            assert np.array_equal(_out(srv, t, r, w), exp), (n, w)
            srv.release(t)


def test_server_admission_budget(cuda, oracle):
    """Requests wait for arena space in arrival order; a release admits the next one."""
    import gpu_compressstore2_b200 as cs

    n, w = 65_536, 4  # 256 KiB reservation each, all elements selected (no shrink)
    reqs = _requests(oracle, [(n, w, "b", 1.0)] * 6, seed0=200)
    with cs.Server(out_budget_bytes=1 * MIB, max_batch=4, slots=2) as srv:
        tickets = [srv.submit(d_in, d_mask, nn, ww) for d_in, d_mask, nn, ww, _ in reqs]
        first = [srv.wait(t, timeout_s=30) for t in tickets[:4]]
        assert all(r.status == 0 and r.count == n for r in first)
        time.sleep(0.05)
        assert srv.poll(tickets[4]) is None  # arena full: not admitted
        assert srv.stats()["arena_used"] == 1 * MIB
        srv.release(tickets[0])
        r4 = srv.wait(tickets[4], timeout_s=30)
        assert r4.status == 0 and np.array_equal(_out(srv, tickets[4], r4, w), reqs[4][4])
        srv.release(tickets[1])
        r5 = srv.wait(tickets[5], timeout_s=30)
        assert r5.status == 0 and np.array_equal(_out(srv, tickets[5], r5, w), reqs[5][4])
        for t in tickets[2:]:
            srv.release(t)
        st = srv.stats()
        assert st["arena_peak"] <= 1 * MIB and st["arena_used"] == 0

        # never admissible / unsupported / misaligned requests are refused at submit
        big = _requests(oracle, [(300_000, 4, "b", 0.5)], seed0=300)[0]
        with pytest.raises(cs.CsError) as e:
            srv.submit(big[0], big[1], 300_000, 4)
        assert e.value.status == cs._lib.ERR_ADMISSION
        d_in, d_mask = reqs[0][0], reqs[0][1]
        with pytest.raises(cs.CsError) as e:
            srv.submit(d_in.data_ptr() + 4, d_mask, 1000, 4)
        assert e.value.status == cs._lib.ERR_MISALIGNED
        with pytest.raises(cs.CsError) as e:
            srv.submit(d_in, d_mask, 1000, 3)
        assert e.value.status == cs._lib.ERR_INVALID_VALUE
        assert srv.stats()["rejected"] == 3


def test_server_shrinks_reservation(cuda, oracle):
    """A completed request keeps only count * elem_bytes of the arena."""
    import gpu_compressstore2_b200 as cs

    reqs = _requests(oracle, [(1_000_000, 4, "b", 0.001)], seed0=400)
    with cs.Server(out_budget_bytes=8 * MIB) as srv:
        d_in, d_mask, n, w, exp = reqs[0]
        t = srv.submit(d_in, d_mask, n, w)
        r = srv.wait(t, timeout_s=30)
        assert r.status == 0 and r.count == len(exp)
        used = srv.stats()["arena_used"]
        assert used == ((len(exp) * 4 + 255) // 256) * 256
        srv.release(t)


def test_server_limits(cuda):
    import torch
    import gpu_compressstore2_b200 as cs

    with cs.Server(out_budget_bytes=4 * MIB, max_batch_elems=1 << 16) as srv:
        x = torch.zeros(1 << 17, dtype=torch.int32, device="cuda")
        m = torch.zeros(1 << 12, dtype=torch.int32, device="cuda")
        with pytest.raises(cs.CsError) as e:
            srv.submit(x, m, (1 << 16) + 1, 4)
        assert e.value.status == cs._lib.ERR_NOT_SUPPORTED
        with pytest.raises(cs.CsError):
            srv.release(12345)
        with pytest.raises(cs.CsError):
            srv.poll(12345)
    with pytest.raises(cs.CsError):
        cs.Server(mode=7)


def test_server_next_completion_order(cuda, oracle):
    import gpu_compressstore2_b200 as cs

    reqs = _requests(oracle, SPECS[:12], seed0=500)
    with cs.Server(out_budget_bytes=64 * MIB, max_batch=4, slots=3) as srv:
        want = {}
        for d_in, d_mask, n, w, exp in reqs:
            want[srv.submit(d_in, d_mask, n, w)] = (w, exp)
        seen = set()
        while len(seen) < len(want):
            got = srv.next(timeout_s=30)
            assert got is not None
            t, r = got
            assert t in want and t not in seen
            w, exp = want[t]
            assert r.status == 0 and np.array_equal(_out(srv, t, r, w), exp)
            srv.release(t)
            seen.add(t)
        assert srv.next(timeout_s=0.01) is None


@pytest.mark.parametrize("mode", ["batch", "per_call"])
def test_server_replay_poisson(cuda, oracle, mode):
    """The native load generator: Poisson arrivals over a device-resident pool."""
    import torch
    import gpu_compressstore2_b200 as cs

    rng = np.random.default_rng(7)
    pool_n = 1 << 24
    d_pool = torch.empty(pool_n, dtype=torch.int32, device="cuda")
    cs.gen_payload(d_pool, pool_n, seed=11)
    masks = []
    ps = [0.01, 0.3, 0.5, 0.99]
    for i, p in enumerate(ps):
        m = torch.empty(cs.mask_words(pool_n), dtype=torch.int32, device="cuda")
        cs.gen_mask_bernoulli(m, pool_n, p, seed=20 + i)
        masks.append(m)
    k = 200
    ns = np.exp(rng.uniform(np.log(2 ** 12), np.log(2 ** 20), k)).astype(np.int64)
    offs = (rng.integers(0, (pool_n - ns) // 128) * 128).astype(np.int64)
    which = rng.integers(0, len(ps), k)
    arrivals = np.cumsum(rng.exponential(20e3, k)).astype(np.int64)  # 50k requests/s offered
    reqs = [cs.Server.request(d_pool.data_ptr() + int(o) * 4, masks[int(j)].data_ptr() + int(o) // 8, int(n), 4)
            for n, o, j in zip(ns, offs, which)]
    m = cs.SERVE_BATCH if mode == "batch" else cs.SERVE_PER_CALL
    with cs.Server(out_budget_bytes=256 * MIB, mode=m, slots=3 if mode == "batch" else 1) as srv:
        res = srv.replay(reqs, arrivals)
        st = srv.stats()
    assert all(r.status == 0 for r in res)
    assert all(r.latency_ns > 0 for r in res)
    pool_h = d_pool.cpu().numpy().view(np.uint32)
    masks_h = [mm.cpu().numpy().view(np.uint32) for mm in masks]
    for r, n, o, j in zip(res, ns, offs, which):
        mw = masks_h[int(j)][int(o) // 32: int(o) // 32 + (int(n) + 31) // 32]
        assert r.count == oracle.count(mw, int(n)), (n, o, j)
    assert st["completed"] == k and st["arena_used"] == 0

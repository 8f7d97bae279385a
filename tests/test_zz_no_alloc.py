"""GPU test of compressstore_noalloc, the entry point for callers that may not allocate
device memory (their memory is owned by a host application's pool, or an allocation's
implicit synchronisation is unacceptable): its scratch is a fixed array inside the library.
Called through the C ABI, its results must equal the plain compressstore's, on two calls in
a row. This file is collected last so a failure here stops a -x run only after every
other test has run."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu

CASES = [(1_000_003, 4, 0.5), (3_000_001, 8, 0.01), (777_777, 1, 0.9), (123_456, 2, 0.3)]


def _inputs(cs, torch, n, w, p, seed):
    dt = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[w]
    d_in = torch.empty(n, dtype=dt, device="cuda")
    cs.gen_payload(d_in, n, seed)
    d_mask = torch.empty((n + 31) // 32, dtype=torch.int32, device="cuda")
    cs.gen_mask_bernoulli(d_mask, n, p, seed + 1)
    return d_in, d_mask, dt


def test_noalloc_matches_plain_call_on_two_calls(cuda):
    import torch
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        for i, (n, w, p) in enumerate(CASES):
            d_in, d_mask, dt = _inputs(cs, torch, n, w, p, 1000 * call + 10 * i)
            out_a = torch.full((n,), -1, dtype=dt, device="cuda")
            out_b = torch.full((n,), -1, dtype=dt, device="cuda")
            cnt = torch.full((2,), -1, dtype=torch.int64, device="cuda")
            st = L.compressstore_noalloc(d_in.data_ptr(), d_mask.data_ptr(), out_a.data_ptr(), n, w,
                                         cnt[0:1].data_ptr(), stream)
            assert st == 0, L.cs_status_string(st)
            st = L.compressstore(d_in.data_ptr(), d_mask.data_ptr(), out_b.data_ptr(), n, w, cnt[1:2].data_ptr(),
                                 stream)
            assert st == 0, L.cs_status_string(st)
            torch.cuda.synchronize()
            k = int(cnt[1].item())
            assert int(cnt[0].item()) == k, (call, n, w)
            assert torch.equal(out_a, out_b), (call, n, w)  # bit-exact, including the untouched tail
            assert k == int(((d_mask.view(-1, 1) >> torch.arange(32, device="cuda", dtype=torch.int32)) & 1)
                            .view(-1)[:n].sum().item())


def test_noalloc_at_its_maximum_column_length(cuda):
    """The largest column the fixed scratch serves (CS_NOALLOC_MAX_N = 2^30 one-byte
    elements) works and equals the plain call; one element more is refused."""
    import torch
    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    stream = torch.cuda.current_stream().cuda_stream
    n, w = 1 << 30, 1
    d_in, d_mask, dt = _inputs(cs, torch, n, w, 0.5, 4242)
    out_a = torch.full((n,), -1, dtype=dt, device="cuda")
    cnt = torch.full((2,), -1, dtype=torch.int64, device="cuda")
    st = L.compressstore_noalloc(d_in.data_ptr(), d_mask.data_ptr(), out_a.data_ptr(), n, w, cnt[0:1].data_ptr(), stream)
    assert st == 0, L.cs_status_string(st)
    out_b = torch.full((n,), -1, dtype=dt, device="cuda")
    st = L.compressstore(d_in.data_ptr(), d_mask.data_ptr(), out_b.data_ptr(), n, w, cnt[1:2].data_ptr(), stream)
    assert st == 0, L.cs_status_string(st)
    torch.cuda.synchronize()
    assert int(cnt[0].item()) == int(cnt[1].item())
    assert torch.equal(out_a, out_b)
    del out_b
    st = L.compressstore_noalloc(d_in.data_ptr(), d_mask.data_ptr(), out_a.data_ptr(), n + 1, w, cnt[0:1].data_ptr(),
                                 stream)
    assert st == cs._lib.ERR_NOT_SUPPORTED
    del d_in, d_mask, out_a
    torch.cuda.empty_cache()

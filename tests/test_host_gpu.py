"""GPU tests of the host-buffer entry point (compressstore_host): pinned and pageable host
buffers, single and multi-piece columns, against the CPU oracle."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,n,p", [(4, 1000, 0.5), (8, 5_000_003, 0.3), (1, 70_000_123, 0.5), (2, 40_000_000, 0.02),
                                   (4, 9_000_000, 0.0)])
@pytest.mark.parametrize("pinned", [True, False])
def test_host_buffers(cuda, oracle, w, n, p, pinned):
    import torch
    import gpu_compressstore2_b200 as cs

    payload = oracle.payload(n, w, 31 + w)
    mask = oracle.mask_bernoulli(n, p, 37)
    exp = oracle.compact(payload, mask, n, threads=8)
    sdt = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[w]
    h_in = torch.from_numpy(payload.view({1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}[w]))
    h_mask = torch.from_numpy(mask.view(np.int32))
    h_out = torch.full((n + 16,), -1, dtype=sdt)
    if pinned:
        h_in, h_mask, h_out = h_in.pin_memory(), h_mask.pin_memory(), h_out.pin_memory()
    k = cs.compressstore_host(h_in, h_mask, h_out, n)
    assert k == len(exp)
    got = h_out.numpy().view(payload.dtype)
    assert np.array_equal(got[:k], exp)
    assert np.all(got[k:].view(np.uint8) == 0xFF)  # nothing written past the count
    # numpy buffers work too
    out2 = np.zeros(n, dtype=payload.dtype)
    assert cs.compressstore_host(payload, mask, out2, n) == k
    assert np.array_equal(out2[:k], exp)


def test_scratch_release_and_reuse(cuda, oracle):
    """compressstore_release frees a stream's library-owned scratch and compressstore_host_release
    the host path's state; later calls set them up again and still match the oracle."""
    import torch
    import gpu_compressstore2_b200 as cs

    n, w = 300_001, 4
    payload = oracle.payload(n, w, 5)
    mask = oracle.mask_bernoulli(n, 0.4, 6)
    exp = oracle.compact(payload, mask, n)
    d_in = torch.from_numpy(payload.view(np.int32)).cuda()
    d_mask = torch.from_numpy(mask.view(np.int32)).cuda()
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    for _ in range(3):
        s = torch.cuda.Stream()
        d_out = torch.zeros(n, dtype=torch.int32, device="cuda")
        with torch.cuda.stream(s):
            cs.compressstore(d_in, d_mask, d_out, n, cnt, stream=s)
            cs.compressstore_check(stream=s)
            cs.compressstore_release(stream=s)
            cs.compressstore_release(stream=s)  # nothing left: a no-op
        s.synchronize()
        k = int(cnt.item())
        assert k == len(exp) and np.array_equal(d_out.cpu().numpy().view(np.uint32)[:k], exp)
        del s
    for _ in range(2):
        out = np.zeros(n, dtype=payload.dtype)
        assert cs.compressstore_host(payload, mask, out, n) == len(exp)
        assert np.array_equal(out[:len(exp)], exp)
        cs._lib.check(cs.lib().compressstore_host_release(), "compressstore_host_release")

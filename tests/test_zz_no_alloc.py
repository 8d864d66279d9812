"""sk_radix_argsort_noalloc, the argsort whose workspace is the library's own fixed device array.

It is compared with sk_radix_argsort_device (caller workspace) on the same device keys, on two
calls in a row: the second call finds the scratch as the first one left it, so it checks that
the sort leaves its counters and accumulators ready for the next call. The file sorts last so
that it also runs after every other GPU test in one session; it passes alone too.
"""
from __future__ import annotations

import numpy as np
import pytest

import splatkit_b200 as sk


def _device_sort(torch, k, count, capacity, bits, noalloc):
    dev = k.device
    order = torch.full((capacity,), -1, dtype=torch.int32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    if noalloc:
        sk.radix_argsort_noalloc(k.data_ptr(), count.data_ptr(), capacity, bits, order.data_ptr(),
                                 err.data_ptr(), stream)
    else:
        ws = torch.zeros(sk.sort_workspace_bytes(capacity), dtype=torch.uint8, device=dev)
        sk.radix_argsort_device(k.data_ptr(), count.data_ptr(), capacity, bits, order.data_ptr(),
                                ws.data_ptr(), ws.numel(), err.data_ptr(), stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return order.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("bits,n,capacity", [
    (32, 300_001, 300_001),
    (16, 1 << 20, 1 << 20),            # the largest capacity the scratch holds
    (32, 77_777, 100_000),             # count below capacity
])
def test_noalloc_sort_matches_workspace_sort_twice(cuda_device, bits, n, capacity):
    import torch

    rng = np.random.default_rng(1000 + bits + n)
    keys = rng.integers(0, 1 << bits, size=n, dtype=np.uint64).astype(np.uint32)
    keys[rng.integers(0, n, size=n // 8)] = keys[0]  # many ties: stability matters
    dev = torch.device("cuda", cuda_device)
    k = torch.from_numpy(keys.view(np.int32).copy()).to(dev)
    count = torch.tensor([n], dtype=torch.int32, device=dev)
    want = np.argsort(keys, kind="stable").astype(np.int32)

    expected = _device_sort(torch, k, count, capacity, bits, noalloc=False)
    assert np.array_equal(expected[:n], want)
    for call in range(2):
        got = _device_sort(torch, k, count, capacity, bits, noalloc=True)
        assert np.array_equal(got[:n], expected[:n]), f"call {call}"
        assert np.all(got[n:] == -1), f"call {call} wrote past the count"


@pytest.mark.gpu
def test_noalloc_sort_after_a_different_sort_and_beyond_its_limit(cuda_device):
    import torch

    dev = torch.device("cuda", cuda_device)
    rng = np.random.default_rng(7)
    # a small 16-bit sort right after a large 32-bit one reuses the same scratch
    for bits, n in ((32, 500_000), (16, 5_000), (32, 1)):
        keys = rng.integers(0, 1 << bits, size=n, dtype=np.uint64).astype(np.uint32)
        k = torch.from_numpy(keys.view(np.int32).copy()).to(dev)
        count = torch.tensor([n], dtype=torch.int32, device=dev)
        got = _device_sort(torch, k, count, n, bits, noalloc=True)
        assert np.array_equal(got, np.argsort(keys, kind="stable").astype(np.int32))

    # one key more than the limit is refused before anything is enqueued
    k = torch.zeros(1, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    order = torch.zeros(1, dtype=torch.int32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    with pytest.raises(sk.SplatError) as info:
        sk.radix_argsort_noalloc(k.data_ptr(), count.data_ptr(), sk.NOALLOC_SORT_MAX_KEYS + 1, 32,
                                 order.data_ptr(), err.data_ptr(),
                                 torch.cuda.current_stream().cuda_stream)
    assert info.value.status == sk.SK_E_LIMIT
    torch.cuda.synchronize()
    assert int(err.item()) == 0

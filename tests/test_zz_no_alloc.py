"""The allocation-free u32 device sort (ts_sort_dev_noalloc_u32).

It exists for callers that cannot call cudaMalloc (a framework that owns all
device memory, a latency-critical path that cannot take an allocation's
synchronisation, a fixed memory budget). Its output must equal the ordinary
device sort's (ts_sort_dev_u32) bit for bit, call after call, although every
call reuses the same fixed scratch array; sizes above its maximum are refused.
This file is collected last so that a failure here stops no other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 22
TS_ERR_TOO_LARGE = 8


def _entry(L):
    f = L.ts_sort_dev_noalloc_u32
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def test_noalloc_matches_the_device_sort_on_consecutive_calls():
    import torch

    import turbosort_b200 as ts

    L = ts.lib()
    noalloc = _entry(L)
    ctx = ts.Context(0)
    stream = torch.cuda.current_stream().cuda_stream
    # the first two calls may load the library's device code (lazy loading)
    # into memory; from the third on, free device memory must not move
    sizes = [5_000, 3_000_017, 3_000_017, 5_000, MAX_KEYS]  # small tier, LSD passes, the maximum
    for call, n in enumerate(sizes):
        rng = np.random.default_rng(100 + call)
        a = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
        if call == 4:
            a &= np.uint32(0xFFFF)  # digits that never vary: skipped passes
        mine = torch.from_numpy(a.view(np.int32)).cuda()
        theirs = mine.clone()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        assert noalloc(mine.data_ptr(), n, stream) == 0
        free_after = torch.cuda.mem_get_info()[0]
        if call >= 2:
            assert free_after == free_before, "the allocation-free sort changed free device memory"
        assert L.ts_sort_dev_u32(ctx.handle, theirs.data_ptr(), n) == 0
        ctx.synchronize()
        torch.cuda.synchronize()
        assert torch.equal(mine, theirs), f"call {call}: outputs differ"
        assert np.all(np.diff(mine.cpu().numpy().view(np.uint32).astype(np.int64)) >= 0)


def test_noalloc_unaligned_keys_match_the_oracle():
    """Keys that start 4 bytes past a 16-byte boundary take the unvectorised
    loads of the scan, histogram and finishing kernels on the shared scratch;
    the result must still be the oracle's sort, bit for bit, twice in a row."""
    import torch

    import turbosort_b200 as ts
    from oracle import oracle as O

    noalloc = _entry(ts.lib())
    stream = torch.cuda.current_stream().cuda_stream
    for call, n in enumerate([1_000_003, 77_777]):
        rng = np.random.default_rng(900 + call)
        a = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
        buf = torch.zeros(n + 4, dtype=torch.int32, device="cuda")
        buf[1:n + 1] = torch.from_numpy(a.view(np.int32)).cuda()
        torch.cuda.synchronize()
        assert (buf.data_ptr() + 4) % 16 != 0
        assert noalloc(buf.data_ptr() + 4, n, stream) == 0
        got = buf[1:n + 1].cpu().numpy().view(np.uint32)
        assert got.tobytes() == O.sort(a).tobytes(), f"call {call}: differs from the oracle"
        assert int(buf[0]) == 0 and int(buf[n + 1:].abs().sum()) == 0, "wrote outside the keys"


def test_noalloc_refuses_more_than_its_maximum():
    import torch

    import turbosort_b200 as ts

    noalloc = _entry(ts.lib())
    x = torch.zeros(16, dtype=torch.int32, device="cuda")
    assert noalloc(x.data_ptr(), MAX_KEYS + 1, None) == TS_ERR_TOO_LARGE
    assert int(x.abs().sum()) == 0  # refused before touching anything

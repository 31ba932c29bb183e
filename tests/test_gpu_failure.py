"""Failure detection on the device without a fault: a bounded wait runs out.

The test hook ts_ctx_test_stall_lookback makes tile 0 of the next sort's
first scatter pass withhold its look-back entry, so every later tile's wait
on it gives up after a short limit. The call must return TS_ERR_TIMEOUT
quickly (the kernels end by themselves), keep every write inside the keys and
the caller's scratch buffer (guard words around both stay untouched), and
leave the context able to sort correctly right after."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TS_ERR_TIMEOUT = 4
GUARD = 4096
SENTINEL = 0x5A5A5A5A


@pytest.mark.parametrize("what", ["sort", "order"])
def test_a_withheld_lookback_entry_times_out_cleanly(what):
    import torch

    import turbosort_b200 as ts
    from oracle import oracle as O

    L = ts.lib()
    ctx = ts.Context(0)
    n = 3_000_017
    a = np.random.default_rng(41).integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    data = torch.full((n + 2 * GUARD,), SENTINEL, dtype=torch.int32, device="cuda")
    buf = torch.full((n + 2 * GUARD,), SENTINEL, dtype=torch.int32, device="cuda")
    order = torch.full((n + 2 * GUARD,), SENTINEL, dtype=torch.int32, device="cuda")
    data[GUARD:GUARD + n] = torch.from_numpy(a.view(np.int32)).cuda()
    torch.cuda.synchronize()
    dp, bp, op = (t.data_ptr() + 4 * GUARD for t in (data, buf, order))

    def call():
        if what == "sort":
            return L.ts_sort_dev_with_buffer_u32(ctx.handle, dp, n, bp, n)
        return L.ts_sort_keys_order_dev_u32(ctx.handle, dp, n, op)

    assert L.ts_ctx_test_stall_lookback(ctx.handle, 2048) == 0
    t0 = time.perf_counter()
    st = call()
    if st == 0:
        st = L.ts_ctx_synchronize(ctx.handle)
    elapsed = time.perf_counter() - t0
    assert st == TS_ERR_TIMEOUT, f"status {st}"
    assert elapsed < 5.0, f"the timed-out sort took {elapsed:.2f} s"
    torch.cuda.synchronize()
    for t in (data, buf, order):
        h = t.cpu().numpy()
        assert np.all(h[:GUARD] == SENTINEL) and np.all(h[GUARD + n:] == SENTINEL), "wrote outside the buffers"

    # the same context, armed no more, sorts correctly
    data[GUARD:GUARD + n] = torch.from_numpy(a.view(np.int32)).cuda()
    torch.cuda.synchronize()
    assert call() == 0 and L.ts_ctx_synchronize(ctx.handle) == 0
    if what == "sort":
        got = data[GUARD:GUARD + n].cpu().numpy().view(np.uint32)
        assert got.tobytes() == O.sort(a).tobytes()
    else:
        got = order[GUARD:GUARD + n].cpu().numpy().view(np.uint32)
        assert got.tobytes() == O.sort_by_key_order(a).tobytes()

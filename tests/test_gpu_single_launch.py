"""The single-launch LSD (k_lsd_coop): a keys-only sort of 2- or 4-byte keys
whose tiles fit one wave runs in one cooperative launch with bounded grid
barriers. Its output is the oracle's (src/dispatch.rs:31) byte for byte for
every 2- and 4-byte key type, across its tile sizes, at the edge of its
capacity (one key more takes the multi-launch LSD), for presorted and
descending input, an odd and an even number of live passes, duplicates and
constant input; repeated calls replay it from a CUDA graph; and a grid
barrier that nobody completes times out cleanly."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KINDS = [np.uint16, np.int16, np.uint32, np.int32, np.float32]
TS_ERR_TIMEOUT = 4


@pytest.fixture(scope="module")
def env():
    import torch

    import turbosort_b200 as ts
    from oracle import oracle as O

    ctx = ts.Context(0)
    return torch, ts, O, ctx


def _keys(t, n, seed):
    rng = np.random.default_rng(seed)
    w = rng.integers(0, 2**32, size=n, dtype=np.uint64)
    a = w.astype({2: np.uint16, 4: np.uint32}[np.dtype(t).itemsize]).view(t).copy()
    if np.dtype(t).kind == "f":
        a[::89] = np.nan
        a[1::89] = -np.nan
        a[2::97] = 0.0
        a[3::97] = -0.0
        a[4::101] = np.inf
        a[5::101] = -np.inf
    return a


def _tdt(torch, dt):
    return {"u2": torch.uint16, "i2": torch.int16, "u4": torch.uint32, "i4": torch.int32,
            "f4": torch.float32}[dt.kind + str(dt.itemsize)]


def _sort(env, a):
    torch, ts, O, ctx = env
    iview = {2: np.int16, 4: np.int32}[a.dtype.itemsize]
    d = torch.from_numpy(a.view(iview).copy()).cuda()
    ts.sort(d.view(_tdt(torch, a.dtype)), ctx)
    ctx.synchronize()
    return d.cpu().numpy().view(a.dtype), ctx.last_sort_info()


def _capacity(ts):
    import torch

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    return min(2 * sms, 512) * 512 * 11


@pytest.mark.parametrize("t", KINDS)
def test_matches_the_oracle_across_tile_sizes(env, t):
    """Lengths that take the 7- and 11-key-a-thread tiles, and ragged ones."""
    _, ts, O, _ = env
    cap = _capacity(ts)
    for i, n in enumerate([4_097, 70_001, 1 << 20, (1 << 20) + 12_345, 1_500_007, cap]):
        a = _keys(t, n, 31 * i + np.dtype(t).itemsize)
        got, info = _sort(env, a)
        assert got.tobytes() == O.sort(a).tobytes(), f"{np.dtype(t)} n={n}"
        assert info["tier"] == 4 and info["passes"] == np.dtype(t).itemsize, info


def test_one_key_past_capacity_takes_the_multi_launch_sort(env):
    _, ts, O, _ = env
    n = _capacity(ts) + 1
    a = _keys(np.uint32, n, 5)
    got, info = _sort(env, a)
    assert got.tobytes() == O.sort(a).tobytes()
    assert info["tier"] == 3, info


@pytest.mark.parametrize("n", [5_000, 1 << 20])
def test_plan_shapes(env, n):
    """Presorted (no pass), descending (reversed in place), 3 live passes (odd:
    the copy back), 2 live passes, duplicates, constant input."""
    _, _, O, _ = env
    rng = np.random.default_rng(n)
    a = _keys(np.uint32, n, 9)
    s = np.sort(a)
    got, info = _sort(env, s)
    assert got.tobytes() == s.tobytes() and info["tier"] == 4 and info["mode"] == 1 and info["passes"] == 0, info
    got, info = _sort(env, s[::-1].copy())
    assert got.tobytes() == s.tobytes() and info["mode"] == 2, info
    d = s[::-1].copy()
    d[n // 3] = d[n // 3 + 1]  # descending with one tie: not strictly reversed input, still mode 2
    got, info = _sort(env, d)
    assert got.tobytes() == O.sort(d).tobytes()
    for bits, passes in [(24, 3), (16, 2), (8, 1)]:
        b = rng.integers(0, 1 << bits, size=n, dtype=np.uint32)
        got, info = _sort(env, b)
        assert got.tobytes() == O.sort(b).tobytes() and info["passes"] == passes, (bits, info)
    c = rng.integers(0, 5, size=n, dtype=np.uint32) * np.uint32(0x01010101)
    got, _ = _sort(env, c)
    assert got.tobytes() == O.sort(c).tobytes()
    e = np.full(n, 0xDEADBEEF, dtype=np.uint32)
    got, info = _sort(env, e)
    assert got.tobytes() == e.tobytes() and info["passes"] == 0, info


def test_same_output_with_the_multi_launch_sort(env):
    torch, ts, O, ctx = env
    a = _keys(np.float32, 777_777, 3)
    want, info = _sort(env, a)
    assert info["tier"] == 4
    ctx.set_single_launch(False)
    try:
        got, info = _sort(env, a)
        assert info["tier"] == 3 and got.tobytes() == want.tobytes()
    finally:
        ctx.set_single_launch(True)


@pytest.mark.parametrize("t", [np.uint16, np.uint32])
def test_unaligned_keys(env, t):
    """Keys one element past a 16-byte boundary take the scalar tile loads
    and stores; the caller's buffer serves as the scratch."""
    torch, ts, O, ctx = env
    L = ts.lib()
    n = 300_007
    a = _keys(t, n, 11)
    iview = {2: np.int16, 4: np.int32}[a.dtype.itemsize]
    big = torch.from_numpy(np.concatenate([np.zeros(1, a.dtype), a]).view(iview).copy()).cuda()
    buf = torch.empty(n + 1, dtype=big.dtype, device="cuda")
    w = a.dtype.itemsize
    fn = getattr(L, f"ts_sort_dev_with_buffer_u{8 * w}")
    assert fn(ctx.handle, big.data_ptr() + w, n, buf.data_ptr() + w, n) == 0
    assert L.ts_ctx_synchronize(ctx.handle) == 0
    assert ctx.last_sort_info()["tier"] == 4
    got = big.cpu().numpy().view(a.dtype)
    assert got[0] == 0 and got[1:].tobytes() == O.sort(a).tobytes()


def test_graph_replay(env):
    """Repeated calls with the same pointers replay a captured graph."""
    torch, ts, O, _ = env
    ctx = ts.Context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    n = 600_001
    d = torch.empty(n, dtype=torch.int32, device="cuda")
    for r in range(4):
        a = _keys(np.int32, n, 100 + r)
        d.copy_(torch.from_numpy(a.view(np.int32)))
        ts.sort(d, ctx)
        torch.cuda.synchronize()
        assert d.cpu().numpy().tobytes() == O.sort(a).tobytes(), f"call {r}"
        assert ctx.last_sort_info()["tier"] == 4


def test_a_barrier_nobody_completes_times_out_cleanly(env):
    """CTA 0 withholds its arrival at the first grid barrier (test hook): every
    wait gives up after the limit, the call reports TS_ERR_TIMEOUT within
    seconds, nothing outside the keys and the scratch is written, and the
    context sorts correctly right after."""
    torch, ts, O, _ = env
    L = ts.lib()
    ctx = ts.Context(0)
    n, guard, sentinel = 100_003, 4096, 0x5A5A5A5A
    a = _keys(np.uint32, n, 77)
    data = torch.full((n + 2 * guard,), sentinel, dtype=torch.int32, device="cuda")
    buf = torch.full((n + 2 * guard,), sentinel, dtype=torch.int32, device="cuda")
    data[guard:guard + n] = torch.from_numpy(a.view(np.int32)).cuda()
    torch.cuda.synchronize()
    dp, bp = data.data_ptr() + 4 * guard, buf.data_ptr() + 4 * guard
    assert L.ts_ctx_test_stall_lookback(ctx.handle, 4096) == 0
    t0 = time.perf_counter()
    st = L.ts_sort_dev_with_buffer_u32(ctx.handle, dp, n, bp, n)
    if st == 0:
        st = L.ts_ctx_synchronize(ctx.handle)
    assert st == TS_ERR_TIMEOUT, f"status {st}"
    assert time.perf_counter() - t0 < 5.0
    torch.cuda.synchronize()
    for t in (data, buf):
        h = t.cpu().numpy()
        assert np.all(h[:guard] == sentinel) and np.all(h[guard + n:] == sentinel)
    # nothing passed the first barrier, so the keys are as they were
    assert data[guard:guard + n].cpu().numpy().view(np.uint32).tobytes() == a.tobytes()
    assert L.ts_sort_dev_with_buffer_u32(ctx.handle, dp, n, bp, n) == 0 and L.ts_ctx_synchronize(ctx.handle) == 0
    assert data[guard:guard + n].cpu().numpy().view(np.uint32).tobytes() == O.sort(a).tobytes()

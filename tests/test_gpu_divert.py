"""Diverting on the device (src/radix/divert.rs:38-81; src/radix/mod.rs:240-270):
8-byte keys whose top digits already split them into short runs get passes
only for those digits, and the runs are finished directly. Every output is
compared byte for byte with the oracle's sort (which diverts the same way on
the CPU); the plan the device chose is read back through ts_ctx_last_sort_info.

Shapes: random u64/i64/f64 (runs of one or two keys, finished by threads);
keys whose top four bytes are one repeated random byte (256 prefixes: long
runs, finished a CTA each on chip, and beyond shared memory through the CTA
LSD); run lengths around the crate's SHORT_RUN of 16; and inputs that must
not divert (top digits that barely split the keys)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    import turbosort_b200 as ts
    from oracle import oracle as O

    ctx = ts.Context(0)
    return torch, ts, O, ctx


def _sort_dev(env, a):
    torch, ts, O, ctx = env
    dev = torch.from_numpy(a.view(np.int64)).cuda()
    tdt = {np.dtype(np.uint64): torch.uint64, np.dtype(np.int64): torch.int64,
           np.dtype(np.float64): torch.float64}[a.dtype]
    ts.sort(dev.view(tdt), ctx)
    ctx.synchronize()
    info = ctx.last_sort_info()
    return dev.cpu().numpy().view(a.dtype), info


def _words(n, seed):
    return np.random.default_rng(seed).integers(0, 2**64, size=n, dtype=np.uint64)


@pytest.mark.parametrize("lg", [13, 16, 20, 23])
def test_random_u64_diverts_and_equals_the_oracle(env, lg):
    _, _, O, _ = env
    a = _words(1 << lg, lg)
    got, info = _sort_dev(env, a)
    assert got.tobytes() == O.sort(a).tobytes()
    assert info["tier"] == 3 and info["divert_shift"] > 0, info
    # the passes that ran are the top live digits only
    assert info["pass_digit"] == list(range(info["divert_shift"] // 8, 8)), info


@pytest.mark.parametrize("t", [np.int64, np.float64])
def test_signed_and_float_keys_divert(env, t):
    _, _, O, _ = env
    a = _words(1 << 21, 5).view(t).copy()
    if t is np.float64:  # NaN of both signs, +-0 and +-inf among random bit patterns
        a[::97] = np.nan
        a[1::97] = -np.nan
        a[2::101] = 0.0
        a[3::101] = -0.0
        a[4::103] = np.inf
        a[5::103] = -np.inf
    got, info = _sort_dev(env, a)
    assert got.tobytes() == O.sort(a).tobytes()
    assert info["divert_shift"] > 0, info


@pytest.mark.parametrize("lg", [20, 23])
def test_long_runs_of_a_shared_prefix(env, lg):
    """Top four bytes one repeated byte: every top digit looks uniform, so the
    sort diverts, yet only 256 prefixes exist: runs of 2^lg / 256 keys (4096
    on chip at 2^20; 32768, beyond shared memory, at 2^23)."""
    _, _, O, _ = env
    n = 1 << lg
    w = _words(n, 100 + lg)
    b = (w >> np.uint64(56)) * np.uint64(0x0101010100000000)
    a = b | (w & np.uint64(0xFFFFFFFF))
    got, info = _sort_dev(env, a)
    assert info["divert_shift"] > 0, info
    assert got.tobytes() == O.sort(a).tobytes()


def test_run_lengths_around_the_short_run_limit(env):
    _, _, O, _ = env
    rng = np.random.default_rng(8)
    lengths = rng.integers(1, 41, size=60000)
    prefixes = rng.choice(np.arange(1 << 24, dtype=np.uint64), size=lengths.size, replace=False)
    pre = np.repeat(prefixes, lengths)
    a = (pre << np.uint64(40)) | (rng.integers(0, 2**40, size=pre.size, dtype=np.uint64))
    rng.shuffle(a)
    got, info = _sort_dev(env, a)
    assert info["divert_shift"] == 40, info
    assert got.tobytes() == O.sort(a).tobytes()


def test_no_divert_when_the_top_digits_barely_split(env):
    """Keys confined to 16 low bits and a heavily skewed top byte: no credit."""
    _, _, O, _ = env
    rng = np.random.default_rng(9)
    a = _words(1 << 20, 9) & np.uint64(0xFFFF)
    a[rng.random(a.size) < 0.001] |= np.uint64(1 << 63)
    got, info = _sort_dev(env, a)
    assert info["divert_shift"] == 0, info
    assert got.tobytes() == O.sort(a).tobytes()


def test_host_slice_and_repeated_calls(env):
    """The host entry point and the captured-graph replay of a repeated
    device call divert the same way."""
    torch, ts, O, ctx = env
    a = _words(3 << 20, 11)
    want = O.sort(a)
    h = a.copy()
    ts.sort(h, ctx)
    assert h.tobytes() == want.tobytes()
    dev = torch.empty(a.size, dtype=torch.int64, device="cuda")
    for _ in range(4):
        dev.copy_(torch.from_numpy(a.view(np.int64)))
        ts.sort(dev.view(torch.uint64), ctx)
        ctx.synchronize()
        assert dev.cpu().numpy().view(np.uint64).tobytes() == want.tobytes()

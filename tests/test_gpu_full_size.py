"""The plain sort at the benchmark's full sizes, checked byte for byte
against the oracle's sort of the same keys (the crate's algorithm restated;
tests/correctness.rs:6-8 defines the expected output as the sort by
to_radix_key, which is unique for these types).

2^28 keys each of u32, i32 and f32 (f32 with 1% NaN of both signs, 1% +-0.0
and 0.5% +-inf mixed in) and 2^27 u64 keys, each in three distributions:
full-entropy words, the AND of three words (low entropy), and keys confined
to 16 low bits (constant high digits, skipped). Keys sit on the device and are
sorted in place through the device entry point, as the benchmark does."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(k, d) for k in ("u32", "i32", "f32", "u64") for d in (0, 1, 2)]
DIST = ("full", "low_entropy", "range16")


@pytest.mark.parametrize("kind, dist", CASES, ids=[f"{k}-{DIST[d]}" for k, d in CASES])
def test_full_size_sort_equals_the_oracle(kind, dist):
    import torch

    import turbosort_b200 as ts
    from oracle import oracle as O
    from turbosort_b200 import workloads as W

    lg = 27 if kind == "u64" else 28
    n = 1 << lg
    host = W.scale(kind, dist, n, seed=0x5151 + 7 * dist)
    tdt = {"u32": torch.uint32, "i32": torch.int32, "f32": torch.float32, "u64": torch.uint64}[kind]
    idt = torch.int64 if kind == "u64" else torch.int32
    dev = torch.from_numpy(host.view(np.int64 if kind == "u64" else np.int32)).cuda()
    ts.sort(dev.view(tdt))
    torch.cuda.synchronize()
    got = dev.view(idt).cpu().numpy()
    del dev
    torch.cuda.empty_cache()
    want = O.sort_parallel(host)
    assert got.tobytes() == want.view(got.dtype).tobytes(), f"{kind} {DIST[dist]} 2^{lg}: differs from the oracle"

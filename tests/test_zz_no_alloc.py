"""og_segment_sum_noalloc through the C ABI: the allocation-free variant of og_segment_sum,
for callers that cannot allocate device memory when they call (their process has given the
free device memory to another allocator's pool, or allocation calls are not acceptable on
their path).  It must return what og_segment_sum returns, on two calls in a row (the second
call reuses the static scratch that the first one left filled), and refuse sizes beyond its
fixed scratch.  Collected last on purpose (file name), so a failure here stops a `-x` run
only after every other test has run."""
import ctypes

import numpy as np
import pytest

from omegagene_b200 import engine

pytestmark = pytest.mark.gpu


def _fns():
    L = engine.load_library()
    out = []
    for name in ("og_segment_sum", "og_segment_sum_noalloc"):
        f = getattr(L, name)
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                      ctypes.c_void_p, ctypes.c_void_p]
        out.append(f)
    return out


def _run(fn, vals, base, max_len):
    import torch
    out = torch.full((base.numel() - 1,), float("nan"), dtype=torch.float64, device="cuda")
    rc = fn(vals.data_ptr(), 1, base.data_ptr(), base.numel() - 1, max_len, out.data_ptr(),
            torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    sum_alloc, sum_noalloc = _fns()
    rng = np.random.default_rng(7)
    cases = []
    for lens in ([3, 5000, 0, 123457, 4096], [70000, 1, 9999]):
        vals = torch.tensor(rng.normal(size=sum(lens)) * 1e2, device="cuda")
        base = torch.tensor(np.concatenate([[0], np.cumsum(lens)]), dtype=torch.int32, device="cuda")
        cases.append((vals, base, max(lens)))
    for vals, base, max_len in cases:
        rc_a, ref = _run(sum_alloc, vals, base, max_len)
        assert rc_a == engine.OG_OK
        for _ in range(2):  # two calls in a row share (and overwrite) the static scratch
            rc, got = _run(sum_noalloc, vals, base, max_len)
            assert rc == engine.OG_OK
            np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-9)
            assert np.array_equal(got, ref)  # same kernels, same chunking: same bits


def test_noalloc_exact_fit_uses_the_whole_scratch():
    """16 segments x 4096 chunks fill the 65,536 scratch entries exactly; the last segment is
    long enough to write (and read back) the last entry.  Same bits as og_segment_sum, twice."""
    import torch
    sum_alloc, sum_noalloc = _fns()
    rng = np.random.default_rng(11)
    lens = [5, 0, 4096, 70000] + [3] * 11 + [4095 * 4096 + 17]  # ceil(len / 4096) = 4096 for the last
    max_len = 4096 * 4096
    vals = torch.tensor(rng.normal(size=sum(lens)), device="cuda")
    base = torch.tensor(np.concatenate([[0], np.cumsum(lens)]), dtype=torch.int32, device="cuda")
    rc_a, ref = _run(sum_alloc, vals, base, max_len)
    assert rc_a == engine.OG_OK
    for _ in range(2):
        rc, got = _run(sum_noalloc, vals, base, max_len)
        assert rc == engine.OG_OK
        assert np.array_equal(got, ref)
    last = vals[int(base[-2]):].cpu().numpy()
    np.testing.assert_allclose(got[-1], last.sum(), rtol=1e-10, atol=1e-8)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    sum_alloc, sum_noalloc = _fns()
    vals = torch.zeros(16, dtype=torch.float64, device="cuda")
    base = torch.zeros(70001, dtype=torch.int32, device="cuda")
    rc, _ = _run(sum_noalloc, vals, base, 4096)  # 70000 segments x 1 chunk > 65536 entries
    assert rc == engine.OG_ERR_CAPACITY
    # one more chunk than the scratch holds: 16 segments x 4097 chunks
    rc, _ = _run(sum_noalloc, vals, torch.zeros(17, dtype=torch.int32, device="cuda"), 4096 * 4096 + 1)
    assert rc == engine.OG_ERR_CAPACITY
    # the grid's segment limit: 65,535 segments fit, 65,536 (which the scratch alone would
    # hold) are refused by both entry points instead of failing at launch
    for fn in (sum_alloc, sum_noalloc):
        rc, out = _run(fn, vals, torch.zeros(65536, dtype=torch.int32, device="cuda"), 4096)
        assert rc == engine.OG_OK and np.array_equal(out, np.zeros(65535))
        rc, _ = _run(fn, vals, torch.zeros(65537, dtype=torch.int32, device="cuda"), 4096)
        assert rc == engine.OG_ERR_CAPACITY

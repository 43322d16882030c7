"""og_segment_sum (the engine's fixed-order reduction) through the C ABI."""
import ctypes

import numpy as np
import pytest

from omegagene_b200 import engine

pytestmark = pytest.mark.gpu


def _call(fn, vals, base, max_len, stride=1):
    import torch
    out = torch.zeros(len(base) - 1, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    rc = fn(ctypes.c_void_p(vals.data_ptr()), stride, ctypes.c_void_p(base.data_ptr()), len(base) - 1, max_len,
            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(st))
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


def test_segment_sum_matches_numpy_and_is_order_independent():
    import torch
    L = engine.load_library()
    fn = L.og_segment_sum
    fn.restype = ctypes.c_int
    rng = np.random.default_rng(0)
    lens = [1, 4095, 4096, 4097, 100000, 0, 777]
    vals = rng.normal(size=sum(lens)) * 1e3
    base = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    tv = torch.tensor(vals, device="cuda")
    tb = torch.tensor(base, device="cuda")
    rc, out = _call(fn, tv, tb, max(lens))
    assert rc == 0
    ref = np.array([vals[base[i]:base[i + 1]].sum() for i in range(len(lens))])
    np.testing.assert_allclose(out, ref, rtol=1e-12, atol=1e-9)
    # the same segment alone gives the same bits
    sub = torch.tensor(vals[base[4]:base[5]], device="cuda")
    rc2, out2 = _call(fn, sub, torch.tensor([0, lens[4]], dtype=torch.int32, device="cuda"), lens[4])
    assert rc2 == 0 and out2[0] == out[4]

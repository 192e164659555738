"""smmp_sur_predict_noalloc: the surrogate's forward pass for callers that
cannot allocate device memory when they need a prediction (for example while
a framework's caching allocator holds the device's memory budget, or inside a
loop where allocation is forbidden).  It runs on device buffers the caller
owns and keeps its intermediate activations in one fixed device array of the
library, so its results must equal smmp_sur_predict's; two calls in a row
check that nothing left in the shared array from the first call leaks into
the second.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(s, ang, stream=None):
    import torch
    from smmp._lib import check, lib
    a = torch.tensor(np.asarray(ang, dtype=np.float32), device="cuda")
    out = torch.full((a.shape[0],), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    h = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
    check(lib.smmp_sur_predict_noalloc(s._h, ctypes.c_void_p(a.data_ptr()), a.shape[0],
                                       ctypes.c_void_p(out.data_ptr()), h))
    if stream is None:
        torch.cuda.synchronize()
    else:
        stream.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("nang", [24, 365])
def test_noalloc_predict_equals_predict_on_two_calls(nang):
    from smmp.surrogate import Surrogate
    s = Surrogate(nang, seed=21)
    p, _ = s.params()
    s.set_params(p, np.array([-3.5, 7.25], dtype=np.float32))   # exercise the denormalisation
    rng = np.random.default_rng(nang)
    for n in (1200, 333):            # a large call, then a smaller one over its leftovers
        ang = rng.uniform(-np.pi, np.pi, (n, nang))
        want = s.predict(ang)
        got = _noalloc(s, ang)
        assert np.all(np.isfinite(got))
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-6)


def test_noalloc_rejects_more_rows_than_the_scratch_holds():
    from smmp import SmmpError
    from smmp.surrogate import Surrogate
    s = Surrogate(24, seed=3)
    with pytest.raises(SmmpError) as ei:
        _noalloc(s, np.zeros((5000, 24)))
    assert ei.value.status == 1
    assert "exceed the fixed scratch" in str(ei.value)


def test_noalloc_allocates_no_device_memory_on_a_side_stream():
    """After one warm-up call (which loads the kernels and looks up the
    array's address), a call on a non-default stream leaves the device's free
    memory unchanged and still equals predict()."""
    import torch
    from smmp._lib import check, lib
    from smmp.surrogate import Surrogate
    s = Surrogate(24, seed=5)
    rng = np.random.default_rng(9)
    ang = rng.uniform(-np.pi, np.pi, (700, 24))
    want = s.predict(ang)
    side = torch.cuda.Stream()
    _noalloc(s, ang, side)                       # warm-up
    a = torch.tensor(ang.astype(np.float32), device="cuda")
    out = torch.full((700,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    check(lib.smmp_sur_predict_noalloc(s._h, ctypes.c_void_p(a.data_ptr()), 700,
                                       ctypes.c_void_p(out.data_ptr()),
                                       ctypes.c_void_p(side.cuda_stream)))
    side.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=1e-6, atol=1e-6)

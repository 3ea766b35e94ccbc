"""hg_dot_noalloc: the dot product for callers that may not allocate device memory while they
run. Its partial sums live in a static device array instead of storage-allocated scratch; the
result must equal hg_dot's (same partition, same reduction order) on consecutive calls, which
share that array. Collected last on purpose, so that a run stopping at the first failure has
run every other test first."""
import ctypes

import numpy as np
import pytest

import hyteg_b200 as hg
from hyteg_b200 import _capi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_noalloc_dot_matches_dot_on_two_calls(dtype):
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    import torch

    L = 5
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    a = hg.P1Function("a", st, L, L, dtype=dtype)
    b = hg.P1Function("b", st, L, L, dtype=dtype)
    n = st.level_size(L)
    rng = np.random.default_rng(7)
    a.from_numpy(L, rng.uniform(-1, 1, n))
    b.from_numpy(L, rng.uniform(-1, 1, n))
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    prec = 8 if dtype == np.float64 else 4
    for flag in (hg.Inner, hg.All):
        ref = a.dotGlobal(b, L, flag)
        for k in range(2):  # two calls in a row share the static scratch
            _capi.call("hg_dot_noalloc", st.handle, ctypes.c_void_p(a.device_ptr(L)), ctypes.c_void_p(b.device_ptr(L)),
                       prec, L, flag, ctypes.c_void_p(out.data_ptr() + 8 * k))
        st.synchronize()
        got = out.cpu().numpy()
        assert abs(got[0] - ref) <= 1e-13 * abs(ref)
        assert abs(got[1] - ref) <= 1e-13 * abs(ref)


def test_noalloc_dot_rejects_bad_arguments():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 1, 1, 1, 2)
    rc = _capi.lib.hg_dot_noalloc(st.handle, None, None, 8, 2, hg.Inner, None)
    assert rc == _capi.HG_ERR_ARG

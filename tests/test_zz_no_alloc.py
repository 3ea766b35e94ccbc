"""hg_dot_noalloc: the dot product for callers that may not allocate device memory while they
run (for example a solve service that commits its device-memory budget at start-up). Its
partial sums live in a static device array instead of storage-allocated scratch. It runs the
same partial-sum and reduction kernels over the same block partition as hg_dot, so its result
must equal hg_dot's bit for bit, on consecutive calls that share that array, and after a call on
a larger level has left more partial sums in it. Collected last on purpose, so that a run
stopping at the first failure has run every other test first."""
import ctypes

import numpy as np
import pytest

import hyteg_b200 as hg
from hyteg_b200 import _capi

pytestmark = pytest.mark.gpu


def _noalloc(st, a, b, prec, L, flag, out_ptr):
    return _capi.lib.hg_dot_noalloc(st.handle, ctypes.c_void_p(a), ctypes.c_void_p(b), prec, L, flag,
                                    ctypes.c_void_p(out_ptr))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_noalloc_dot_matches_dot_on_two_calls(dtype):
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    import torch

    L = 5
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    prec = 8 if dtype == np.float64 else 4
    rng = np.random.default_rng(7)
    fa, fb = {}, {}
    for lv in (L, 3):
        fa[lv] = hg.P1Function("a%d" % lv, st, lv, lv, dtype=dtype)
        fb[lv] = hg.P1Function("b%d" % lv, st, lv, lv, dtype=dtype)
        n = st.level_size(lv)
        fa[lv].from_numpy(lv, rng.uniform(-1, 1, n))
        fb[lv].from_numpy(lv, rng.uniform(-1, 1, n))
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    # level 5 first (many partial sums), then level 3 (few): the second level must not read the
    # first level's stale slots
    for lv in (L, 3):
        for flag in (hg.Inner, hg.All):
            ref = fa[lv].dotGlobal(fb[lv], lv, flag)
            for k in range(2):  # two calls in a row share the static scratch
                rc = _noalloc(st, fa[lv].device_ptr(lv), fb[lv].device_ptr(lv), prec, lv, flag, out.data_ptr() + 8 * k)
                assert rc == _capi.HG_OK, _capi.lib.hg_last_error().decode()
            st.synchronize()
            got = out.cpu().numpy()
            assert got[0] == ref and got[1] == ref, (lv, flag, got, ref)
            out.zero_()


def test_noalloc_dot_rejects_bad_arguments():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    import torch

    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 1, 1, 1, 2)
    a = hg.P1Function("a", st, 2, 2)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = a.device_ptr(2)
    assert _capi.lib.hg_dot_noalloc(st.handle, None, None, 8, 2, hg.Inner, None) == _capi.HG_ERR_ARG
    assert _noalloc(st, p, p, 2, 2, hg.Inner, out.data_ptr()) == _capi.HG_ERR_ARG      # precision
    assert "precision" in _capi.lib.hg_last_error().decode()
    assert _noalloc(st, p, p, 8, 3, hg.Inner, out.data_ptr()) == _capi.HG_ERR_ARG      # level > max level
    assert _noalloc(st, p, p, 8, -1, hg.Inner, out.data_ptr()) == _capi.HG_ERR_ARG
    assert "level" in _capi.lib.hg_last_error().decode()


def test_noalloc_dot_rejects_levels_beyond_its_scratch():
    """3,072 macro-cells at level 5 need about 89,000 partial sums, more than the 65,536 of the
    static array: the call is rejected before any launch, and the message names hg_dot."""
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    import torch

    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 8, 8, 8, 5)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    # the buffers are never read: the size check comes first
    rc = _noalloc(st, out.data_ptr(), out.data_ptr(), 8, 5, hg.Inner, out.data_ptr())
    assert rc == _capi.HG_ERR_ARG
    msg = _capi.lib.hg_last_error().decode()
    assert "hg_dot_noalloc" in msg and "use hg_dot" in msg
    # a smaller level of the same storage still fits
    a = hg.P1Function("a", st, 2, 2)
    a.interpolate(1.0, 2, hg.All)
    assert _noalloc(st, a.device_ptr(2), a.device_ptr(2), 8, 2, hg.All, out.data_ptr()) == _capi.HG_OK
    st.synchronize()
    assert out.item() == a.dotGlobal(a, 2, hg.All)

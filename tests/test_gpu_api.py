"""Host-facing entry points: the asynchronous upload on a caller's stream gives the same level
buffer as the synchronous one, and a double-buffered pipeline (upload of the next right-hand
side overlapping the current cycle) gives the same iterates as the plain loop. The packed
owned-DoF transfers: a download gives the owned slots of the level buffer; an upload of them
gives back the whole level buffer (every copy slot refreshed from its owner), bit for bit, in
FP64 and FP32, twice in a row through the same staging buffer."""
import numpy as np
import pytest

import hyteg_b200 as hg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    import torch
    L = 4
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    stream = torch.cuda.Stream()
    st.set_stream(stream.cuda_stream)
    return st, L, stream


def test_upload_async_matches_upload(env):
    import torch
    st, L, stream = env
    n = st.level_size(L)
    host = torch.empty(n, dtype=torch.float64, pin_memory=True)
    host.numpy()[:] = np.random.default_rng(1).uniform(-1, 1, n)
    a, b = hg.P1Function("a", st, L, L), hg.P1Function("b", st, L, L)
    a.from_numpy(L, host.numpy())
    cs = torch.cuda.Stream()
    b.upload_async(L, host.numpy(), cs.cuda_stream)
    cs.synchronize()
    assert np.array_equal(a.to_numpy(L), b.to_numpy(L))
    with pytest.raises(ValueError):
        b.upload_async(L, host.numpy().astype(np.float32), cs.cuda_stream)


def test_double_buffered_pipeline_gives_the_same_iterates(env):
    import torch
    st, L, stream = env
    n = st.level_size(L)
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    rhs = []
    for k in range(4):
        h = torch.empty(n, dtype=torch.float64, pin_memory=True)
        h.numpy()[:] = np.random.default_rng(10 + k).uniform(-1, 1, n)
        rhs.append(h)

    def solver():
        return hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 50, 1e-16),
                                           hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3)

    # plain loop
    x, b = hg.P1Function("x", st, 0, L), hg.P1Function("b", st, 0, L)
    g = solver()
    for h in rhs:
        b.from_numpy(L, h.numpy())
        g.solve(A, x, b, L)
    plain = x.to_numpy(L)
    # pipelined loop: two buffers, uploads on a copy stream ordered by events
    y = hg.P1Function("y", st, 0, L)
    bufs = (hg.P1Function("b0", st, 0, L), hg.P1Function("b1", st, 0, L))
    g2 = solver()
    cs = torch.cuda.Stream()
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    released = [torch.cuda.Event(), torch.cuda.Event()]
    bufs[0].upload_async(L, rhs[0].numpy(), cs.cuda_stream)
    copied[0].record(cs)
    for k in range(len(rhs)):
        cur = k % 2
        if k + 1 < len(rhs):
            if k >= 1:
                cs.wait_event(released[1 - cur])
            bufs[1 - cur].upload_async(L, rhs[k + 1].numpy(), cs.cuda_stream)
            copied[1 - cur].record(cs)
        stream.wait_event(copied[cur])
        g2.solve(A, y, bufs[cur], L)
        released[cur].record(stream)
    torch.cuda.synchronize()
    assert np.array_equal(plain, y.to_numpy(L))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_owned_transfers_round_trip(env, dtype):
    import torch
    st, L, stream = env
    slots = st.host().owned_slots(L)
    assert st.owned_count(L) == len(slots)
    _, owned = st.host().slot_info(L)
    dof = owned >= 0  # owned DoFs and their copies (not the alignment padding)
    src, dst = hg.P1Function("src", st, L, L, dtype=dtype), hg.P1Function("dst", st, L, L, dtype=dtype)
    cs = torch.cuda.Stream()
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    packed = torch.empty(len(slots), dtype=tdt, pin_memory=True)
    for seed in (3, 4):  # twice: the staging buffer is reused
        src.fill_random(seed, L, hg.All)
        full = src.to_numpy(L)
        src.download_owned_async(L, packed.numpy(), cs.cuda_stream)
        cs.synchronize()
        assert np.array_equal(packed.numpy(), full[slots])
        dst.interpolate(0.0, L)
        dst.upload_owned_async(L, packed.numpy(), cs.cuda_stream)
        st.synchronize()
        assert np.array_equal(dst.to_numpy(L)[dof], full[dof])
    with pytest.raises(hg.HygError):
        dst.upload_owned_async(L, packed.numpy()[:-1], cs.cuda_stream)


def test_packed_pipeline_gives_the_same_iterates(env):
    """The bench's end-to-end loop: per step a cycle, the packed download of its solution and the
    packed upload of the next right-hand side, on two copy streams, two (x, b) pairs. Every
    downloaded solution equals the plain loop's iterate at that step."""
    import torch
    st, L, stream = env
    slots = st.host().owned_slots(L)
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    rhs = []
    for k in range(5):
        h = torch.empty(len(slots), dtype=torch.float64, pin_memory=True)
        h.numpy()[:] = np.random.default_rng(20 + k).uniform(-1, 1, len(slots))
        rhs.append(h)

    def solver():
        return hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 50, 1e-16),
                                           hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3)

    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    # plain loop, one pair: x is carried from step to step on each pair below, so the plain loop
    # keeps one x per pair as well
    xs = (hg.P1Function("px0", st, 0, L), hg.P1Function("px1", st, 0, L))
    b = hg.P1Function("pb", st, 0, L)
    g = solver()
    expect = []
    for k, h in enumerate(rhs):
        b.upload_owned_async(L, h.numpy(), up.cuda_stream)
        g.solve(A, xs[k % 2], b, L)
        expect.append(xs[k % 2].to_numpy(L)[slots])
    # pipelined loop
    xp = (hg.P1Function("qx0", st, 0, L), hg.P1Function("qx1", st, 0, L))
    bp = (hg.P1Function("qb0", st, 0, L), hg.P1Function("qb1", st, 0, L))
    out = [torch.empty(len(slots), dtype=torch.float64, pin_memory=True) for _ in rhs]
    g2 = solver()
    bp[0].upload_owned_async(L, rhs[0].numpy(), up.cuda_stream)
    for k in range(len(rhs)):
        cur = k % 2
        g2.solve(A, xp[cur], bp[cur], L)
        xp[cur].download_owned_async(L, out[k].numpy(), down.cuda_stream)
        if k + 1 < len(rhs):
            bp[1 - cur].upload_owned_async(L, rhs[k + 1].numpy(), up.cuda_stream)
    torch.cuda.synchronize()
    for k in range(len(rhs)):
        assert np.array_equal(out[k].numpy(), expect[k]), k

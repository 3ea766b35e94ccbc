"""The single-pass (z-wavefront, double-buffered) multicolour SOR and the colour passes on
colour-split copies (schedule 3) against the four in-place colour passes and against the oracle,
at levels where a macro-cell spans several tiles (32 x 24 or 32 x 28, and the shorter 32 x 12
tiles of schedule 2). Schedule 3 also runs inside multigrid cycles, where the copies are made once
per smoothing step and the right-hand side's copy is kept from the pre- to the post-smoothing.

Tolerances: FP64 1e-13 relative (max-norm over inner DoFs); FP32 1e-5 relative (the two
schedules round the relaxation differently)."""
import numpy as np
import pytest

import hyteg_b200 as hg
from tests import helpers as H

pytestmark = pytest.mark.gpu


def run_sor(st, L, x0, b0, dtype, schedule, sweeps, backwards, omega=1.3):
    st.set_sor_schedule(schedule)
    A = hg.P1ConstantLaplaceOperator(st, L, L)
    x = hg.P1Function("x", st, L, L, dtype=dtype)
    b = hg.P1Function("b", st, L, L, dtype=dtype)
    x.from_numpy(L, x0)
    b.from_numpy(L, b0)
    for _ in range(sweeps):
        if backwards:
            A.smooth_sor_backwards(x, b, omega, L, hg.Inner)
        else:
            A.smooth_sor(x, b, omega, L, hg.Inner)
    out = x.to_numpy(L).astype(np.float64)
    st.set_sor_schedule(0)
    return out


@pytest.fixture(scope="module")
def cube6():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, 6)
    mesh = hg.HostMesh.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, 6)
    return st, mesh


@pytest.mark.parametrize("L", [5, 6])
@pytest.mark.parametrize("backwards", [False, True])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-13), (np.float32, 1e-5)])
@pytest.mark.parametrize("schedule", [0, 2, 3])
def test_single_pass_equals_colour_passes(cube6, L, backwards, dtype, tol, schedule):
    # schedule 0: 32 x 24 (FP64) / 32 x 28 (FP32) tiles; schedule 2: 32 x 12 tiles; schedule 3:
    # colour passes on colour-split copies
    st, mesh = cube6
    n = st.level_size(L)
    _, owned = mesh.slot_info(L)
    rng = np.random.default_rng(L + 10 * backwards)
    x0 = rng.uniform(-1, 1, n).astype(dtype)
    b0 = rng.uniform(-1, 1, n).astype(dtype)
    got = run_sor(st, L, x0, b0, dtype, schedule, 2, backwards)
    ref = run_sor(st, L, x0, b0, dtype, 1, 2, backwards)
    m = owned == 1
    assert np.abs(got[m] - ref[m]).max() / np.abs(ref[m]).max() < tol
    # copies are refreshed identically under both schedules
    used = owned >= 0
    assert np.abs(got[used] - ref[used]).max() / np.abs(ref[used]).max() < tol


@pytest.mark.parametrize("schedule", [0, 3])
def test_single_pass_matches_oracle_level5(schedule):
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    L = 5
    coords, tets, mesh, orc = H.cube(L)
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    st.set_sor_schedule(schedule)
    xyz, owned = mesh.slot_info(L)
    node = H.match_slots(xyz, orc.nodes(L)[0])
    n = orc.n(L)
    rng = np.random.default_rng(55)
    u0, f0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    x, b = hg.P1Function("x", st, 0, L), hg.P1Function("b", st, 0, L)
    x.from_numpy(L, H.scatter(node, u0))
    b.from_numpy(L, H.scatter(node, f0))
    for _ in range(2):
        A.smooth_sor(x, b, 0.9, L, hg.Inner)
    got = H.gather_owned(x.to_numpy(L), node, owned, n)
    ref = orc.sor(L, u0, f0, 0.9, sweeps=2, multicolour=True)
    inner = ~orc.dirichlet(L)
    assert np.abs(got - ref)[inner].max() / np.abs(ref[inner]).max() < 1e-13


def test_buffer_exchange_and_padding(cube6):
    """The sweep exchanges the level buffer with the spare; an even number of sweeps restores the
    original address, and alignment padding stays zero."""
    st, mesh = cube6
    L = 6
    n = st.level_size(L)
    _, owned = mesh.slot_info(L)
    A = hg.P1ConstantLaplaceOperator(st, L, L)
    x = hg.P1Function("x", st, L, L)
    b = hg.P1Function("b", st, L, L)
    rng = np.random.default_rng(3)
    v = rng.uniform(-1, 1, n)
    v[owned < 0] = 0.0
    x.from_numpy(L, v)
    b.from_numpy(L, rng.uniform(-1, 1, n))
    p0 = x.device_ptr(L)
    A.smooth_sor(x, b, 1.0, L, hg.Inner)
    p1 = x.device_ptr(L)
    A.smooth_sor(x, b, 1.0, L, hg.Inner)
    p2 = x.device_ptr(L)
    assert p1 != p0 and p2 == p0
    out = x.to_numpy(L)
    assert np.all(out[owned < 0] == 0.0)
    assert np.all(np.isfinite(out))


def test_colour_split_keeps_the_buffer(cube6):
    """Schedule 3 copies the result back: the level buffer keeps its address after any number of
    sweeps, and alignment padding stays zero."""
    st, mesh = cube6
    L = 6
    n = st.level_size(L)
    _, owned = mesh.slot_info(L)
    st.set_sor_schedule(3)
    try:
        A = hg.P1ConstantLaplaceOperator(st, L, L)
        x = hg.P1Function("x", st, L, L)
        b = hg.P1Function("b", st, L, L)
        rng = np.random.default_rng(4)
        v = rng.uniform(-1, 1, n)
        v[owned < 0] = 0.0
        x.from_numpy(L, v)
        b.from_numpy(L, rng.uniform(-1, 1, n))
        p0 = x.device_ptr(L)
        A.smooth_sor(x, b, 1.0, L, hg.Inner)
        assert x.device_ptr(L) == p0
        out = x.to_numpy(L)
        assert np.all(out[owned < 0] == 0.0)
        assert np.all(np.isfinite(out))
    finally:
        st.set_sor_schedule(0)


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
@pytest.mark.parametrize("graphs", [False, True])
def test_colour_split_cycles_equal_colour_pass_cycles(cube6, dtype, tol, graphs):
    """V(3,3) and V(2,1) cycles (the right-hand side's split copy reused from pre- to
    post-smoothing) under schedule 3 against the same cycles under schedule 1."""
    st, mesh = cube6
    L = 6
    _, owned = mesh.slot_info(L)
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    for pre, post in ((3, 3), (2, 1)):
        res = []
        for schedule in (1, 3):
            st.set_sor_schedule(schedule)
            try:
                x, b = hg.P1Function("x", st, 0, L, dtype=dtype), hg.P1Function("b", st, 0, L, dtype=dtype)
                b.fill_random(21, L, hg.Inner)
                gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 100, 1e-16),
                                                  hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L,
                                                  pre, post, dtype=dtype)
                gmg.set_graphs(A, graphs)
                for _ in range(3):
                    gmg.solve(A, x, b, L)
                res.append(x.to_numpy(L).astype(np.float64))
            finally:
                st.set_sor_schedule(0)
        m = owned == 1
        assert np.abs(res[0][m] - res[1][m]).max() / np.abs(res[0][m]).max() < tol


@pytest.mark.parametrize("L", [3, 6])
@pytest.mark.parametrize("backwards", [False, True])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("schedule", [0, 1, 3])
def test_fused_phases_equal_per_colour_launches(cube6, L, backwards, dtype, schedule):
    """The face, edge and vertex phases as one launch each (halo refreshes folded in where no
    owner changes) against one launch per colour and per refresh: the whole level buffer, copies
    included, must agree bit for bit after two sweeps."""
    st, mesh = cube6
    n = st.level_size(L)
    rng = np.random.default_rng(40 + L + 3 * backwards)
    x0 = rng.uniform(-1, 1, n).astype(dtype)
    b0 = rng.uniform(-1, 1, n).astype(dtype)
    out = []
    try:
        for fused in (True, False):
            st.set_sor_fused_phases(fused)
            out.append(run_sor(st, L, x0, b0, dtype, schedule, 2, backwards))
    finally:
        st.set_sor_fused_phases(True)
    assert np.array_equal(out[0], out[1])

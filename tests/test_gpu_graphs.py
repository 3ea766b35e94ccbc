"""Multigrid cycles replayed from captured CUDA graphs, and the one-block coarse CG on the device.

- Cycles through graphs give bit-identical iterates to eager cycles, in FP64 and FP32, also
  when another function's odd number of SOR sweeps exchanges the smoother's spare buffer of a
  level between cycles (the cached graph must not be replayed then; a new one is captured).
- On the 3x3x3 cube (162 tetrahedra, 8 inner DoFs on level 0, so the coarse CG iterates) the
  V-cycles with the device coarse solve agree with the oracle to 1e-12 relative."""
import numpy as np
import pytest

import hyteg_b200 as hg
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")


def cycles(dtype, graphs, L=4, n=5, disturb=False):
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    x, b = hg.P1Function("x", st, 0, L, dtype=dtype), hg.P1Function("b", st, 0, L, dtype=dtype)
    y, f = hg.P1Function("y", st, 0, L, dtype=dtype), hg.P1Function("f", st, 0, L, dtype=dtype)
    b.fill_random(3, L, hg.Inner)
    f.fill_random(4, L - 1, hg.Inner)
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 100, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3,
                                      dtype=dtype)
    gmg.set_graphs(A, graphs)
    launches = []
    for i in range(n):
        l0 = st.launch_count()
        gmg.solve(A, x, b, L)
        launches.append(st.launch_count() - l0)
        if disturb and i == 2:  # one sweep on another function: exchanges the spare of level L-1
            A.smooth_sor(y, f, 1.0, L - 1, hg.Inner)
    return x.to_numpy(L), launches


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("disturb", [False, True])
def test_graph_replay_is_bit_identical(gpu, dtype, disturb):
    eager, le = cycles(dtype, False, disturb=disturb)
    graph, lg = cycles(dtype, True, disturb=disturb)
    assert np.array_equal(eager, graph)
    assert le == lg  # the launch counter counts the kernels inside a replayed graph


def test_device_coarse_cg_against_oracle_on_3x3x3_cube(gpu):
    L = 3
    coords, tets, mesh, orc = H.cube(L, nx=3)
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 3, 3, 3, L)
    xyz, owned = mesh.slot_info(L)
    node = H.match_slots(xyz, orc.nodes(L)[0])
    n = orc.n(L)
    assert (~orc.dirichlet(0)).sum() == 8
    bg = np.random.default_rng(21).uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    x, b = hg.P1Function("x", st, 0, L), hg.P1Function("b", st, 0, L)
    b.from_numpy(L, H.scatter(node, bg))
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 100, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3)
    for _ in range(3):
        gmg.solve(A, x, b, L)
    ref, _ = orc.gmg(L, 0, np.zeros(n), bg, 3, 3, 3, 1.0, multicolour=True, cg_iter=100, cg_tol=1e-16)
    got = H.gather_owned(x.to_numpy(L), node, owned, n)
    inner = ~orc.dirichlet(L)
    assert np.abs(got - ref)[inner].max() / np.abs(ref[inner]).max() < 1e-12


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_autotuned_schedules_give_the_same_cycles(gpu, dtype):
    L = 5
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    res = []
    for tune in (False, True):
        if tune:
            picks = st.autotune_sor(2, L, dtype=dtype, reps=2)
            assert set(picks) == set(range(2, L + 1))
            assert all(c in (0, 1, 2, 3) and min(ts) > 0 for c, *ts in picks.values())
        x, b = hg.P1Function("x", st, 0, L, dtype=dtype), hg.P1Function("b", st, 0, L, dtype=dtype)
        b.fill_random(8, L, hg.Inner)
        gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 100, 1e-16),
                                          hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3,
                                          dtype=dtype)
        for _ in range(3):
            gmg.solve(A, x, b, L)
        res.append(x.to_numpy(L).astype(np.float64))
    tol = 1e-12 if dtype == np.float64 else 1e-5
    assert np.abs(res[0] - res[1]).max() / np.abs(res[0]).max() < tol

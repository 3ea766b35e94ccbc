"""The compact coarse cycle (the coarse levels of a V-cycle as one launch per cycle, on
owner-indexed vectors) against the level-by-level cycle and the CPU oracle.

The compact cycle runs the same multicolour order and the same coarse CG as the level-by-level
cycle; only the order of the sums differs. Tolerances: FP64 iterates agree with the
level-by-level cycle and with the oracle to 1e-12 relative (max-norm over inner DoFs), FP32
iterates with the oracle's FP64 cycle to 2e-5."""
import numpy as np
import pytest

import hyteg_b200 as hg
from tests import helpers as H

pytestmark = pytest.mark.gpu
LMAX = 5


@pytest.fixture(scope="module")
def env():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    coords, tets, mesh, orc = H.cube(LMAX)
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, LMAX)
    maps = {}
    for L in range(LMAX + 1):
        xyz, owned = mesh.slot_info(L)
        maps[L] = (H.match_slots(xyz, orc.nodes(L)[0]), owned)
    return st, orc, maps


def up(f, L, g, maps):
    node, _ = maps[L]
    f.from_numpy(L, H.scatter(node, g).astype(f.dtype))


def down(f, L, maps, n):
    node, owned = maps[L]
    return H.gather_owned(f.to_numpy(L).astype(np.float64), node, owned, n)


def relerr(a, b, mask):
    return np.abs(a[mask] - b[mask]).max() / max(np.abs(b[mask]).max(), 1e-300)


def solver(st, maxL, dtype=np.float64, cycle=hg.VCYCLE):
    return hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 100, 1e-16),
                                       hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, maxL, 3, 3,
                                       cycleType=cycle, dtype=dtype)


def cycles(env, L, count, compact, dtype=np.float64, seed=11):
    """x after `count` V(3,3) cycles from x = 0 with a seeded right-hand side; compact = (max
    unknowns per group, blocks per group) or None for the default."""
    st, orc, maps = env
    n = orc.n(L)
    bg = np.random.default_rng(seed).uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    x = hg.P1Function("x", st, 0, LMAX, dtype=dtype)
    b = hg.P1Function("b", st, 0, LMAX, dtype=dtype)
    up(b, L, bg, maps)
    gmg = solver(st, LMAX, dtype)
    if compact is not None:
        gmg.set_compact(A, *compact)
    top = gmg.compact_top(A)
    for _ in range(count):
        gmg.solve(A, x, b, L)
    return down(x, L, maps, n), bg, top


def test_compact_top_follows_the_size_limit(env):
    st, orc, maps = env
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    gmg = solver(st, LMAX)
    gmg.set_compact(A, 6000, 1)  # an explicit request reports a failed build
    # unknowns per level of the 48-tet cube: (2^(L+1) + 1)^3
    assert gmg.compact_top(A) == 3  # at most 6000 unknowns (level 3: 4913)
    assert solver(st, LMAX).compact_top(A) == 3  # the default
    gmg.set_compact(A, 0)
    assert gmg.compact_top(A) == -1
    gmg.set_compact(A, 40000, 8)
    assert gmg.compact_top(A) == 4  # level 4: 35937
    gmg.set_compact(A, 10 ** 7, 2)
    assert gmg.compact_top(A) == 5
    gmg.set_compact(A, 100, 1)  # level 1: 125 unknowns, more than 100
    assert gmg.compact_top(A) == -1
    with pytest.raises(hg.HygError):
        gmg.set_compact(A, 6000, 3)
    w = solver(st, LMAX, cycle=hg.WCYCLE)
    assert w.compact_top(A) == -1


@pytest.mark.parametrize("L", [3, 4, 5])
@pytest.mark.parametrize("compact", [(6000, 1), (40000, 8), (10 ** 7, 1), (10 ** 7, 4)])
def test_compact_cycle_matches_level_by_level_and_oracle(env, L, compact):
    st, orc, maps = env
    got, bg, top = cycles(env, L, 3, compact)
    assert top >= 3
    ref, _, off = cycles(env, L, 3, (0, 1))
    assert off == -1
    inner = ~orc.dirichlet(L)
    assert relerr(got, ref, inner) < 1e-12
    oref, _ = orc.gmg(L, 0, np.zeros(orc.n(L)), bg, 3, 3, 3, 1.0, multicolour=True, cg_iter=100, cg_tol=1e-16)
    assert relerr(got, oref, inner) < 1e-12


@pytest.mark.parametrize("compact", [(6000, 1), (10 ** 7, 8)])
def test_compact_cycle_fp32(env, compact):
    st, orc, maps = env
    L = 4
    got, bg, top = cycles(env, L, 3, compact, dtype=np.float32)
    assert top >= 3
    oref, _ = orc.gmg(L, 0, np.zeros(orc.n(L)), bg, 3, 3, 3, 1.0, multicolour=True, cg_iter=100, cg_tol=1e-16)
    assert relerr(got, oref, ~orc.dirichlet(L)) < 2e-5


def test_compact_cycle_is_deterministic_and_graph_replays_agree(env):
    st, orc, maps = env
    L = 5
    n = orc.n(L)
    bg = np.random.default_rng(5).uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    runs = []
    for graphs in (True, False, True):
        x, b = hg.P1Function("x", st, 0, LMAX), hg.P1Function("b", st, 0, LMAX)
        up(b, L, bg, maps)
        gmg = solver(st, LMAX)
        gmg.set_compact(A, 40000, 8)
        gmg.set_graphs(A, graphs)
        for _ in range(4):  # eager, captured, replayed, replayed
            gmg.solve(A, x, b, L)
        runs.append(x.to_numpy(L))
    assert np.array_equal(runs[0], runs[1]) and np.array_equal(runs[0], runs[2])


def test_timing_tree_keeps_the_level_by_level_cycle(env):
    st, orc, maps = env
    L = 4
    got, bg, _ = cycles(env, L, 2, None)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    x, b = hg.P1Function("x", st, 0, LMAX), hg.P1Function("b", st, 0, LMAX)
    up(b, L, bg, maps)
    gmg = solver(st, LMAX)
    gmg.set_timing(A, True)
    for _ in range(2):
        gmg.solve(A, x, b, L)
    assert relerr(down(x, L, maps, orc.n(L)), got, ~orc.dirichlet(L)) < 1e-12


@pytest.mark.parametrize("minL", [1, 2])
def test_compact_cycle_above_level_zero(env, minL):
    """Coarsest level 1 or 2: the coarse CG then has edge, face and cell unknowns (on level 2)
    and runs inside the compact cycle on the device."""
    st, orc, maps = env
    L = 4
    n = orc.n(L)
    bg = np.random.default_rng(13).uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    out = {}
    for compact in (True, False):
        x, b = hg.P1Function("x", st, 0, LMAX), hg.P1Function("b", st, 0, LMAX)
        up(b, L, bg, maps)
        gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 2000, 1e-16),
                                          hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), minL, LMAX,
                                          3, 3)
        gmg.set_compact(A, 6000 if compact else 0, 1)
        assert gmg.compact_top(A) == (3 if compact else -1)
        for _ in range(3):
            gmg.solve(A, x, b, L)
        out[compact] = down(x, L, maps, n)
    inner = ~orc.dirichlet(L)
    oref, _ = orc.gmg(L, minL, np.zeros(n), bg, 3, 3, 3, 1.0, multicolour=True, cg_iter=2000, cg_tol=1e-16)
    assert relerr(out[True], oref, inner) < 1e-12
    assert relerr(out[False], oref, inner) < 1e-12

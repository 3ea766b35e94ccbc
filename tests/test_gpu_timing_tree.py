"""Device-timed timing tree of the multigrid (hg_gmg_set_timing / hg_gmg_timing_json): the
reference's node names and nesting (GeometricMultigridSolver.hpp:127-234), counts that follow the
cycle structure, the waLBerla timer fields, consistent times, and unchanged iterates."""
import numpy as np
import pytest

import hyteg_b200 as hg

pytestmark = pytest.mark.gpu
L = 5
FIELDS = {"total", "average", "count", "min", "max", "variance"}


@pytest.fixture(scope="module")
def gpu():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")


def solver(st, pre=3, post=3):
    return hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 100, 1e-16),
                                       hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, pre, post)


@pytest.mark.parametrize("pre,post", [(3, 3), (2, 1)])
def test_tree_structure_and_counts(gpu, pre, post):
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    x, b = hg.P1Function("x", st, 0, L), hg.P1Function("b", st, 0, L)
    b.fill_random(3, L, hg.Inner)
    gmg = solver(st, pre, post)
    gmg.solve(A, x, b, L)  # creates the solver
    gmg.set_timing(A, True)
    cycles = 3
    for _ in range(cycles):
        gmg.solve(A, x, b, L)
    tree = gmg.timing_tree(A)
    assert list(tree) == ["Geometric Multigrid Solver"]
    g = tree["Geometric Multigrid Solver"]
    assert FIELDS <= set(g) and g["count"] == cycles
    levels = [k for k in g if k.startswith("Level ")]
    assert sorted(levels) == sorted("Level %d" % l for l in range(L + 1))
    covered = 0.0
    for l in range(L + 1):
        n = g["Level %d" % l]
        assert FIELDS <= set(n) and n["total"] > 0 and n["min"] <= n["average"] <= n["max"]
        covered += n["total"]
        if l == 0:
            assert n["count"] == cycles
            assert n["Coarse Grid Solver"]["count"] == cycles
            assert n["Coarse Grid Solver"]["CG Solver"]["count"] == cycles
        else:
            assert n["count"] == 2 * cycles  # before and after the coarser levels
            assert n["Smoother"]["count"] == (pre + post) * cycles
            assert n["Restriction"]["count"] == cycles
            assert n["Prolongation"]["count"] == cycles
            kids = sum(n[k]["total"] for k in ("Smoother", "Restriction", "Prolongation"))
            assert kids <= n["total"] * (1 + 1e-6) + 1e-7
            assert abs(n["Remainder"]["total"] - max(n["total"] - kids, 0.0)) < 1e-6
    assert covered <= g["total"] * (1 + 1e-6) + 1e-7
    assert g["Remainder"]["total"] >= 0.0
    # the finest level dominates
    assert g["Level %d" % L]["total"] > g["Level 1"]["total"]
    gmg.set_timing(A, False)


@pytest.mark.parametrize("compact", [False, True])
def test_timing_does_not_change_the_iterates(gpu, compact):
    """Timed cycles run level by level: the same iterates bit for bit as untimed level-by-level
    cycles, and up to rounding (1e-12 relative) as cycles whose coarse levels run compact."""
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    out = []
    for timed in (False, True):
        x, b = hg.P1Function("x", st, 0, L), hg.P1Function("b", st, 0, L)
        b.fill_random(5, L, hg.Inner)
        gmg = solver(st)
        if not compact:
            gmg.set_compact(A, 0)
        gmg.solve(A, x, b, L)
        gmg.set_timing(A, timed)
        for _ in range(3):
            gmg.solve(A, x, b, L)
        out.append(x.to_numpy(L))
    if compact:
        assert np.abs(out[0] - out[1]).max() <= 1e-12 * np.abs(out[1]).max()
    else:
        assert np.array_equal(out[0], out[1])


def test_timing_off_is_an_error_to_read(gpu):
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 1, 1, 1, 2)
    A = hg.P1ConstantLaplaceOperator(st, 0, 2)
    x, b = hg.P1Function("x", st, 0, 2), hg.P1Function("b", st, 0, 2)
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 100, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, 2, 1, 1)
    gmg.solve(A, x, b, 2)
    with pytest.raises(hg.HygError):
        gmg.timing_tree(A)

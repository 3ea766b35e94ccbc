"""Multigrid convergence of the GPU path, level by level, against the reference's own
lexicographic smoother order.

1. The 48-tet cube, levels 3-6: the manufactured problem of the plain FP64 configuration
   (b = M I(3 pi^2 u), u = sin(pi x) sin(pi y) sin(pi z), x0 = 0, MultigridStudies.cpp:488-495),
   20 GPU V(3,3) cycles with CG on level 0. The golden fixture tests/golden/convergence_cube.json
   holds the oracle's residual histories for the reference's lexicographic SOR order and for the
   GPU's multicolour order (tests/golden/make_convergence_factors.py). Checked per level:
   - the mean factor of the first ten cycles and the asymptotic factor (geometric mean of cycles
     15-20) within 10 % of the lexicographic ones;
   - every cycle factor equal to the multicolour oracle's within 1e-6 (the same algorithm);
   - at levels 5 and 6, the discrete L2 error against u after ten cycles
     (sqrt(e.e / #inner), MultigridStudies.cpp:229-256) equal to the multicolour oracle's within
     1e-6 and to the lexicographic one within the algebraic error left after ten cycles.
   The factors grow with the level for both orders (0.22 at level 3 to 0.41 at level 6): a
   property of the reference's multigrid on this mesh, which the oracle shows for the
   lexicographic order too, and the GPU reproduces.
2. The reference's P1GMG3DConvergenceTest (tests/hyteg/convergence/P1GMG3DConvergenceTest.cpp:
   46-144) through the GPU solver: the regular octahedron (8 macro-tets), levels 0-3, u random in
   [0, 1) on inner DoFs and sin(x) sinh(y) z on the Dirichlet boundary, f = 0, ten V(3,3) cycles;
   every cycle must reduce the discrete squared residual (r.r / #inner) by a factor below 3.2e-2.
"""
import json
import os

import numpy as np
import pytest

import hyteg_b200 as hg
from tests import helpers as H

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "convergence_cube.json")) as _f:
    GOLD = json.load(_f)["levels"]
CYCLES = 20


@pytest.fixture(scope="module")
def cube():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    return hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, 6)


def gpu_run(st, L):
    inn = hg.Inner | hg.NeumannBoundary
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    M = hg.P1ConstantMassOperator(st, L, L)
    x, b, r, f, u = (hg.P1Function(n, st, 0, L) for n in ("x", "b", "r", "f", "u"))
    f.interpolate_sines(3 * np.pi ** 2, 1.0, L)
    u.interpolate_sines(1.0, 1.0, L)
    M.apply(f, b, L, hg.Inner)
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 1000, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3)
    n_inner = GOLD[str(L)]["inner_dofs"]

    def res():
        A.residual(x, b, r, L, inn)
        return np.sqrt(r.dotGlobal(r, L, inn))

    hist, err10 = [res()], None
    for c in range(CYCLES):
        gmg.solve(A, x, b, L)
        hist.append(res())
        if c == 9:
            r.assign([1.0, -1.0], [x, u], L, hg.All)
            err10 = float(np.sqrt(r.dotGlobal(r, L, hg.Inner) / n_inner))
    del gmg
    return np.array(hist), err10


def factors(h):
    h = np.asarray(h)
    return h[1:] / h[:-1]


@pytest.fixture(scope="module")
def runs(cube):
    return {L: gpu_run(cube, L) for L in (3, 4, 5, 6)}


@pytest.mark.parametrize("L", [3, 4, 5, 6])
def test_cycle_factors_match_the_lexicographic_order(runs, L):
    hist, _ = runs[L]
    lex = np.array(GOLD[str(L)]["lexicographic"]["residuals"])
    assert abs(hist[0] / lex[0] - 1) < 1e-12  # the same right-hand side
    f_gpu, f_lex = factors(hist), factors(lex)
    mean10 = lambda f: float(np.exp(np.log(f[:10]).mean()))  # noqa: E731
    asym = lambda f: float(np.exp(np.log(f[14:20]).mean()))  # noqa: E731
    assert abs(mean10(f_gpu) / mean10(f_lex) - 1) < 0.10, (mean10(f_gpu), mean10(f_lex))
    assert abs(asym(f_gpu) / asym(f_lex) - 1) < 0.10, (asym(f_gpu), asym(f_lex))


@pytest.mark.parametrize("L", [3, 4, 5, 6])
def test_cycle_factors_equal_the_multicolour_oracle(runs, L):
    hist, _ = runs[L]
    mc = np.array(GOLD[str(L)]["multicolour"]["residuals"])
    keep = mc[1:] / mc[0] > 1e-8  # well above the rounding floor of the residual
    d = np.abs(factors(hist) - factors(mc))[keep]
    assert d.max() < 1e-6, d.max()


@pytest.mark.parametrize("L", [5, 6])
def test_discretisation_error_after_ten_cycles(runs, L):
    hist, err = runs[L]
    g = GOLD[str(L)]
    assert abs(err / g["multicolour"]["l2_error_after_10"] - 1) < 1e-6, (err, g["multicolour"]["l2_error_after_10"])
    # the two orders differ only by the algebraic error left after ten cycles
    lex = g["lexicographic"]
    alg = lex["residuals"][10] / lex["residuals"][0]
    assert abs(err / lex["l2_error_after_10"] - 1) < max(1e-4, 10 * alg), (err, lex["l2_error_after_10"], alg)


def test_octahedron_reference_convergence_bound():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    from oracle import oracle

    with open(os.path.join(HERE, "golden", "meshes.json")) as f:
        m = json.load(f)["regular_octahedron_8el"]
    coords, tets = np.array(m["coords"], dtype=np.float64), np.array(m["tets"], dtype=np.int32)
    L = 3
    st = hg.PrimitiveStorage.from_tets(coords, tets, L)
    orc = oracle.Oracle(coords, tets, L)
    nodes = orc.nodes(L)[0]
    dirichlet = orc.dirichlet(L)
    xyz, _ = st.host().slot_info(L)
    node = H.match_slots(xyz, nodes)
    rng = np.random.default_rng(2024)
    un = rng.uniform(0.0, 1.0, len(nodes))
    p = nodes[dirichlet]
    un[dirichlet] = np.sin(p[:, 0]) * np.sinh(p[:, 1]) * p[:, 2]
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    x, b, r = (hg.P1Function(n, st, 0, L) for n in ("x", "b", "r"))
    x.from_numpy(L, np.where(node >= 0, un[np.maximum(node, 0)], 0.0))
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 10000, 1e-17),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3)
    n_inner = float((~dirichlet).sum())

    def sq_res():
        A.apply(x, r, L, hg.Inner)
        return r.dotGlobal(r, L, hg.Inner) / n_inner

    last = sq_res()
    rates = []
    for _ in range(10):
        gmg.solve(A, x, b, L)
        cur = sq_res()
        rates.append(cur / last)
        last = cur
    assert max(rates) < 3.2e-2, rates

"""Uzawa smoother and the geometric multigrid on the whole Taylor-Hood system against the
oracle's restatement (oracle.Oracle.uzawa_smooth / stokes_uzawa_cycle: assembled operators, the
multicolour P2 SOR, the composite transfers and a numpy pseudo-inverse on the coarsest level).

Tolerances: one smoothing step and the pressure transfers 1e-13 relative; two V-cycles 1e-11
relative (the oracle sums in another order, so the agreement is one of rounding); the
relaxation estimate (15 power iterations from the same seeded start) 1e-11 relative; V(3,3)
cycles with the estimated relaxation reduce the residual monotonically."""
import numpy as np
import pytest

import hyteg_b200 as hg
from tests import helpers as H

pytestmark = pytest.mark.gpu
LMAX = 2


@pytest.fixture(scope="module")
def env():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    coords, tets, mesh, orc = H.cube(LMAX + 1)
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, LMAX + 1)
    maps = {}
    for L in range(LMAX + 2):
        xyz, owned = mesh.slot_info(L)
        maps[L] = (H.match_slots(xyz, orc.nodes(L)[0]), owned, xyz)
    return st, orc, maps


def funcs(st, name):
    u = [hg.P2Function("%su%d" % (name, k), st, 0, LMAX) for k in range(3)]
    p = hg.P1Function(name + "p", st, 0, LMAX)
    return u, p


def put(maps, L, u, p, uu, pp):
    for k in range(3):
        u[k].from_numpy(L, H.scatter(maps[L + 1][0], uu[k]))
    p.from_numpy(L, H.scatter(maps[L][0], pp))


def get(maps, orc, L, u, p):
    nv, npr = orc.n(L + 1), orc.n(L)
    uu = [H.gather_owned(x.to_numpy(L), maps[L + 1][0], maps[L + 1][1], nv) for x in u]
    return uu, H.gather_owned(p.to_numpy(L), maps[L][0], maps[L][1], npr)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def random_state(orc, L, seed):
    rng = np.random.default_rng(seed)
    nv, npr = orc.n(L + 1), orc.n(L)
    dv = orc.dirichlet(L + 1)
    uu = [rng.uniform(-1, 1, nv) for _ in range(3)]
    ff = [np.where(dv, 0.0, rng.uniform(-1, 1, nv)) for _ in range(3)]
    return uu, rng.uniform(-1, 1, npr), ff, rng.uniform(-1, 1, npr)


def test_pressure_transfers_on_every_node(env):
    st, orc, maps = env
    L = 2
    rng = np.random.default_rng(3)
    fine, coarse = rng.uniform(-1, 1, orc.n(L)), rng.uniform(-1, 1, orc.n(L - 1))
    p = hg.P1Function("tp", st, 0, LMAX)
    p.from_numpy(L, H.scatter(maps[L][0], fine))
    hg.P1toP1LinearRestriction().restrict(p, L, hg.All)
    got = H.gather_owned(p.to_numpy(L - 1), maps[L - 1][0], maps[L - 1][1], orc.n(L - 1))
    assert rel(got, orc.restrict_all(L, fine)) < 1e-13
    p.from_numpy(L - 1, H.scatter(maps[L - 1][0], coarse))
    p.from_numpy(L, H.scatter(maps[L][0], fine))
    hg.P1toP1LinearProlongation().prolongateAndAdd(p, L - 1, hg.All)
    got = H.gather_owned(p.to_numpy(L), maps[L][0], maps[L][1], orc.n(L))
    assert rel(got, orc.prolongate_all(L - 1, coarse, fine, add=True)) < 1e-13


def test_pspg_diagonal(env):
    st, orc, maps = env
    for L in (1, 2):
        op = hg.P1PSPGOperator(st, L, L)
        n = orc.n(L)
        x, y = hg.P1Function("dx", st, L, L), hg.P1Function("dy", st, L, L)
        # the operator's diagonal through applies to unit vectors at a few nodes
        for i in np.random.default_rng(L).choice(np.where(~orc.dirichlet(L))[0], 5, replace=False):
            e = np.zeros(n)
            e[i] = 1.0
            x.from_numpy(L, H.scatter(maps[L][0], e))
            op.apply(x, y, L, hg.Inner)
            got = H.gather_owned(y.to_numpy(L), maps[L][0], maps[L][1], n)
            assert abs(got[i] - orc.pspg_diag(L)[i]) <= 1e-13 * abs(orc.pspg_diag(L)[i])


@pytest.mark.parametrize("L", [1, 2])
def test_uzawa_smoothing_step(env, L):
    st, orc, maps = env
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, LMAX)
    sm = hg.UzawaSmoother(st, S, 0, LMAX, 0.37, 2)
    uu, pp, ff, gg = random_state(orc, L, 10 + L)
    u, p = funcs(st, "x")
    f, g = funcs(st, "b")
    put(maps, L, u, p, uu, pp)
    put(maps, L, f, g, ff, gg)
    sm.solve(u, p, f, g, L)
    gu, gp = get(maps, orc, L, u, p)
    ru, rp = orc.uzawa_smooth(L, uu, pp, ff, gg, 0.37, 2)
    for k in range(3):
        assert rel(gu[k], ru[k]) < 1e-13
    assert rel(gp, rp) < 1e-13


def test_uzawa_vcycles_match_oracle(env):
    st, orc, maps = env
    L = 2
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, LMAX)
    sm = hg.UzawaSmoother(st, S, 0, LMAX, 0.3, 2)
    mg = hg.StokesGeometricMultigridSolver(st, S, sm, 0, LMAX, 2, 2)
    uu, pp, ff, gg = random_state(orc, L, 77)
    u, p = funcs(st, "x")
    f, g = funcs(st, "b")
    put(maps, L, u, p, uu, pp)
    put(maps, L, f, g, ff, gg)
    for _ in range(2):
        mg.solve(u, p, f, g, L)
        uu, pp = orc.stokes_uzawa_cycle(L, 0, uu, pp, ff, gg, 2, 2, 0.3)
    gu, gp = get(maps, orc, L, u, p)
    for k in range(3):
        assert rel(gu[k], uu[k]) < 1e-11
    assert rel(gp, pp) < 1e-11


def test_uzawa_relaxation_estimate_matches_oracle(env):
    st, orc, maps = env
    L = 2
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, LMAX)
    omega = hg.estimateUzawaRelaxationParameter(st, S, L, 15, 2, seed=42)
    start = hg.P1Function("st", st, L, L)
    start.fill_random(42, L, hg.All, 0.0, 1.0)  # the estimate's seeded start vector
    s0 = H.gather_owned(start.to_numpy(L), maps[L][0], maps[L][1], orc.n(L))
    ref = orc.uzawa_estimate(L, s0, 15, 2)
    assert abs(omega - ref) <= 1e-11 * abs(ref)
    assert 0.1 < omega < 1.0


def test_uzawa_multigrid_reduces_the_residual(env):
    # zero Dirichlet data, random body force: V(3,3) cycles with the estimated relaxation contract
    st, orc, maps = env
    L = 2
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, LMAX)
    omega = hg.estimateUzawaRelaxationParameter(st, S, L, 20, 2)
    sm = hg.UzawaSmoother(st, S, 0, LMAX, omega, 2)
    mg = hg.StokesGeometricMultigridSolver(st, S, sm, 0, LMAX, 3, 3)
    u, p = funcs(st, "x")
    f, g = funcs(st, "b")
    dv = orc.dirichlet(L + 1)
    rng = np.random.default_rng(5)
    for k in range(3):
        f[k].from_numpy(L, H.scatter(maps[L + 1][0], np.where(dv, 0.0, rng.uniform(-1, 1, orc.n(L + 1)))))
    it, relres, hist = mg.solve_to(u, p, f, g, L, 1e-3, 15)
    assert relres <= 1e-3, (it, hist)
    assert np.all(np.diff(hist) < 0)


def test_reference_uzawa_convergence_test_on_cube_24el():
    """The reference's P2P1Stokes3DUzawaConvergenceTest
    (tests/hyteg/convergence/P2P1Stokes3DUzawaConvergenceTest.cpp:56-203) through the GPU solver:
    mesh cube_24el, P2 levels 2..3, multigrid V(3,3) on the whole Taylor-Hood system with the Uzawa
    smoother (two block Gauss-Seidel velocity sweeps, relaxation 0.4), an exact solve on the
    coarsest level (the reference uses LU; here MINRES to 1e-11), the colliding-flow velocity
    u = (20 x y^3, 5 x^4 - 5 y^4, 0) on the Dirichlet boundary, zero interior start, f = g = 0;
    three cycles, the pressure projected to zero mean after each. Checked with the reference's
    bounds: sum of the velocity components' discrete L2 errors < 3e-3, pressure error < 0.8,
    scaled residual sqrt(r.r / (3 #velocity DoFs + #pressure DoFs)) < 5e-5."""
    import json
    import os

    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "meshes.json")) as f:
        m = json.load(f)["cube_24el"]
    coords, tets = np.array(m["coords"], dtype=np.float64), np.array(m["tets"], dtype=np.int32)
    minL, maxL = 2, 3
    st = hg.PrimitiveStorage.from_tets(coords, tets, maxL + 1)
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, maxL)
    mesh = st.host()
    xyzv, ownv = mesh.slot_info(maxL + 1)
    xyzp, ownp = mesh.slot_info(maxL)
    X, Y, Z = xyzv[:, 0], xyzv[:, 1], xyzv[:, 2]
    boundary = np.any((np.abs(xyzv) < 1e-12) | (np.abs(xyzv - 1.0) < 1e-12), axis=1)
    exact_u = [20 * X * Y ** 3, 5 * X ** 4 - 5 * Y ** 4, np.zeros_like(X)]
    xp, yp = xyzp[:, 0], xyzp[:, 1]
    exact_p = 60 * xp ** 2 * yp - 20 * yp ** 3
    ov, op = ownv == 1, ownp == 1
    nV, nP = int(ov.sum()), int(op.sum())
    exact_p = exact_p - exact_p[op].mean()

    u = [hg.P2Function("ru%d" % k, st, minL, maxL) for k in range(3)]
    f = [hg.P2Function("rf%d" % k, st, minL, maxL) for k in range(3)]
    v = [hg.P2Function("rv%d" % k, st, minL, maxL) for k in range(3)]
    p, g, q = (hg.P1Function(n, st, minL, maxL) for n in ("rp", "rg", "rq"))
    for k in range(3):
        u[k].from_numpy(maxL, np.where(boundary, exact_u[k], 0.0))
    sm = hg.UzawaSmoother(st, S, minL, maxL, 0.4, 2)
    mg = hg.StokesGeometricMultigridSolver(st, S, sm, minL, maxL, 3, 3)
    inn = hg.Inner | hg.NeumannBoundary
    for _ in range(3):
        mg.solve(u, p, f, g, maxL)
        pv = p.to_numpy(maxL)
        p.from_numpy(maxL, pv - pv[op].mean())
        for x in v:
            x.interpolate(0.0, maxL, hg.All)
        q.interpolate(0.0, maxL, hg.All)
        S.apply(u, p, v, q, maxL, inn, hg.All)
        rr = sum(x.dotGlobal(x, maxL, inn) for x in v) + q.dotGlobal(q, maxL, hg.All)
        residual = np.sqrt(rr / (3 * nV + nP))
    err_u = [np.sqrt(((u[k].to_numpy(maxL) - exact_u[k])[ov] ** 2).sum() / nV) for k in range(3)]
    err_p = np.sqrt(((p.to_numpy(maxL) - exact_p)[op] ** 2).sum() / nP)
    assert sum(err_u) < 3e-3, err_u
    assert err_p < 0.8, err_p
    assert residual < 5e-5, residual


def test_uzawa_concurrent_components_match_in_order(env):
    """The velocity sweeps of each Uzawa smoothing step on three streams (one per component) give
    the cycles of the same sweeps one after another, bit for bit."""
    st, orc, maps = env
    L = 2
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, LMAX)
    uu, pp, ff, gg = random_state(orc, L, 91)
    out = []
    for concurrent in (False, True):
        st.set_concurrent_components(concurrent)
        sm = hg.UzawaSmoother(st, S, 0, LMAX, 0.3, 3)
        mg = hg.StokesGeometricMultigridSolver(st, S, sm, 0, LMAX, 2, 2)
        u, p = funcs(st, "c%d" % concurrent)
        f, g = funcs(st, "d%d" % concurrent)
        put(maps, L, u, p, uu, pp)
        put(maps, L, f, g, ff, gg)
        for _ in range(3):  # the first smoothing of every level runs in order, the later ones not
            mg.solve(u, p, f, g, L)
        out.append(([x.to_numpy(L) for x in u], p.to_numpy(L)))
    st.set_concurrent_components(True)
    for k in range(3):
        assert np.array_equal(out[0][0][k], out[1][0][k])
    assert np.array_equal(out[0][1], out[1][1])

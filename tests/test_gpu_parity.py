"""Device kernels through the C-ABI against the CPU oracle (48-tet cube, levels 0-4).

Tolerances: FP64 results agree with the oracle to 1e-13 relative (max-norm over inner DoFs),
FP32 results to 2e-5 relative."""
import numpy as np
import pytest

import hyteg_b200 as hg
from tests import helpers as H

pytestmark = pytest.mark.gpu
LMAX = 4
TOL64 = 1e-13


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
    return st, mesh, orc, maps


def up(f, L, g, maps):
    node, _ = maps[L]
    f.from_numpy(L, H.scatter(node, g).astype(f.dtype))


def down(f, L, maps, n):
    node, owned = maps[L]
    return H.gather_owned(f.to_numpy(L).astype(np.float64), node, owned, n)


def relerr(a, b, mask):
    return np.abs(a[mask] - b[mask]).max() / max(np.abs(b[mask]).max(), 1e-300)


@pytest.mark.parametrize("L", [2, 3, 4])
@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("update", [hg.Replace, hg.Add])
def test_apply(env, L, form, update):
    st, mesh, orc, maps = env
    n = orc.n(L)
    rng = np.random.default_rng(100 * L + 10 * form + update)
    g = rng.uniform(-1, 1, n)
    d0 = rng.uniform(-1, 1, n)
    A = (hg.P1ConstantLaplaceOperator if form == 0 else hg.P1ConstantMassOperator)(st, 0, LMAX)
    src = hg.P1Function("src", st, 0, LMAX)
    dst = hg.P1Function("dst", st, 0, LMAX)
    up(src, L, g, maps)
    up(dst, L, d0, maps)
    A.apply(src, dst, L, hg.Inner, update)
    got = down(dst, L, maps, n)
    ref = orc.apply(L, g, form=form)
    inner = ~orc.dirichlet(L)
    if update == hg.Add:
        ref = np.where(inner, ref + d0, ref)
    assert relerr(got, ref, inner) < TOL64
    # Dirichlet DoFs are not written
    assert np.array_equal(got[~inner], d0[~inner])


@pytest.mark.parametrize("L", [2, 4])
def test_apply_fp32(env, L):
    st, mesh, orc, maps = env
    n = orc.n(L)
    g = np.random.default_rng(7).uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    src = hg.P1Function("src", st, 0, LMAX, dtype=np.float32)
    dst = hg.P1Function("dst", st, 0, LMAX, dtype=np.float32)
    up(src, L, g, maps)
    A.apply(src, dst, L, hg.Inner)
    ref = orc.apply(L, g.astype(np.float32).astype(np.float64))
    inner = ~orc.dirichlet(L)
    assert relerr(down(dst, L, maps, n), ref, inner) < 2e-5


@pytest.mark.parametrize("L", [2, 3, 4])
def test_residual_and_dot(env, L):
    st, mesh, orc, maps = env
    n = orc.n(L)
    rng = np.random.default_rng(5 + L)
    xg, bg = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    x, b, r = (hg.P1Function(s, st, 0, LMAX) for s in "xbr")
    up(x, L, xg, maps)
    up(b, L, bg, maps)
    A.residual(x, b, r, L, hg.Inner)
    inner = ~orc.dirichlet(L)
    ref = bg - orc.apply(L, xg)
    got = down(r, L, maps, n)
    assert relerr(got, ref, inner) < TOL64
    d = r.dotGlobal(r, L, hg.Inner)
    dref = orc.dot(L, np.where(inner, ref, 0), np.where(inner, ref, 0))
    assert abs(d - dref) / dref < 1e-13
    assert abs(x.dotGlobal(b, L, hg.All) - float(xg @ bg)) / abs(float(xg @ bg)) < 1e-12


@pytest.mark.parametrize("L", [1, 2, 3, 4])
@pytest.mark.parametrize("sweeps", [1, 3])
@pytest.mark.parametrize("omega", [1.0, 1.3])
def test_multicolour_sor(env, L, sweeps, omega):
    st, mesh, orc, maps = env
    n = orc.n(L)
    rng = np.random.default_rng(L * 31 + sweeps)
    ug, fg = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    u, f = hg.P1Function("u", st, 0, LMAX), hg.P1Function("f", st, 0, LMAX)
    up(u, L, ug, maps)
    up(f, L, fg, maps)
    for _ in range(sweeps):
        A.smooth_sor(u, f, omega, L, hg.Inner | hg.NeumannBoundary)
    ref = orc.sor(L, ug, fg, omega, sweeps, multicolour=True)
    assert relerr(down(u, L, maps, n), ref, np.ones(n, bool)) < TOL64


@pytest.mark.parametrize("L", [2, 4])
def test_multicolour_sor_backwards(env, L):
    st, mesh, orc, maps = env
    n = orc.n(L)
    rng = np.random.default_rng(L)
    ug, fg = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    u, f = hg.P1Function("u", st, 0, LMAX), hg.P1Function("f", st, 0, LMAX)
    up(u, L, ug, maps)
    up(f, L, fg, maps)
    A.smooth_sor_backwards(u, f, 1.0, L, hg.Inner)
    ref = orc.sor(L, ug, fg, 1.0, 1, multicolour=True, backwards=True)
    assert relerr(down(u, L, maps, n), ref, np.ones(n, bool)) < TOL64


@pytest.mark.parametrize("Lf", [1, 2, 3, 4])
def test_restrict(env, Lf):
    st, mesh, orc, maps = env
    rng = np.random.default_rng(Lf)
    g = rng.uniform(-1, 1, orc.n(Lf))
    f = hg.P1Function("f", st, 0, LMAX)
    up(f, Lf, g, maps)
    hg.P1toP1LinearRestriction().restrict(f, Lf, hg.Inner)
    ref = orc.restrict(Lf, g)
    inner = ~orc.dirichlet(Lf - 1)
    assert relerr(down(f, Lf - 1, maps, orc.n(Lf - 1)), ref, inner) < TOL64


@pytest.mark.parametrize("Lc", [0, 1, 2, 3])
@pytest.mark.parametrize("add", [False, True])
def test_prolongate(env, Lc, add):
    st, mesh, orc, maps = env
    rng = np.random.default_rng(Lc + 10 * add)
    cg_, fg = rng.uniform(-1, 1, orc.n(Lc)), rng.uniform(-1, 1, orc.n(Lc + 1))
    f = hg.P1Function("f", st, 0, LMAX)
    up(f, Lc, cg_, maps)
    up(f, Lc + 1, fg, maps)
    P = hg.P1toP1LinearProlongation()
    (P.prolongateAndAdd if add else P.prolongate)(f, Lc, hg.Inner)
    ref = orc.prolongate(Lc, cg_, fg, add=add)
    inner = ~orc.dirichlet(Lc + 1)
    got = down(f, Lc + 1, maps, orc.n(Lc + 1))
    assert relerr(got, ref, inner) < TOL64
    assert np.array_equal(got[~inner], fg[~inner])


def test_cg(env):
    st, mesh, orc, maps = env
    L = 2
    n = orc.n(L)
    bg = np.random.default_rng(3).uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    x, b = hg.P1Function("x", st, 0, LMAX), hg.P1Function("b", st, 0, LMAX)
    up(b, L, bg, maps)
    cg = hg.CGSolver(st, 0, LMAX, maxIter=500, tolerance=1e-13)
    cg.solve(A, x, b, L)
    ref, it, res = orc.cg(L, np.zeros(n), bg, 500, 1e-13)
    inner = ~orc.dirichlet(L)
    assert cg.residual < 1e-13
    assert relerr(down(x, L, maps, n), ref, inner) < 1e-10


@pytest.mark.parametrize("cycles", [1, 3])
def test_gmg_vcycle_matches_oracle(env, cycles):
    st, mesh, orc, maps = env
    L = LMAX
    n = orc.n(L)
    bg = np.random.default_rng(11).uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    x, b = hg.P1Function("x", st, 0, LMAX), hg.P1Function("b", st, 0, LMAX)
    up(b, L, bg, maps)
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 100, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3)
    for _ in range(cycles):
        gmg.solve(A, x, b, L)
    ref, res = orc.gmg(L, 0, np.zeros(n), bg, cycles, 3, 3, 1.0, multicolour=True, cg_iter=100, cg_tol=1e-16)
    inner = ~orc.dirichlet(L)
    assert relerr(down(x, L, maps, n), ref, inner) < 1e-12

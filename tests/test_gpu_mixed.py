"""Device interpolation and the mixed-precision (FP32 cycles inside FP64 defect correction)
multigrid, checked against the CPU oracle's FP64 solve and the manufactured solution
u = sin(pi x) sin(pi y) sin(pi z) on the 48-tet unit cube (homogeneous Dirichlet boundary).

Tolerances: interpolation 1e-14 absolute (FP64) / 1e-6 (FP32); a mixed solve driven to a 1e-10
relative residual agrees with the oracle's FP64 solution to 1e-8 relative, and its error
against the manufactured solution equals the FP64 error to 1e-6 relative."""
import numpy as np
import pytest

import hyteg_b200 as hg
from tests import helpers as H

pytestmark = pytest.mark.gpu
LMAX = 4


@pytest.fixture(scope="module")
def env():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    coords, tets, mesh, orc = H.cube(LMAX)
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, LMAX)
    maps = {}
    for L in range(LMAX + 1):
        xyz, owned = mesh.slot_info(L)
        maps[L] = (H.match_slots(xyz, orc.nodes(L)[0]), owned, xyz)
    return st, mesh, orc, maps


def down(f, L, maps, n):
    node, owned, _ = maps[L]
    return H.gather_owned(f.to_numpy(L).astype(np.float64), node, owned, n)


def sines(xyz, a=1.0, k=1.0):
    return a * np.sin(k * np.pi * xyz[:, 0]) * np.sin(k * np.pi * xyz[:, 1]) * np.sin(k * np.pi * xyz[:, 2])


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-14), (np.float32, 1e-6)])
@pytest.mark.parametrize("L", [0, 2, 4])
def test_interpolate_expressions(env, L, dtype, tol):
    st, mesh, orc, maps = env
    _, owned, xyz = maps[L]
    used = owned >= 0
    f = hg.P1Function("f", st, 0, LMAX, dtype=dtype)
    f.interpolate_sines(2.5, 2.0, L)
    got = f.to_numpy(L).astype(np.float64)
    assert np.abs(got[used] - sines(xyz[used], 2.5, 2.0)).max() < tol
    f.interpolate_linear(1.0, -2.0, 0.5, 3.0, L)
    got = f.to_numpy(L).astype(np.float64)
    lin = 1.0 - 2.0 * xyz[:, 0] + 0.5 * xyz[:, 1] + 3.0 * xyz[:, 2]
    assert np.abs(got[used] - lin[used]).max() < 10 * tol
    # flags restrict the write: the Dirichlet boundary keeps its value
    f.interpolate(0.0, L, hg.All)
    f.interpolate_linear(1.0, 0.0, 0.0, 0.0, L, hg.Inner)
    n = orc.n(L)
    g = down(f, L, maps, n)
    dir_ = orc.dirichlet(L)
    assert np.all(g[dir_] == 0.0) and np.all(g[~dir_] == 1.0)


def manufactured(env, L, dtype):
    st, mesh, orc, maps = env
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    M = hg.P1ConstantMassOperator(st, 0, LMAX)
    f = hg.P1Function("f", st, 0, LMAX)
    b = hg.P1Function("b", st, 0, LMAX)
    x = hg.P1Function("x", st, 0, LMAX)
    f.interpolate_sines(3 * np.pi ** 2, 1.0, L)
    M.apply(f, b, L, hg.Inner)
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 200, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3,
                                      dtype=dtype)
    return A, b, x, gmg


@pytest.mark.parametrize("L", [3, 4])
def test_mixed_precision_solve_matches_fp64(env, L):
    st, mesh, orc, maps = env
    n = orc.n(L)
    nodes = orc.nodes(L)[0]
    inner = ~orc.dirichlet(L)
    # oracle FP64 solution of the same system
    fn = 3 * np.pi ** 2 * sines(nodes)
    bref = orc.apply(L, fn, form=1)
    xref, _, res = orc.cg(L, np.zeros(n), bref, 20000, 1e-15)
    exact = sines(nodes)
    err_ref = np.abs(xref - exact)[inner].max()

    out = {}
    for dtype in (np.float64, np.float32):
        A, b, x, gmg = manufactured(env, L, dtype)
        it, rel, hist = gmg.solve_to(A, x, b, L, 1e-10, 60)
        assert rel <= 1e-10 and len(hist) == it
        assert np.all(np.diff(hist) < 0)
        got = down(x, L, maps, n)
        assert np.abs(got - xref)[inner].max() / np.abs(xref[inner]).max() < 1e-8
        err = np.abs(got - exact)[inner].max()
        assert abs(err - err_ref) / err_ref < 1e-6
        out[dtype] = (it, got)
    # defect correction around FP32 cycles needs at most a few more iterations than FP64 cycles
    assert out[np.float32][0] <= out[np.float64][0] + 3


def kcoef(c):
    """k(x) = 1 + 0.5 sin(2 pi x) cos(2 pi y) z at the macro-cell centroid."""
    return 1.0 + 0.5 * np.sin(2 * np.pi * c[:, 0]) * np.cos(2 * np.pi * c[:, 1]) * c[:, 2]


def test_mixed_precision_variable_coefficient(env):
    """Piecewise-constant k per macro-cell: the mixed solve reproduces the oracle's FP64 solve."""
    st0, mesh0, orc0, maps = env
    coords, tets, _, _ = H.cube(LMAX)
    k_st, k_orc = H.cell_coefficients(mesh0, coords, tets, kcoef)
    assert np.allclose(np.sort(k_st), np.sort(k_orc)) and np.ptp(k_st) > 0.2
    from oracle.oracle import Oracle
    orc = Oracle(coords, tets, LMAX, k=k_orc)
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, LMAX)
    st.set_cell_coefficients(k_st)
    L = LMAX
    n = orc.n(L)
    inner = ~orc.dirichlet(L)
    bg = np.random.default_rng(5).uniform(-1, 1, n)
    xref, _, _ = orc.cg(L, np.zeros(n), bg, 20000, 1e-15)
    node, owned, _ = maps[L]
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    b = hg.P1Function("b", st, 0, LMAX)
    x = hg.P1Function("x", st, 0, LMAX)
    b.from_numpy(L, H.scatter(node, bg))
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 200, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3,
                                      dtype=np.float32)
    it, rel, hist = gmg.solve_to(A, x, b, L, 1e-10, 80)
    assert rel <= 1e-10
    got = H.gather_owned(x.to_numpy(L), node, owned, n)
    assert np.abs(got - xref)[inner].max() / np.abs(xref[inner]).max() < 1e-8


@pytest.mark.parametrize("L", [2, 4])
def test_variable_coefficient_apply(env, L):
    st0, mesh0, orc0, maps = env
    coords, tets, _, _ = H.cube(LMAX)
    k_st, k_orc = H.cell_coefficients(mesh0, coords, tets, kcoef)
    from oracle.oracle import Oracle
    orc = Oracle(coords, tets, LMAX, k=k_orc)
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, LMAX)
    st.set_cell_coefficients(k_st)
    n = orc.n(L)
    node, owned, _ = maps[L]
    g = np.random.default_rng(9).uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    src = hg.P1Function("src", st, 0, LMAX)
    dst = hg.P1Function("dst", st, 0, LMAX)
    src.from_numpy(L, H.scatter(node, g))
    A.apply(src, dst, L, hg.Inner)
    got = H.gather_owned(dst.to_numpy(L), node, owned, n)
    ref = orc.apply(L, g)
    inner = ~orc.dirichlet(L)
    assert np.abs(got - ref)[inner].max() / np.abs(ref[inner]).max() < 1e-13


def test_solve_to_rejects_fp32_functions(env):
    st, mesh, orc, maps = env
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    x = hg.P1Function("x", st, 0, LMAX, dtype=np.float32)
    b = hg.P1Function("b", st, 0, LMAX, dtype=np.float32)
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 50, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, 2, 3, 3,
                                      dtype=np.float32)
    with pytest.raises(hg.HygError):
        gmg.solve_to(A, x, b, 2, 1e-8, 5)

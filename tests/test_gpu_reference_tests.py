"""The reference's own known-answer tests for this path, run through the GPU path on its 3-D mesh
fixtures (tests/golden/meshes.json, the reference's .msh files):

- VertexDoFLinearProlongation3DTest (tests/hyteg/vertexdofspace/VertexDoFLinearProlongation3DTest.cpp):
  linear prolongation reproduces constants and linear functions, err.err < 1e-15 over
  Inner | NeumannBoundary (lower levels 0, 1 and 3); prolongateAndAdd equals prolongate followed
  by add, err.err < 1e-15 (lower levels 0, 1 and 3).
- P1LaplaceOperator3DTest (tests/hyteg/P1/P1LaplaceOperator3DTest.cpp): A u = 0 at the inner
  DoFs for u = 0, 1, 42 x and 42 x + y + 1337 z, discrete L2 error sqrt(e.e / #inner) < 2.8e-13,
  on its seven (mesh, level) cases.
- P1GSConvergenceTest (tests/hyteg/convergence/P1GSConvergenceTest.cpp): level 4, Dirichlet data
  sin(x) sinh(y), random inner start, zero right-hand side; every one of 20 forward (and,
  separately, backward) SOR sweeps with omega = 1 reduces the residual norm over the inner DoFs.
  The smoother here is the GPU's multicolour SOR, not the reference's lexicographic one.
- P1CG3DConvergenceTest (tests/hyteg/convergence/P1CG3DConvergenceTest.cpp): CG (tolerance
  1e-16, no iteration limit) on the octahedron at levels 3 and 4 from a random inner start with
  Dirichlet data sin(x) sinh(y) z and f = 0: residual sqrt(r.r / #inner) < 6.9e-17 and < 3.88e-17,
  error against the interpolated solution < 4.4e-4 and < 1e-4.
- P2GSConvergenceTest (tests/hyteg/convergence/P2GSConvergenceTest.cpp): the same for P2 at
  level 4 on tet_1el and the octahedron, 20 forward (and, separately, backward) sweeps of the
  GPU's multicolour P2 SOR.
- P2QuadraticProlongation3DTest (tests/hyteg/P2/P2QuadraticProlongation3DTest.cpp): quadratic
  prolongation reproduces constants, linears and 2x^2 + 3x + 13 + 4y + 5y^2 + z^2 + 6, err.err <
  1e-15 over Inner | NeumannBoundary (lower levels 0, 1 and 3); prolongateAndAdd equals
  prolongate followed by add.
- P2LaplaceOperator3DTest (tests/hyteg/P2/P2LaplaceOperator3DTest.cpp): the P2 Laplacian
  annihilates constants and linears at the inner DoFs, discrete L2 error < 4e-12, on its eleven
  (mesh, level) cases.
- P2GMG3DConvergenceTest (tests/hyteg/convergence/P2GMG3DConvergenceTest.cpp): the octahedron,
  P2 levels 0-3, random inner start, Dirichlet data sin(x) sinh(y) z, f = 0, ten V(2,2) cycles;
  every cycle reduces the discrete squared residual (r.r / #inner) by a factor below 3e-2. The
  smoother is the GPU's multicolour P2 SOR (the reference's Gauss-Seidel smoother is
  lexicographic) and the coarsest level is solved exactly (the reference runs CG to 1e-16).
- P2P1Stokes3DMinResConvergenceTest (tests/hyteg/convergence/P2P1Stokes3DMinResConvergenceTest.cpp):
  cube_24el, P2 level 2, colliding-flow Dirichlet data, zero right-hand sides, 20 MINRES
  iterations at tolerance 1e-13; the sum of the velocity components' discrete L2 errors < 0.6417,
  the pressure's < 4.003 (both pressures with zero mean) and the residual's < 0.01934, each
  sqrt(e.e / #DoFs of the Taylor-Hood function). The reference preconditions the pressure block
  only; this solver adds P2 V(2,2) cycles on the velocity, which can only lower the errors after
  20 iterations."""
import json
import os

import numpy as np
import pytest

import hyteg_b200 as hg

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "meshes.json")) as _f:
    MESHES = json.load(_f)
MESHES_3D = ["tet_1el", "pyramid_2el", "pyramid_4el", "pyramid_tilted_4el", "regular_octahedron_8el"]
FREE = hg.Inner | hg.NeumannBoundary


@pytest.fixture(scope="module")
def gpu():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")


def storage(name, max_level):
    m = MESHES[name]
    return hg.PrimitiveStorage.from_tets(np.array(m["coords"], dtype=np.float64), np.array(m["tets"], dtype=np.int32),
                                         max_level)


@pytest.mark.parametrize("name", MESHES_3D)
@pytest.mark.parametrize("lower", [0, 1, 3])
def test_linear_prolongation_is_exact(gpu, name, lower):
    st = storage(name, lower + 1)
    u, exact, err = (hg.P1Function(n, st, lower, lower + 1) for n in ("u", "exact", "err"))
    P = hg.P1toP1LinearProlongation()
    # 0, 1, 42, 42 x, 42 x + y as a + b x + c y + d z
    for coef in ((0, 0, 0, 0), (1, 0, 0, 0), (42, 0, 0, 0), (0, 42, 0, 0), (0, 42, 1, 0)):
        u.interpolate_linear(*coef, lower, hg.All)
        exact.interpolate_linear(*coef, lower + 1, FREE)
        P.prolongate(u, lower, FREE)
        err.assign([1.0, -1.0], [u, exact], lower + 1, FREE)
        assert err.dotGlobal(err, lower + 1, FREE) < 1e-15, (name, lower, coef)


@pytest.mark.parametrize("name", MESHES_3D)
@pytest.mark.parametrize("lower", [0, 1, 3])
def test_prolongate_and_add(gpu, name, lower):
    st = storage(name, lower + 1)
    up, ua, upa, err = (hg.P1Function(n, st, lower, lower + 1) for n in ("up", "ua", "upa", "err"))

    def term_prolongate(x, y, z):
        return np.sin(x) + np.sinh(y) + z * z

    def term_add(x, y, z):
        return np.cos(x) + np.cosh(y) + z * z * z

    up.interpolate(term_prolongate, lower, hg.All)
    up.interpolate(term_add, lower + 1, hg.All)
    ua.interpolate(term_add, lower + 1, hg.All)
    upa.interpolate(term_prolongate, lower, hg.All)
    upa.interpolate(term_add, lower + 1, hg.All)
    P = hg.P1toP1LinearProlongation()
    P.prolongate(up, lower, FREE)
    P.prolongateAndAdd(upa, lower, FREE)
    up.add([1.0], [ua], lower + 1, FREE)
    err.assign([1.0, -1.0], [up, upa], lower + 1, FREE)
    assert err.dotGlobal(err, lower + 1, FREE) < 1e-15, (name, lower)


@pytest.mark.parametrize("name", ["tet_1el", "regular_octahedron_8el"])
@pytest.mark.parametrize("backwards", [False, True])
def test_gauss_seidel_reduces_the_residual_every_sweep(gpu, name, backwards):
    L = 4
    st = storage(name, L)
    A = hg.P1ConstantLaplaceOperator(st, L, L)
    x, rhs, Lu, res = (hg.P1Function(n, st, L, L) for n in ("x", "rhs", "Lu", "res"))
    x.interpolate(lambda px, py, pz: np.sin(px) * np.sinh(py), L, hg.DirichletBoundary)
    x.fill_random(0, L, hg.Inner, 0.0, 1.0)
    rhs.interpolate(0.0, L)

    def norm():
        A.apply(x, Lu, L, hg.Inner)
        res.assign([1.0, -1.0], [rhs, Lu], L, hg.Inner)
        return np.sqrt(res.dotGlobal(res, L, hg.Inner))

    old = norm()
    assert old > 0
    for i in range(20):
        if backwards:
            A.smooth_sor_backwards(x, rhs, 1.0, L, hg.Inner)
        else:
            A.smooth_sor(x, rhs, 1.0, L, hg.Inner)
        new = norm()
        assert new < old, (name, backwards, i, new, old)
        old = new


@pytest.mark.parametrize("name,L", [("tet_1el", 2), ("tet_1el", 3), ("pyramid_2el", 2), ("pyramid_2el", 3),
                                    ("pyramid_4el", 3), ("pyramid_tilted_4el", 3), ("regular_octahedron_8el", 3)])
def test_laplace_annihilates_constants_and_linears(gpu, name, L):
    st = storage(name, L)
    A = hg.P1ConstantLaplaceOperator(st, L, L)
    u, result, err, one = (hg.P1Function(n, st, L, L) for n in ("u", "result", "err", "one"))
    one.interpolate(1.0, L, hg.All)
    n_points = one.dotGlobal(one, L, hg.Inner)
    for coef in ((0, 0, 0, 0), (1, 0, 0, 0), (0, 42, 0, 0), (0, 42, 1, 1337)):
        u.interpolate_linear(*coef, L, hg.All)
        result.interpolate(0.0, L, hg.DirichletBoundary)
        A.apply(u, result, L, hg.Inner)
        err.assign([1.0], [result], L, hg.All)  # the exact result is 0 everywhere
        l2 = np.sqrt(err.dotGlobal(err, L, hg.Inner) / n_points)
        assert l2 < 2.8e-13, (name, L, coef, l2)


QUADRATICS = [lambda x, y, z: 0.0 * x, lambda x, y, z: 1.0 + 0.0 * x, lambda x, y, z: 42.0 + 0.0 * x,
              lambda x, y, z: 42.0 * x, lambda x, y, z: 42.0 * x + y + 1337.0 * z,
              lambda x, y, z: 2.0 * x * x + 3.0 * x + 13.0 + 4.0 * y + 5.0 * y * y + z * z + 6.0]


@pytest.mark.parametrize("name", MESHES_3D)
@pytest.mark.parametrize("lower", [0, 1, 3])
def test_quadratic_prolongation_is_exact(gpu, name, lower):
    st = storage(name, lower + 2)  # P2 level lower + 1 lives on the vertex lattice lower + 2
    u, exact, err = (hg.P2Function(n, st, lower, lower + 1) for n in ("u", "exact", "err"))
    P = hg.P2toP2QuadraticProlongation()
    for i, fn in enumerate(QUADRATICS):
        u.interpolate(fn, lower, hg.All)
        exact.interpolate(fn, lower + 1, FREE)
        P.prolongate(u, lower, FREE)
        err.assign([1.0, -1.0], [u, exact], lower + 1, FREE)
        assert err.dotGlobal(err, lower + 1, FREE) < 1e-15, (name, lower, i)


@pytest.mark.parametrize("name", MESHES_3D)
@pytest.mark.parametrize("lower", [0, 1, 3])
def test_p2_prolongate_and_add(gpu, name, lower):
    st = storage(name, lower + 2)
    up, ua, upa, err = (hg.P2Function(n, st, lower, lower + 1) for n in ("up", "ua", "upa", "err"))

    def term_prolongate(x, y, z):
        return np.sin(x) + np.sinh(y) + z * z

    def term_add(x, y, z):
        return np.cos(x) + np.cosh(y) + z * z * z

    up.interpolate(term_prolongate, lower, hg.All)
    up.interpolate(term_add, lower + 1, hg.All)
    ua.interpolate(term_add, lower + 1, hg.All)
    upa.interpolate(term_prolongate, lower, hg.All)
    upa.interpolate(term_add, lower + 1, hg.All)
    P = hg.P2toP2QuadraticProlongation()
    P.prolongate(up, lower, FREE)
    P.prolongateAndAdd(upa, lower, FREE)
    up.assign([1.0, 1.0], [up, ua], lower + 1, FREE)
    err.assign([1.0, -1.0], [up, upa], lower + 1, FREE)
    assert err.dotGlobal(err, lower + 1, FREE) < 1e-15, (name, lower)


def test_p2_multigrid_reference_convergence_bound(gpu):
    minL, maxL = 0, 3
    st = storage("regular_octahedron_8el", maxL + 1)
    A = hg.P2ConstantLaplaceOperator(st, minL, maxL)
    u, f, res, one = (hg.P2Function(n, st, minL, maxL) for n in ("u", "f", "res", "one"))
    u.fill_random(0, maxL, hg.Inner, 0.0, 1.0)
    u.interpolate(lambda x, y, z: np.sin(x) * np.sinh(y) * z, maxL, hg.DirichletBoundary)
    f.interpolate(0.0, maxL, hg.All)
    one.interpolate(1.0, maxL, hg.All)
    n_points = one.dotGlobal(one, maxL, hg.Inner)
    gmg = hg.P2GeometricMultigridSolver(st, A, minL, maxL, 2, 2)

    def sq_res():
        A.apply(u, res, maxL, hg.Inner)
        return res.dotGlobal(res, maxL, hg.Inner) / n_points

    last = sq_res()
    rates = []
    for _ in range(10):
        gmg.solve(u, f, maxL)
        cur = sq_res()
        rates.append(cur / last)
        last = cur
    assert max(rates) < 3.0e-2, rates


@pytest.mark.parametrize("name,L", [("regular_octahedron_8el", 0), ("cube_24el", 0), ("tet_1el", 1), ("tet_1el", 2),
                                    ("tet_1el", 3), ("tet_1el", 4), ("tet_tilted_1el", 3), ("pyramid_2el", 2),
                                    ("pyramid_2el", 3), ("pyramid_4el", 3), ("pyramid_tilted_4el", 3),
                                    ("regular_octahedron_8el", 3)])
def test_p2_laplace_annihilates_constants_and_linears(gpu, name, L):
    st = storage(name, L + 1)
    A = hg.P2ConstantLaplaceOperator(st, L, L)
    u, result, err, one = (hg.P2Function(n, st, L, L) for n in ("u", "result", "err", "one"))
    one.interpolate(1.0, L, hg.All)
    n_points = one.dotGlobal(one, L, hg.Inner)
    for i, fn in enumerate([lambda x, y, z: 0.0 * x, lambda x, y, z: 1.0 + 0.0 * x, lambda x, y, z: 42.0 * x,
                            lambda x, y, z: x + y, lambda x, y, z: 42.0 * x + y + 1337.0 * z]):
        u.interpolate(fn, L, hg.All)
        result.interpolate(0.0, L, hg.DirichletBoundary)
        A.apply(u, result, L, hg.Inner)
        err.assign([1.0], [result], L, hg.All)  # the exact result is 0 everywhere
        l2 = np.sqrt(err.dotGlobal(err, L, hg.Inner) / n_points) if n_points > 0 else 0.0
        assert l2 < 4.0e-12, (name, L, i, l2)


def test_stokes_minres_reference_bounds(gpu):
    L = 2
    st = storage("cube_24el", L + 1)
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, L)
    u = [hg.P2Function("u%d" % k, st, 0, L) for k in range(3)]
    f = [hg.P2Function("f%d" % k, st, 0, L) for k in range(3)]
    r = [hg.P2Function("r%d" % k, st, 0, L) for k in range(3)]
    p, g, q = (hg.P1Function(n, st, 0, L) for n in ("p", "g", "q"))
    exact_u = [lambda x, y, z: 20.0 * x * y ** 3, lambda x, y, z: 5.0 * x ** 4 - 5.0 * y ** 4,
               lambda x, y, z: 0.0 * x]
    u[0].interpolate(exact_u[0], L, hg.DirichletBoundary)
    u[1].interpolate(exact_u[1], L, hg.DirichletBoundary)
    S.minres(u, p, f, g, L, nu=2, max_iter=20, tol=1e-13)
    host = st.host()
    sv, sp = host.owned_slots(L + 1), host.owned_slots(L)  # every velocity / pressure DoF once
    xv, xp = host.slot_info(L + 1)[0][sv], host.slot_info(L)[0][sp]
    n_dofs = 3 * len(sv) + len(sp)
    err_u = sum(np.sqrt(np.sum((u[k].to_numpy(L)[sv] - exact_u[k](*xv.T)) ** 2) / n_dofs) for k in range(3))
    pn = p.to_numpy(L)[sp]
    pe = 60.0 * xp[:, 0] ** 2 * xp[:, 1] - 20.0 * xp[:, 1] ** 3
    err_p = np.sqrt(np.sum(((pn - pn.mean()) - (pe - pe.mean())) ** 2) / n_dofs)
    S.apply(u, p, r, q, L, hg.Inner | hg.NeumannBoundary, hg.All)
    res = np.sqrt((sum(r[k].dotGlobal(r[k], L) for k in range(3)) + q.dotGlobal(q, L)) / n_dofs)
    assert err_u < 0.6417 and err_p < 4.003 and res < 0.01934, (err_u, err_p, res)


def test_cg_reference_convergence_bounds(gpu):
    lower, higher = 3, 4
    st = storage("regular_octahedron_8el", higher)
    A = hg.P1ConstantLaplaceOperator(st, lower, higher)
    u, f, res, exact, err, one = (hg.P1Function(n, st, lower, higher) for n in ("u", "f", "res", "exact", "err", "one"))

    def solution(x, y, z):
        return np.sin(x) * np.sinh(y) * z

    cg = hg.CGSolver(st, lower, higher, 2 ** 31 - 1, 1e-16)
    for L, res_bound, err_bound in ((lower, 6.9e-17, 4.4e-4), (higher, 3.88e-17, 1.0e-4)):
        u.fill_random(7 + L, L, hg.Inner, 0.0, 1.0)
        u.interpolate(solution, L, hg.DirichletBoundary)
        f.interpolate(0.0, L, hg.All)
        exact.interpolate(solution, L, hg.All)
        one.interpolate(1.0, L, hg.All)
        n_points = one.dotGlobal(one, L, hg.Inner)
        cg.solve(A, u, f, L)
        err.assign([1.0, -1.0], [u, exact], L, hg.All)
        A.apply(u, res, L, hg.Inner)
        l2_err = np.sqrt(err.dotGlobal(err, L, hg.Inner) / n_points)
        l2_res = np.sqrt(res.dotGlobal(res, L, hg.Inner) / n_points)
        assert l2_res < res_bound and l2_err < err_bound, (L, l2_res, l2_err)


@pytest.mark.parametrize("name", ["tet_1el", "regular_octahedron_8el"])
@pytest.mark.parametrize("backwards", [False, True])
def test_p2_gauss_seidel_reduces_the_residual_every_sweep(gpu, name, backwards):
    L = 4
    st = storage(name, L + 1)
    A = hg.P2ConstantLaplaceOperator(st, L, L)
    x, rhs, Lu, res = (hg.P2Function(n, st, L, L) for n in ("x", "rhs", "Lu", "res"))
    x.interpolate(lambda px, py, pz: np.sin(px) * np.sinh(py), L, hg.DirichletBoundary)
    x.fill_random(0, L, hg.Inner, 0.0, 1.0)
    rhs.interpolate(0.0, L)

    def norm():
        A.apply(x, Lu, L, hg.Inner)
        res.assign([1.0, -1.0], [rhs, Lu], L, hg.Inner)
        return np.sqrt(res.dotGlobal(res, L, hg.Inner))

    old = norm()
    assert old > 0
    for i in range(20):
        if backwards:
            A.smooth_sor_backwards(x, rhs, 1.0, L, hg.Inner)
        else:
            A.smooth_sor(x, rhs, 1.0, L, hg.Inner)
        new = norm()
        assert new < old, (name, backwards, i, new, old)
        old = new

"""P2 Laplace apply and residual on the device against the oracle's globally assembled P2
matrix (48-tet cube, P2 levels 0-4 = vertex lattices 1-5; 3x3x3 cube for coarse levels with
inner DoFs on every primitive kind). From lattice 8 per macro-cell on, every parity class has
interior nodes, which take the constant-stencil kernels; the closure nodes take the element
gather.

Tolerances: 1e-13 relative in FP64 and 2e-5 in FP32 (max-norm over inner DoFs); Dirichlet DoFs
are not written."""
import numpy as np
import pytest

import hyteg_b200 as hg
from tests import helpers as H

pytestmark = pytest.mark.gpu


def setup(nx, Lmax):
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    coords, tets, mesh, orc = H.cube(Lmax + 1, nx=nx)
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), nx, nx, nx, Lmax + 1)
    maps = {}
    for L in range(Lmax + 1):
        xyz, owned = mesh.slot_info(L + 1)
        maps[L] = (H.match_slots(xyz, orc.nodes(L + 1)[0]), owned)
    return st, orc, maps


@pytest.fixture(scope="module")
def cube2():
    return setup(2, 3)


@pytest.fixture(scope="module")
def cube3():
    return setup(3, 1)


def rel(a, b, m):
    return np.abs(a[m] - b[m]).max() / np.abs(b[m]).max()


def run_apply(env, L, dtype, residual, seed):
    st, orc, maps = env
    node, owned = maps[L]
    n = orc.n(L + 1)
    rng = np.random.default_rng(seed)
    u, f, d0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    Lmax = max(maps)
    A = hg.P2ConstantLaplaceOperator(st, 0, Lmax)
    x, b, y = (hg.P2Function(nm, st, 0, Lmax, dtype=dtype) for nm in ("x", "b", "y"))
    x.from_numpy(L, H.scatter(node, u).astype(dtype))
    b.from_numpy(L, H.scatter(node, f).astype(dtype))
    y.from_numpy(L, H.scatter(node, d0).astype(dtype))
    if residual:
        A.residual(x, b, y, L, hg.Inner)
    else:
        A.apply(x, y, L, hg.Inner)
    got = H.gather_owned(y.to_numpy(L).astype(np.float64), node, owned, n)
    uu = u.astype(dtype).astype(np.float64)
    ref = orc.p2_apply(L, uu)
    if residual:
        ref = f.astype(dtype).astype(np.float64) - ref
    inner = ~orc.dirichlet(L + 1)
    # copies of every DoF are consistent with its owner after the operation
    full = y.to_numpy(L).astype(np.float64)
    used = owned >= 0
    assert np.array_equal(full[used], got[node[used]])
    return got, ref, inner, d0.astype(dtype).astype(np.float64)


@pytest.mark.parametrize("L", [0, 1, 2, 3])
@pytest.mark.parametrize("residual", [False, True])
def test_p2_apply_fp64(cube2, L, residual):
    got, ref, inner, d0 = run_apply(cube2, L, np.float64, residual, 10 * L + residual)
    assert rel(got, ref, inner) < 1e-13
    assert np.array_equal(got[~inner], d0[~inner])


@pytest.mark.parametrize("L", [1, 3])
def test_p2_apply_fp32(cube2, L):
    got, ref, inner, _ = run_apply(cube2, L, np.float32, False, 77)
    assert rel(got, ref, inner) < 2e-5


@pytest.mark.parametrize("L", [0, 1])
def test_p2_apply_inner_vertices_and_edges(cube3, L):
    # the 3x3x3 cube has inner macro-vertices and inner macro-edges: sums over up to 24 cells
    got, ref, inner, _ = run_apply(cube3, L, np.float64, False, 5 + L)
    assert rel(got, ref, inner) < 1e-13


@pytest.mark.parametrize("L", [0, 1, 2, 3])
@pytest.mark.parametrize("backwards", [False, True])
def test_p2_multicolour_sor(cube2, L, backwards):
    st, orc, maps = cube2
    node, owned = maps[L]
    n = orc.n(L + 1)
    rng = np.random.default_rng(30 + L + 7 * backwards)
    u0, f0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    A = hg.P2ConstantLaplaceOperator(st, 0, 3)
    x, b = hg.P2Function("x", st, 0, 3), hg.P2Function("b", st, 0, 3)
    x.from_numpy(L, H.scatter(node, u0))
    b.from_numpy(L, H.scatter(node, f0))
    for _ in range(2):
        (A.smooth_sor_backwards if backwards else A.smooth_sor)(x, b, 0.8, L)
    got = H.gather_owned(x.to_numpy(L), node, owned, n)
    ref = orc.p2_sor(L, u0, f0, 0.8, sweeps=2, backwards=backwards)
    inner = ~orc.dirichlet(L + 1)
    assert rel(got, ref, inner) < 1e-13
    assert np.array_equal(got[~inner], u0[~inner])


def test_p2_sor_fp32(cube2):
    st, orc, maps = cube2
    L = 3
    node, owned = maps[L]
    n = orc.n(L + 1)
    rng = np.random.default_rng(99)
    u0, f0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    A = hg.P2ConstantLaplaceOperator(st, 0, 3)
    x, b = hg.P2Function("x", st, 0, 3, dtype=np.float32), hg.P2Function("b", st, 0, 3, dtype=np.float32)
    x.from_numpy(L, H.scatter(node, u0).astype(np.float32))
    b.from_numpy(L, H.scatter(node, f0).astype(np.float32))
    A.smooth_sor(x, b, 1.0, L)
    got = H.gather_owned(x.to_numpy(L).astype(np.float64), node, owned, n)
    ref = orc.p2_sor(L, u0.astype(np.float32).astype(np.float64), f0.astype(np.float32).astype(np.float64), 1.0)
    assert rel(got, ref, ~orc.dirichlet(L + 1)) < 2e-5


@pytest.mark.parametrize("Lc", [0, 1, 2])
@pytest.mark.parametrize("add", [False, True])
def test_p2_prolongation(cube2, Lc, add):
    st, orc, maps = cube2
    nc, nf = orc.n(Lc + 1), orc.n(Lc + 2)
    rng = np.random.default_rng(40 + Lc + 3 * add)
    c0, f0 = rng.uniform(-1, 1, nc), rng.uniform(-1, 1, nf)
    f = hg.P2Function("f", st, 0, 3)
    f.from_numpy(Lc, H.scatter(maps[Lc][0], c0))
    f.from_numpy(Lc + 1, H.scatter(maps[Lc + 1][0], f0))
    P = hg.P2toP2QuadraticProlongation()
    (P.prolongateAndAdd if add else P.prolongate)(f, Lc, hg.Inner)
    got = H.gather_owned(f.to_numpy(Lc + 1), maps[Lc + 1][0], maps[Lc + 1][1], nf)
    ref = orc.p2_prolongate(Lc, c0, f0, add=add)
    inner = ~orc.dirichlet(Lc + 2)
    assert rel(got, ref, inner) < 1e-13
    assert np.array_equal(got[~inner], f0[~inner])


@pytest.mark.parametrize("Lf", [1, 2, 3])
def test_p2_restriction(cube2, Lf):
    st, orc, maps = cube2
    nc, nf = orc.n(Lf), orc.n(Lf + 1)
    rng = np.random.default_rng(60 + Lf)
    fine = rng.uniform(-1, 1, nf)
    f = hg.P2Function("f", st, 0, 3)
    f.from_numpy(Lf, H.scatter(maps[Lf][0], fine))
    hg.P2toP2QuadraticRestriction().restrict(f, Lf, hg.Inner)
    got = H.gather_owned(f.to_numpy(Lf - 1), maps[Lf - 1][0], maps[Lf - 1][1], nc)
    ref = orc.p2_restrict(Lf, fine)
    inner = ~orc.dirichlet(Lf)
    assert rel(got, ref, inner) < 1e-13


def test_p2_multigrid_solves_to_oracle_solution(cube2):
    st, orc, maps = cube2
    L = 3
    node, owned = maps[L]
    n = orc.n(L + 1)
    rng = np.random.default_rng(123)
    bg = rng.uniform(-1, 1, n)
    inner = ~orc.dirichlet(L + 1)
    bg[~inner] = 0.0
    A = hg.P2ConstantLaplaceOperator(st, 0, 3)
    x, b = hg.P2Function("x", st, 0, 3), hg.P2Function("b", st, 0, 3)
    b.from_numpy(L, H.scatter(node, bg))
    gmg = hg.P2GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0)
    it, relres, hist = gmg.solve_to(x, b, L, 1e-10, 60)
    assert relres <= 1e-10
    factors = hist[1:] / hist[:-1]
    assert factors.max() < 0.6, factors
    ref = orc.p2_cg(L, np.zeros(n), bg, 20000, 1e-14)
    got = H.gather_owned(x.to_numpy(L), node, owned, n)
    assert rel(got, ref, inner) < 1e-8


@pytest.fixture(scope="module")
def cube2l4():
    return setup(2, 4)


@pytest.mark.parametrize("residual", [False, True])
def test_p2_apply_interior_stencils_level4(cube2l4, residual):
    # lattice 32 per macro-cell: most DoFs are interior and take the constant-stencil kernel
    got, ref, inner, d0 = run_apply(cube2l4, 4, np.float64, residual, 90 + residual)
    assert rel(got, ref, inner) < 1e-13
    assert np.array_equal(got[~inner], d0[~inner])


@pytest.mark.parametrize("backwards", [False, True])
def test_p2_multicolour_sor_level4(cube2l4, backwards):
    st, orc, maps = cube2l4
    L = 4
    node, owned = maps[L]
    n = orc.n(L + 1)
    rng = np.random.default_rng(300 + backwards)
    u0, f0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    A = hg.P2ConstantLaplaceOperator(st, 0, L)
    x, b = hg.P2Function("x", st, 0, L), hg.P2Function("b", st, 0, L)
    x.from_numpy(L, H.scatter(node, u0))
    b.from_numpy(L, H.scatter(node, f0))
    for _ in range(2):
        (A.smooth_sor_backwards if backwards else A.smooth_sor)(x, b, 0.9, L)
    got = H.gather_owned(x.to_numpy(L), node, owned, n)
    ref = orc.p2_sor(L, u0, f0, 0.9, sweeps=2, backwards=backwards)
    inner = ~orc.dirichlet(L + 1)
    assert rel(got, ref, inner) < 1e-13
    # copies of every DoF agree with its owner after the sweeps
    full = x.to_numpy(L)
    used = owned >= 0
    assert np.array_equal(full[used], got[node[used]])


def test_p2_graph_cycles_match_eager_cycles(cube2):
    # replayed CUDA graphs launch the same kernels, and every kernel of the cycle sums in a fixed
    # order (the restriction is a gather), so the two agree bit for bit
    st, orc, maps = cube2
    L = 3
    node, owned = maps[L]
    bg = np.random.default_rng(7).uniform(-1, 1, orc.n(L + 1))
    bg[orc.dirichlet(L + 1)] = 0.0
    out = []
    for graphs in (False, True):
        A = hg.P2ConstantLaplaceOperator(st, 0, 3)
        x, b = hg.P2Function("x", st, 0, 3), hg.P2Function("b", st, 0, 3)
        b.from_numpy(L, H.scatter(node, bg))
        gmg = hg.P2GeometricMultigridSolver(st, A, 0, L, 2, 2, 1.0)
        gmg.set_graphs(graphs)
        launches = []
        for _ in range(5):
            l0 = st.launch_count()
            gmg.solve(x, b, L)
            launches.append(st.launch_count() - l0)
        out.append((x.to_numpy(L), launches))
    (xe, le), (xg, lg) = out
    assert le == lg
    assert np.array_equal(xe, xg)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_p2_restriction_and_cycles_are_bit_reproducible(cube2, dtype):
    """The P2 restriction gathers each coarse value from its fine contributions in a fixed order,
    so repeated restrictions and repeated multigrid solves give identical bits."""
    st, orc, maps = cube2
    L = 3
    f = hg.P2Function("rf", st, 0, L, dtype=dtype)
    outs = []
    for _ in range(2):
        f.fill_random(17, L, hg.Inner)
        hg.P2toP2QuadraticRestriction().restrict(f, L, hg.Inner)
        outs.append(f.to_numpy(L - 1))
    assert np.array_equal(outs[0], outs[1])
    if dtype == np.float32:
        return
    res = []
    for _ in range(2):
        A = hg.P2ConstantLaplaceOperator(st, 0, L)
        x, b = hg.P2Function("x", st, 0, L), hg.P2Function("b", st, 0, L)
        b.fill_random(19, L, hg.Inner)
        gmg = hg.P2GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0)
        gmg.set_graphs(False)
        for _ in range(3):
            gmg.solve(x, b, L)
        res.append(x.to_numpy(L))
        del gmg, A
    assert np.array_equal(res[0], res[1])


def test_p2_multigrid_exact_coarse_solve_on_3x3x3_cube(cube3):
    # 125 unknowns on the coarsest P2 level: solved exactly through the inverse on the device
    st, orc, maps = cube3
    L = 1
    node, owned = maps[L]
    n = orc.n(L + 1)
    inner = ~orc.dirichlet(L + 1)
    assert (~orc.dirichlet(1)).sum() == 125
    bg = np.random.default_rng(11).uniform(-1, 1, n)
    bg[~inner] = 0.0
    A = hg.P2ConstantLaplaceOperator(st, 0, 1)
    x, b = hg.P2Function("x", st, 0, 1), hg.P2Function("b", st, 0, 1)
    b.from_numpy(L, H.scatter(node, bg))
    gmg = hg.P2GeometricMultigridSolver(st, A, 0, L, 2, 2, 1.0)
    it, relres, hist = gmg.solve_to(x, b, L, 1e-11, 40)
    assert relres <= 1e-11
    ref = orc.p2_cg(L, np.zeros(n), bg, 20000, 1e-14)
    got = H.gather_owned(x.to_numpy(L), node, owned, n)
    assert rel(got, ref, inner) < 1e-8
    # a two-level cycle whose coarse level is exact contracts strongly
    assert (hist[1:] / hist[:-1]).max() < 0.4

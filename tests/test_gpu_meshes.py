"""Device kernels on macro-meshes from meshCubedDomain and from Gmsh files, against the CPU oracle
built from the same vertices and tetrahedra.

Meshes: an L-shaped domain of three cubes with 24 tetrahedra each (cube type 1: face-centre and
cube-centre vertices, so vertices with up to 26 macro-edges), a 2 x 1 x 1 block of type-0 cubes,
and the type-1 mesh written as a Gmsh file with foreign node numbering and read back.
Tolerances as in the cube tests: FP64 1e-13 relative (max-norm over inner DoFs); the V-cycle
iterate 1e-12."""
import numpy as np
import pytest

import hyteg_b200 as hg
from tests import helpers as H
from tests.test_mesh_formats import write_shuffled

pytestmark = pytest.mark.gpu
LMAX = 3
L_SHAPE = [(0, 0, 0), (1, 0, 0), (0, 1, 0)]


def coords_tets(mesh):
    v, _, _, c = mesh.counts()
    coords = np.array([mesh.primitive(hg.VERTEX, i)[1] for i in range(v)])
    tets = np.array([mesh.primitive(hg.CELL, k)[0] for k in range(c)], dtype=np.int64)
    return coords, tets


@pytest.fixture(scope="module", params=["cubed1", "cubed0", "gmsh"])
def env(request, tmp_path_factory):
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    from oracle import oracle
    if request.param == "cubed1":
        st = hg.PrimitiveStorage.cubed_domain(L_SHAPE, 1, LMAX)
    elif request.param == "cubed0":
        st = hg.PrimitiveStorage.cubed_domain([(0, 0, 0), (1, 0, 0)], 0, LMAX)
    else:
        src = hg.HostMesh.cubed_domain(L_SHAPE, 1, 1)
        c, t = coords_tets(src)
        bnd = [tuple(src.primitive(hg.FACE, f)[0]) for f in range(src.counts()[2]) if src.primitive(hg.FACE, f)[2] == 1]
        path = tmp_path_factory.mktemp("msh") / "lshape.msh"
        write_shuffled(path, c, t, bnd, 11)
        st = hg.PrimitiveStorage.from_gmsh(path, LMAX)
    mesh = st.host()
    coords, tets = coords_tets(mesh)
    orc = oracle.Oracle(coords, tets, LMAX)
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


@pytest.mark.parametrize("L", [2, 3])
def test_apply(env, L):
    st, orc, maps = env
    n = orc.n(L)
    g = np.random.default_rng(L).uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    x, y = hg.P1Function("x", st, 0, LMAX), hg.P1Function("y", st, 0, LMAX)
    up(x, L, g, maps)
    A.apply(x, y, L, hg.Inner)
    inner = ~orc.dirichlet(L)
    assert relerr(down(y, L, maps, n), orc.apply(L, g), inner) < 1e-13


@pytest.mark.parametrize("L", [2, 3])
def test_multicolour_sor(env, L):
    st, orc, maps = env
    n = orc.n(L)
    rng = np.random.default_rng(10 + L)
    ug, fg = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    u, f = hg.P1Function("u", st, 0, LMAX), hg.P1Function("f", st, 0, LMAX)
    up(u, L, ug, maps)
    up(f, L, fg, maps)
    for _ in range(2):
        A.smooth_sor(u, f, 1.1, L, hg.Inner | hg.NeumannBoundary)
    ref = orc.sor(L, ug, fg, 1.1, 2, multicolour=True)
    assert relerr(down(u, L, maps, n), ref, np.ones(n, bool)) < 1e-13


def test_transfers(env):
    st, orc, maps = env
    Lf = LMAX
    nf, nc = orc.n(Lf), orc.n(Lf - 1)
    rng = np.random.default_rng(4)
    fine, coarse = rng.uniform(-1, 1, nf), rng.uniform(-1, 1, nc)
    r = hg.P1Function("r", st, 0, LMAX)
    up(r, Lf, fine, maps)
    hg.P1toP1LinearRestriction().restrict(r, Lf, hg.Inner)
    inner_c = ~orc.dirichlet(Lf - 1)
    assert relerr(down(r, Lf - 1, maps, nc), orc.restrict(Lf, fine), inner_c) < 1e-13
    p = hg.P1Function("p", st, 0, LMAX)
    up(p, Lf - 1, coarse, maps)
    hg.P1toP1LinearProlongation().prolongate(p, Lf - 1, hg.Inner)
    inner_f = ~orc.dirichlet(Lf)
    assert relerr(down(p, Lf, maps, nf), orc.prolongate(Lf - 1, coarse), inner_f) < 1e-13


def test_vcycles(env):
    st, orc, maps = env
    L = LMAX
    n = orc.n(L)
    rng = np.random.default_rng(8)
    bg = np.where(orc.dirichlet(L), 0.0, rng.uniform(-1, 1, n))
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    x, b = hg.P1Function("x", st, 0, LMAX), hg.P1Function("b", st, 0, LMAX)
    up(b, L, bg, maps)
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 10000, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3)
    for _ in range(2):
        gmg.solve(A, x, b, L)
    ref, _ = orc.gmg(L, 0, np.zeros(n), bg, 2, multicolour=True)
    inner = ~orc.dirichlet(L)
    assert relerr(down(x, L, maps, n), ref, inner) < 1e-12


@pytest.mark.parametrize("max_dofs", [6000, 10 ** 7])
def test_compact_coarse_cycle(env, max_dofs):
    """The compact coarse cycle builds on these meshes (an explicit request reports a failed
    build) and its V-cycles match the oracle's, up to the whole cycle in one launch."""
    st, orc, maps = env
    L = LMAX
    n = orc.n(L)
    rng = np.random.default_rng(9)
    bg = np.where(orc.dirichlet(L), 0.0, rng.uniform(-1, 1, n))
    A = hg.P1ConstantLaplaceOperator(st, 0, LMAX)
    x, b = hg.P1Function("x", st, 0, LMAX), hg.P1Function("b", st, 0, LMAX)
    up(b, L, bg, maps)
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 10000, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3)
    gmg.set_compact(A, max_dofs, 1)
    top = gmg.compact_top(A)
    assert top >= 1 and (max_dofs < 10 ** 7 or top == L)
    for _ in range(2):
        gmg.solve(A, x, b, L)
    ref, _ = orc.gmg(L, 0, np.zeros(n), bg, 2, multicolour=True)
    assert relerr(down(x, L, maps, n), ref, ~orc.dirichlet(L)) < 1e-12

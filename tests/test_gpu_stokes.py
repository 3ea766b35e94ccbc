"""P2-P1 Taylor-Hood Stokes on the 48-tet cube: block apply against the oracle's assembled
operator (1e-13 relative), and MINRES with the block-diagonal multigrid preconditioner on a
lid-driven cavity (u = (1, 0, 0) on z = 1, no slip elsewhere) against a dense solve of the
oracle's system (velocity to 1e-7 relative; pressure to 1e-6 relative up to a constant, on the
pressure DoFs coupled to at least one free velocity DoF: a pressure DoF whose micro-cells all
have Dirichlet velocity DoFs only is a spurious mode of the discrete system and undetermined)."""
import numpy as np
import pytest

import hyteg_b200 as hg
from tests import helpers as H

pytestmark = pytest.mark.gpu
LMAX = 2  # P2 levels 0..2: velocity lattices 1..3, pressure lattices 0..2


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


def funcs(st):
    u = [hg.P2Function("u%d" % k, st, 0, LMAX) for k in range(3)]
    p = hg.P1Function("p", st, 0, LMAX)
    return u, p


def rel(a, b, m):
    return np.abs(a[m] - b[m]).max() / np.abs(b[m]).max()


@pytest.mark.parametrize("L", [0, 1, 2])
def test_stokes_apply(env, L):
    st, orc, maps = env
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, LMAX)
    nv, np_ = orc.n(L + 1), orc.n(L)
    rng = np.random.default_rng(70 + L)
    uu = [rng.uniform(-1, 1, nv) for _ in range(3)]
    pp = rng.uniform(-1, 1, np_)
    u, p = funcs(st)
    v, q = funcs(st)
    for k in range(3):
        u[k].from_numpy(L, H.scatter(maps[L + 1][0], uu[k]))
        v[k].from_numpy(L, np.zeros(st.level_size(L + 1)))
    p.from_numpy(L, H.scatter(maps[L][0], pp))
    S.apply(u, p, v, q, L)
    vr, qr = orc.stokes_apply(L, uu, pp)
    inner = ~orc.dirichlet(L + 1)
    for k in range(3):
        got = H.gather_owned(v[k].to_numpy(L), maps[L + 1][0], maps[L + 1][1], nv)
        assert rel(got, vr[k], inner) < 1e-13
        assert np.all(got[~inner] == 0.0)
    gq = H.gather_owned(q.to_numpy(L), maps[L][0], maps[L][1], np_)
    assert rel(gq, qr, np.ones(np_, dtype=bool)) < 1e-13


def dense_lid_solution(orc, L):
    nv, np_ = orc.n(L + 1), orc.n(L)
    xyz = orc.nodes(L + 1)[0]
    dv = orc.dirichlet(L + 1)
    lid = np.where(dv & (np.abs(xyz[:, 2] - 1.0) < 1e-12), 1.0, 0.0)
    uD = [lid, np.zeros(nv), np.zeros(nv)]
    vD, qD = orc.stokes_apply(L, uD, np.zeros(np_))
    free = np.where(~dv)[0]
    nf = len(free)
    n = 3 * nf + np_

    def unpack(x):
        u = [np.zeros(nv) for _ in range(3)]
        for k in range(3):
            u[k][free] = x[k * nf:(k + 1) * nf]
        return u, x[3 * nf:]

    K = np.zeros((n, n))
    for c in range(n):
        e = np.zeros(n)
        e[c] = 1.0
        u, p = unpack(e)
        v, q = orc.stokes_apply(L, u, p)
        K[:, c] = np.concatenate([v[0][free], v[1][free], v[2][free], q])
    rhs = -np.concatenate([vD[0][free], vD[1][free], vD[2][free], qD])
    x = np.linalg.lstsq(K, rhs, rcond=None)[0]
    u, p = unpack(x)
    u[0] += lid
    coupled = np.abs(K[:3 * nf, 3 * nf:]).max(axis=0) > 0
    return u, p, coupled


def test_minres_lid_driven_cavity(env):
    st, orc, maps = env
    L = 1
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, LMAX)
    u, p = funcs(st)
    f, g = funcs(st)
    xyz = maps[L + 1][2]
    lid = np.where(np.abs(xyz[:, 2] - 1.0) < 1e-12, 1.0, 0.0)
    u[0].from_numpy(L, lid)  # interior values are overwritten by the solve; boundary = lid
    it, relres, hist = S.minres(u, p, f, g, L, nu=2, max_iter=300, tol=1e-11)
    assert relres <= 1e-11, (it, relres)
    ur, pr, coupled = dense_lid_solution(orc, L)
    assert coupled.sum() > 0.9 * len(coupled)
    nv, np_ = orc.n(L + 1), orc.n(L)
    for k in range(3):
        got = H.gather_owned(u[k].to_numpy(L), maps[L + 1][0], maps[L + 1][1], nv)
        scale = max(np.abs(ur[0]).max(), 1.0)
        assert np.abs(got - ur[k]).max() / scale < 1e-7
    gp = H.gather_owned(p.to_numpy(L), maps[L][0], maps[L][1], np_)
    d = gp[coupled] - pr[coupled]
    assert np.abs(d - d.mean()).max() / np.abs(pr[coupled]).max() < 1e-6


def test_minres_converges_on_level_2(env):
    st, orc, maps = env
    L = 2
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, LMAX)
    u, p = funcs(st)
    f, g = funcs(st)
    xyz = maps[L + 1][2]
    u[0].from_numpy(L, np.where(np.abs(xyz[:, 2] - 1.0) < 1e-12, 1.0, 0.0))
    it, relres, hist = S.minres(u, p, f, g, L, nu=2, max_iter=300, tol=1e-8)
    assert relres <= 1e-8 and it < 150, (it, relres)
    # the discrete equations hold: A u + D^T p = 0 at inner velocity DoFs and D u = 0
    v, q = funcs(st)
    S.apply(u, p, v, q, L)
    for k in range(3):
        vv = v[k].to_numpy(L)
        assert np.abs(vv[maps[L + 1][1] == 1]).max() < 1e-6
    assert np.abs(q.to_numpy(L)).max() < 1e-6


def test_minres_with_fp32_preconditioner_matches_fp64(env):
    st, orc, maps = env
    L = 2
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, LMAX)
    xyz = maps[L + 1][2]
    lid = np.where(np.abs(xyz[:, 2] - 1.0) < 1e-12, 1.0, 0.0)
    out = {}
    for dt in (np.float64, np.float32):
        u, p = funcs(st)
        f, g = funcs(st)
        u[0].from_numpy(L, lid)
        it, relres, _ = S.minres(u, p, f, g, L, nu=2, max_iter=300, tol=1e-10, precondition_dtype=dt)
        assert relres <= 1e-10
        out[dt] = (it, [x.to_numpy(L) for x in u], p.to_numpy(L))
    (i64, u64, p64), (i32, u32, p32) = out[np.float64], out[np.float32]
    assert i32 <= i64 + 10
    m = maps[L + 1][1] == 1
    for k in range(3):
        assert np.abs(u32[k][m] - u64[k][m]).max() < 1e-8
    mp = maps[L][1] == 1
    assert np.abs(p32[mp] - p64[mp]).max() / np.abs(p64[mp]).max() < 1e-7


@pytest.fixture(scope="module")
def env3():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    coords, tets, mesh, orc = H.cube(4)
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, 4)
    maps = {}
    for L in (3, 4):
        xyz, owned = mesh.slot_info(L)
        maps[L] = (H.match_slots(xyz, orc.nodes(L)[0]), owned, xyz)
    return st, orc, maps


def test_stokes_apply_level3_interior_stencils(env3):
    # pressure lattice 8, velocity lattice 16 per macro-cell: most nodes take the interior
    # div / divT stencils, the closure nodes the per-node gathers from the closure lists
    st, orc, maps = env3
    L = 3
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, L)
    nv, np_ = orc.n(L + 1), orc.n(L)
    rng = np.random.default_rng(313)
    uu = [rng.uniform(-1, 1, nv) for _ in range(3)]
    pp = rng.uniform(-1, 1, np_)
    u = [hg.P2Function("u%d" % k, st, 0, L) for k in range(3)]
    v = [hg.P2Function("v%d" % k, st, 0, L) for k in range(3)]
    p, q = hg.P1Function("p", st, 0, L), hg.P1Function("q", st, 0, L)
    for k in range(3):
        u[k].from_numpy(L, H.scatter(maps[L + 1][0], uu[k]))
        v[k].from_numpy(L, np.zeros(st.level_size(L + 1)))
    p.from_numpy(L, H.scatter(maps[L][0], pp))
    S.apply(u, p, v, q, L)
    vr, qr = orc.stokes_apply(L, uu, pp)
    inner = ~orc.dirichlet(L + 1)
    for k in range(3):
        got = H.gather_owned(v[k].to_numpy(L), maps[L + 1][0], maps[L + 1][1], nv)
        assert rel(got, vr[k], inner) < 1e-13
    gq = H.gather_owned(q.to_numpy(L), maps[L][0], maps[L][1], np_)
    assert rel(gq, qr, np.ones(np_, dtype=bool)) < 1e-13


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_minres_concurrent_components_match_in_order(env, dtype):
    """The three velocity V-cycles of each preconditioner application on three streams give the
    iterates of the same cycles one after another, bit for bit (FP64 and FP32 cycles)."""
    st, orc, maps = env
    L = LMAX
    S = hg.P2P1TaylorHoodStokesOperator(st, 0, LMAX)
    xyz = maps[L + 1][2]
    lid = np.where(np.abs(xyz[:, 2] - 1.0) < 1e-12, 1.0, 0.0)
    out = []
    for concurrent in (False, True, True):
        st.set_concurrent_components(concurrent)
        u, p = funcs(st)
        f, g = funcs(st)
        u[0].from_numpy(L, lid)
        it, relres, hist = S.minres(u, p, f, g, L, nu=2, max_iter=40, tol=1e-10, precondition_dtype=dtype)
        out.append((it, relres, hist, [uk.to_numpy(L) for uk in u], p.to_numpy(L)))
    st.set_concurrent_components(True)
    for o in out[1:]:
        assert o[0] == out[0][0] and o[1] == out[0][1] and np.array_equal(o[2], out[0][2])
        for k in range(3):
            assert np.array_equal(o[3][k], out[0][3][k])
        assert np.array_equal(o[4], out[0][4])

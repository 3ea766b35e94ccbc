"""The CPU oracle pinned against the reference itself: its generated kernels and FEniCS forms
compiled from the reference sources (oracle/_ref), its mesh fixtures (tests/golden/meshes.json)
and the bound of its GMG convergence test. Arrays handed to the reference kernels are built
here from the reference layout (index functions of indexing/MacroCellIndexing.hpp:40-52 and
p1functionspace/VertexDoFIndexing.cpp:205-225), independently of the product."""
import json
import os

import numpy as np
import pytest
from scipy.spatial import cKDTree

from tests import helpers as H

HERE = os.path.dirname(os.path.abspath(__file__))
OFF15 = H.CELL_OFF


def meshes():
    with open(os.path.join(HERE, "golden", "meshes.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def cube():
    from oracle import oracle
    coords, tets = oracle.cuboid_mesh((0, 0, 0), (1, 1, 1), 2, 2, 2)
    L = 4
    o = oracle.Oracle(coords, tets, L)
    order = sorted(range(len(tets)), key=lambda i: list(tets[i]))
    cells = [list(tets[i]) for i in order]  # creation order of the macro-cells
    return coords, cells, o, L


def lookup(o, L):
    xyz = o.nodes(L)[0]
    return cKDTree(xyz)


def cell_points(N):
    return np.array([(x, y, z) for z in range(N + 1) for y in range(N + 1 - z) for x in range(N + 1 - y - z)])


def cell_array(coords, cell, o, tree, L, g):
    """Reference cell array (tet(w) values, x fastest) of global vector g."""
    N = 2 ** L
    V = coords[cell]
    p = cell_points(N)
    xyz = V[0] + (np.outer(p[:, 0], V[1] - V[0]) + np.outer(p[:, 1], V[2] - V[0]) + np.outer(p[:, 2], V[3] - V[0])) / N
    d, node = tree.query(xyz)
    assert d.max() < 1e-12
    idx = H.cell_idx(N + 1, p[:, 0], p[:, 1], p[:, 2])
    a = np.zeros(H.tet(N + 1))
    a[idx] = g[node]
    return a, idx, node, p


def test_element_matrices_match_reference_forms(ref, oracle_mod):
    rng = np.random.default_rng(0)
    for _ in range(20):
        P = rng.uniform(-1, 1, (4, 3))
        c = np.ascontiguousarray(P.reshape(12))
        K = np.zeros(16)
        ref.ref_p1_tet_diffusion(oracle_mod.dp(c), oracle_mod.dp(K))
        assert np.allclose(oracle_mod.element_laplace(P), K.reshape(4, 4), rtol=1e-12, atol=1e-13 * np.abs(K).max())
        ref.ref_p1_tet_mass(oracle_mod.dp(c), oracle_mod.dp(K))
        assert np.allclose(oracle_mod.element_mass(P), K.reshape(4, 4), rtol=1e-12, atol=1e-15)


def test_cell_apply_matches_reference_kernel(cube, ref, oracle_mod):
    coords, cells, o, L = cube
    tree = lookup(o, L)
    g = np.random.default_rng(1).uniform(-1, 1, o.n(L))
    y = o.apply(L, g)
    N = 2 ** L
    for c in (0, 13, 47):
        src, idx, node, p = cell_array(coords, cells[c], o, tree, L, g)
        w = o.cell_local_stencil(L, c, 1, 1, 1)
        dst = np.zeros_like(src)
        ref.ref_apply_cell(oracle_mod.dp(dst), oracle_mod.dp(src), L, oracle_mod.dp(w), 0)
        inner = (p.min(axis=1) >= 1) & (p.sum(axis=1) <= N - 1)
        assert np.abs(dst[idx[inner]] - y[node[inner]]).max() < 1e-14 * np.abs(y).max()


def test_cell_sor_matches_reference_kernel(cube, ref, oracle_mod):
    coords, cells, o, L = cube
    tree = lookup(o, L)
    rng = np.random.default_rng(2)
    u, f = rng.uniform(-1, 1, o.n(L)), rng.uniform(-1, 1, o.n(L))
    u1 = o.sor_phases(L, u, f, 1.3, 1 << 3)  # cell phase of a lexicographic sweep
    N = 2 ** L
    for c in (0, 29, 47):
        a, idx, node, p = cell_array(coords, cells[c], o, tree, L, u)
        fa, _, _, _ = cell_array(coords, cells[c], o, tree, L, f)
        w = o.cell_local_stencil(L, c, 1, 1, 1)
        ref.ref_sor_cell(oracle_mod.dp(a), oracle_mod.dp(fa), L, oracle_mod.dp(w), 1.3)
        inner = (p.min(axis=1) >= 1) & (p.sum(axis=1) <= N - 1)
        assert np.abs(a[idx[inner]] - u1[node[inner]]).max() < 1e-13


def test_face_apply_matches_reference_kernel(cube, ref, oracle_mod):
    coords, cells, o, L = cube
    tree = lookup(o, L)
    N, w = 2 ** L, 2 ** L + 1
    g = np.random.default_rng(3).uniform(-1, 1, o.n(L))
    y = o.apply(L, g)
    faces = {}
    for ci, cv in enumerate(cells):
        for tri in ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)):
            faces.setdefault(tuple(sorted(cv[t] for t in tri)), []).append(ci)
    inner_faces = [f for f, cs in faces.items() if len(cs) == 2][:6]
    fp = np.array([(x, yy) for yy in range(w) for x in range(w - yy)])
    gp = np.array([(x, yy) for yy in range(w - 1) for x in range(w - 1 - yy)])
    for fv in inner_faces:
        V = coords[list(fv)]
        xyz = V[0] + (np.outer(fp[:, 0], V[1] - V[0]) + np.outer(fp[:, 1], V[2] - V[0])) / N
        face = np.zeros(H.tri(w))
        d, node = tree.query(xyz)
        face[H.face_idx(w, fp[:, 0], fp[:, 1])] = g[node]
        dst = np.zeros(H.tri(w))
        for k, ci in enumerate(faces[fv]):
            cv = cells[ci]
            opp = [v for v in cv if v not in fv][0]
            gxyz = (np.outer(N - gp[:, 0] - gp[:, 1] - 1, V[0]) + np.outer(gp[:, 0], V[1]) + np.outer(gp[:, 1], V[2]) +
                    coords[opp]) / N
            dg, gnode = tree.query(gxyz)
            assert dg.max() < 1e-12
            ghost = np.zeros(H.tri(w - 1))
            ghost[H.face_idx(w - 1, gp[:, 0], gp[:, 1])] = g[gnode]
            lv = [cv.index(v) for v in fv]  # cell-local vertex IDs of the face's vertices
            # face point (1, 1) in cell-local coordinates
            b = np.zeros(4)
            b[lv[0]], b[lv[1]], b[lv[2]] = N - 2, 1, 1
            cp = (int(b[1]), int(b[2]), int(b[3]))
            wst = o.cell_local_stencil(L, ci, cp[0], cp[1], cp[2])
            present = np.array([all(v >= 0 for v in (cp[0] + dd[0], cp[1] + dd[1], cp[2] + dd[2])) and
                                sum(cp) + sum(dd) <= N for dd in OFF15], dtype=np.int32)
            ref.ref_apply_face(oracle_mod.dp(dst), oracle_mod.dp(face), oracle_mod.dp(ghost), L, lv[0], lv[1], lv[2],
                               oracle_mod.dp(wst), present.ctypes.data_as(oracle_mod.P(oracle_mod.c_int)), k)
        inner = (fp.min(axis=1) >= 1) & (fp.sum(axis=1) <= N - 1)
        got = dst[H.face_idx(w, fp[inner, 0], fp[inner, 1])]
        assert np.abs(got - y[node[inner]]).max() < 1e-14 * np.abs(y).max()


def _cell_counts(cells):
    from collections import Counter
    ec, fc, vc = Counter(), Counter(), Counter()
    for cv in cells:
        for a in range(4):
            vc[cv[a]] += 1
            for b in range(a + 1, 4):
                ec[tuple(sorted((cv[a], cv[b])))] += 1
        for tri in ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)):
            fc[tuple(sorted(cv[t] for t in tri))] += 1
    return ec, fc, vc


def _nbr(cv, ec, fc, vc):
    ep = [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (2, 3)]
    fp = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]
    nE = np.array([ec[tuple(sorted((cv[a], cv[b])))] for a, b in ep], dtype=np.float64)
    nF = np.array([fc[tuple(sorted(cv[t] for t in tr))] for tr in fp], dtype=np.float64)
    nV = np.array([vc[v] for v in cv], dtype=np.float64)
    return nE, nF, nV


def test_restriction_matches_reference_kernels(cube, ref, oracle_mod):
    coords, cells, o, L = cube
    tf, tc = lookup(o, L), lookup(o, L - 1)
    g = np.random.default_rng(4).uniform(-1, 1, o.n(L))
    ec, fc, vc = _cell_counts(cells)
    acc = np.zeros(o.n(L - 1))
    for ci, cv in enumerate(cells):
        fine, _, _, _ = cell_array(coords, cv, o, tf, L, g)
        coarse0, idxc, nodec, pc = cell_array(coords, cv, o, tc, L - 1, np.zeros(o.n(L - 1)))
        nE, nF, nV = _nbr(cv, ec, fc, vc)
        coarse = np.zeros_like(coarse0)
        ref.ref_restrict_cell(oracle_mod.dp(coarse), oracle_mod.dp(fine), L - 1, oracle_mod.dp(nE), oracle_mod.dp(nF),
                              oracle_mod.dp(nV))
        np.add.at(acc, nodec, coarse[idxc])  # additive communication into the owners
    ref_r = o.restrict(L, g)
    inner = ~o.dirichlet(L - 1)
    assert np.abs(acc[inner] - ref_r[inner]).max() < 1e-13 * np.abs(ref_r).max()


def test_prolongation_matches_reference_kernels(cube, ref, oracle_mod):
    coords, cells, o, L = cube
    tf, tc = lookup(o, L), lookup(o, L - 1)
    g = np.random.default_rng(5).uniform(-1, 1, o.n(L - 1))
    ec, fc, vc = _cell_counts(cells)
    acc = np.zeros(o.n(L))
    for ci, cv in enumerate(cells):
        coarse, _, _, _ = cell_array(coords, cv, o, tc, L - 1, g)
        fine0, idxf, nodef, _ = cell_array(coords, cv, o, tf, L, np.zeros(o.n(L)))
        nE, nF, nV = _nbr(cv, ec, fc, vc)
        fine = np.zeros_like(fine0)
        ref.ref_prolongate_cell(oracle_mod.dp(coarse), oracle_mod.dp(fine), L - 1, oracle_mod.dp(nE), oracle_mod.dp(nF),
                                oracle_mod.dp(nV))
        np.add.at(acc, nodef, fine[idxf])
    ref_p = o.prolongate(L - 1, g)
    inner = ~o.dirichlet(L)
    assert np.abs(acc[inner] - ref_p[inner]).max() < 1e-13


@pytest.mark.parametrize("name", ["tet_1el", "pyramid_2el", "pyramid_4el", "pyramid_tilted_4el",
                                  "regular_octahedron_8el", "cube_6el"])
def test_laplace_annihilates_constants_and_linears_on_reference_meshes(name, oracle_mod):
    # P1LaplaceOperator3DTest.cpp:40-150 (2.8e-13 discrete L2)
    m = meshes()[name]
    o = oracle_mod.Oracle(np.array(m["coords"]), np.array(m["tets"], dtype=np.int32), 3)
    for L in (2, 3):
        xyz, info = o.nodes(L)
        inner = info[:, 2] == 0
        for u in (np.ones(len(xyz)), xyz[:, 0], xyz[:, 0] + xyz[:, 1] - 2 * xyz[:, 2]):
            y = o.apply(L, u)
            assert np.sqrt((y[inner] ** 2).mean()) < 2.8e-13


@pytest.mark.parametrize("multicolour", [False, True])
def test_gmg_convergence_bound_of_reference_test(multicolour, oracle_mod):
    # P1GMG3DConvergenceTest.cpp:44-157: octahedron, levels 0..3, V(3,3) Gauss-Seidel, CG coarse,
    # u = sin(x) sinh(y) z on the boundary, random inside, f = 0: squared residual ratio < 3.2e-2
    m = meshes()["regular_octahedron_8el"]
    L = 3
    o = oracle_mod.Oracle(np.array(m["coords"]), np.array(m["tets"], dtype=np.int32), L)
    xyz, info = o.nodes(L)
    d = info[:, 2].astype(bool)
    exact = np.sin(xyz[:, 0]) * np.sinh(xyz[:, 1]) * xyz[:, 2]
    u = np.where(d, exact, np.random.default_rng(0).uniform(0, 1, len(d)))
    f = np.zeros(len(d))

    def res2(u):
        r = o.apply(L, u)
        return (r[~d] ** 2).sum() / (~d).sum()

    last = res2(u)
    for _ in range(10):
        u, _ = o.gmg(L, 0, u, f, 1, 3, 3, 1.0, multicolour=multicolour)
        r = res2(u)
        assert r / last < 3.2e-2
        last = r


def test_p2_element_matches_reference_form(ref, oracle_mod):
    # p2_tet_diffusion of the reference's FEniCS forms; UFC numbers the edges
    # (2,3),(1,3),(1,2),(0,3),(0,2),(0,1), the oracle (0,1),(0,2),(0,3),(1,2),(1,3),(2,3)
    perm = [0, 1, 2, 3, 9, 8, 7, 6, 5, 4]
    rng = np.random.default_rng(12)
    for _ in range(5):
        c = rng.uniform(-1, 1, (4, 3))
        K = oracle_mod.p2_element_laplace(c)
        R = np.zeros(100)
        ref.ref_p2_tet_diffusion(oracle_mod.dp(np.ascontiguousarray(c.reshape(12))), oracle_mod.dp(R))
        R = R.reshape(10, 10)[np.ix_(perm, perm)]
        assert np.abs(K - R).max() <= 1e-13 * np.abs(R).max()


@pytest.mark.parametrize("name", ["regular_octahedron_8el", "pyramid_4el", "pyramid_tilted_4el"])
def test_p2_laplace_annihilates_constants_and_linears(name, oracle_mod):
    m = meshes()[name]
    L = 2
    o = oracle_mod.Oracle(np.array(m["coords"]), np.array(m["tets"], dtype=np.int32), L + 1)
    xyz, info = o.nodes(L + 1)
    inner = ~info[:, 2].astype(bool)
    for u in (np.ones(len(xyz)), 1.0 + 2.0 * xyz[:, 0] - xyz[:, 1] + 0.5 * xyz[:, 2]):
        y = o.p2_apply(L, u)
        assert np.abs(y[inner]).max() < 1e-12
    rng = np.random.default_rng(1)
    a, b = rng.uniform(-1, 1, len(xyz)), rng.uniform(-1, 1, len(xyz))
    assert abs(a @ o.p2_apply(L, b) - b @ o.p2_apply(L, a)) < 1e-11


def test_p2p1_divergence_element_matches_reference_forms(ref, oracle_mod):
    # p2_to_p1_tet_div_tet (div) and p1_to_p2_tet_divt_tet (its transpose) of the reference's forms
    perm = [0, 1, 2, 3, 9, 8, 7, 6, 5, 4]
    rng = np.random.default_rng(13)
    for _ in range(4):
        c = rng.uniform(-1, 1, (4, 3))
        D = oracle_mod.p2p1_div_element(c)
        cc = np.ascontiguousarray(c.reshape(12))
        for k in range(3):
            A = np.zeros(40)
            ref.ref_p2_to_p1_div(oracle_mod.dp(cc), k, oracle_mod.dp(A))
            A = A.reshape(4, 10)[:, perm]
            B = np.zeros(40)
            ref.ref_p1_to_p2_divt(oracle_mod.dp(cc), k, oracle_mod.dp(B))
            B = B.reshape(10, 4)[perm, :]
            assert np.abs(D[k] - A).max() <= 1e-13 * np.abs(A).max()
            assert np.abs(D[k].T - B).max() <= 1e-13 * np.abs(B).max()


def test_pspg_element_matches_reference_form(ref, oracle_mod):
    # p1_tet_pspg_tet: -tau grad p . grad q, tau = |T|^(2/3) / 12 (the Uzawa smoother's pressure scaling)
    rng = np.random.default_rng(17)
    for _ in range(10):
        c = np.ascontiguousarray(rng.uniform(-1, 1, (4, 3)).reshape(12))
        K = np.zeros(16)
        ref.ref_p1_tet_pspg(oracle_mod.dp(c), oracle_mod.dp(K))
        mine = np.zeros(16)
        oracle_mod.lib().orc_element_pspg(oracle_mod.dp(c), oracle_mod.dp(mine))
        assert np.abs(mine - K).max() <= 1e-13 * np.abs(K).max()


def test_pspg_diagonal_is_the_element_sum(oracle_mod):
    # the diagonal of the assembled PSPG matrix: on the uniformly refined unit cube every micro-cell
    # of level L has volume 1 / (48 8^L) and tau = vol^(2/3) / 12, so diag = -tau * Laplace diagonal
    coords, tets = oracle_mod.cuboid_mesh((0, 0, 0), (1, 1, 1), 2, 2, 2)
    o = oracle_mod.Oracle(coords, tets, 2)
    for L in (1, 2):
        vol = 1.0 / (48 * 8 ** L)
        tau = vol ** (2.0 / 3.0) / 12.0
        n = o.n(L)
        lap = np.array([o.apply(L, np.eye(1, n, i)[0])[i] for i in range(n)])
        inner = ~o.dirichlet(L)
        assert np.allclose(o.pspg_diag(L)[inner], -tau * lap[inner], rtol=1e-12)

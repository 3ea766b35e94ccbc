"""Host-side tables of the product (layout, halo groups, stencils) against the oracle, on CPU.

The product's exported tables are evaluated with numpy and compared with the oracle's
assembled operator; no device code is involved here (the device kernels are compared with the
oracle in the -m gpu tests)."""
import numpy as np
import pytest

import hyteg_b200 as hg
from tests import helpers as H


@pytest.fixture(scope="module")
def cube4():
    return H.cube(4)


def test_counts_and_sizes(cube4):
    _, _, mesh, orc = cube4
    assert mesh.counts() == (27, 98, 120, 48)
    # level buffer: per-primitive sizes of the reference (VertexDoFMemory.hpp:44-69)
    L = 3
    w = 2 ** L + 1
    for f in range(120):
        ncell = len(mesh.neighbours(hg.FACE, f, hg.CELL))
        assert mesh.layout(L, hg.FACE, f)[1] == H.tri(w) + ncell * H.tri(w - 1)
    for e in range(98):
        nf = len(mesh.neighbours(hg.EDGE, e, hg.FACE))
        nc = len(mesh.neighbours(hg.EDGE, e, hg.CELL))
        assert mesh.layout(L, hg.EDGE, e)[1] == w + nf * (w - 1) + nc * (w - 2)
    for v in range(27):
        assert mesh.layout(L, hg.VERTEX, v)[1] == 1 + len(mesh.neighbours(hg.VERTEX, v, hg.EDGE))
    for c in range(48):
        assert mesh.layout(L, hg.CELL, c)[1] == H.tet(w)


@pytest.mark.parametrize("L", [0, 1, 2, 3, 4])
def test_slots_cover_every_dof_once(cube4, L):
    _, _, mesh, orc = cube4
    xyz, owned = mesh.slot_info(L)
    node = H.match_slots(xyz[owned >= 0], orc.nodes(L)[0])
    assert (node >= 0).all(), "every slot holds a micro-vertex of the mesh"
    own_nodes = node[owned[owned >= 0] == 1]
    assert len(own_nodes) == orc.n(L) and len(np.unique(own_nodes)) == orc.n(L)


@pytest.mark.parametrize("L", [1, 2, 3, 4])
def test_halo_tables_copy_the_same_dof(cube4, L):
    _, _, mesh, orc = cube4
    xyz, owned = mesh.slot_info(L)
    total = 0
    for g in range(5):
        dst, src = mesh.halo_table(L, g)
        total += len(dst)
        assert np.allclose(xyz[dst], xyz[src], atol=1e-12)
        assert (owned[src] == 1).all() and (owned[dst] == 0).all()
    assert total == int((owned == 0).sum()), "every copy slot is refreshed by exactly one table entry"


@pytest.mark.parametrize("L", [2, 3, 4])
@pytest.mark.parametrize("form", [0, 1])
def test_stencil_tables_reproduce_oracle_operator(cube4, L, form):
    _, _, mesh, orc = cube4
    xyz, owned = mesh.slot_info(L)
    node = H.match_slots(xyz, orc.nodes(L)[0])
    rng = np.random.default_rng(42 + L)
    g = rng.uniform(-1, 1, orc.n(L))
    u = H.scatter(node, g)
    y = H.tables_apply(mesh, L, form, u, hg.Inner)
    ref = orc.apply(L, g, form=form)
    inner = ~orc.dirichlet(L)
    got = H.gather_owned(y, node, owned, orc.n(L))
    err = np.abs(got[inner] - ref[inner]).max() / np.abs(ref[inner]).max()
    assert err < 1e-13, err


def test_stencil_annihilates_constants_and_linears(cube4):
    # P1LaplaceOperator3DTest.cpp:40-150: A u = 0 for u = const and u linear (inner DoFs)
    _, _, mesh, orc = cube4
    L = 3
    xyz, owned = mesh.slot_info(L)
    for fn in (lambda x, y, z: 1.0 + 0 * x, lambda x, y, z: x, lambda x, y, z: x + 2 * y - 3 * z + 1):
        u = fn(xyz[:, 0], xyz[:, 1], xyz[:, 2])
        y = H.tables_apply(mesh, L, 0, u, hg.Inner)
        assert np.abs(y[owned == 1]).max() < 1e-12


def test_cell_stencil_scales_with_h_and_sums_to_zero(cube4):
    # VertexDoFStencilAssemblyTest.cpp:53-235: row sum 0, w(L-1) = 2 w(L) for the Laplacian
    _, _, mesh, _ = cube4
    for c in (0, 17, 47):
        w3 = mesh.cell_stencil(3, 0, c)
        w4 = mesh.cell_stencil(4, 0, c)
        assert abs(w4.sum()) < 1e-13 * abs(w4[0])
        assert np.allclose(w3, 2 * w4, rtol=1e-13, atol=1e-15)

"""The union macro-mesh of the solve server's batched solves (hg_mesh_create_cuboid_copies):
`copies` disjoint copies of the k^3 cube in one storage. Batching relies on its layout: every
kind of primitive (cells, faces, edges, vertices, in the level buffer's order) holds the copies'
primitives copy after copy, each copy's block laid out exactly as a single cube's primitives of
that kind, so a slot of copy i sits at the union's first slot of the kind + i * (slots of one
copy's block) + (its offset in a single cube's block). Checked on the host for every level,
primitive by primitive: offsets, sizes, vertex lists (shifted by the copy's vertex offset),
boundary flags and vertex positions."""
import numpy as np
import pytest

import hyteg_b200 as hg

KINDS = (hg.CELL, hg.FACE, hg.EDGE, hg.VERTEX)  # the order of the kinds in a level buffer


@pytest.mark.parametrize("k,copies", [(1, 3), (2, 2), (3, 4)])
def test_union_layout_is_the_copies_back_to_back(k, copies):
    Lmax = 3
    one = hg.HostMesh.cuboid((0, 0, 0), (1, 1, 1), k, k, k, Lmax)
    uni = hg.HostMesh.cuboid_copies(k, copies, Lmax)
    c1, cu = one.counts(), uni.counts()
    assert list(cu) == [copies * c for c in c1]
    nv = c1[0]
    for L in range(Lmax + 1):
        a_base = 0
        for kind in KINDS:
            n = c1[kind]
            u_first = uni.layout(L, kind, 0)[0]
            a_first = one.layout(L, kind, 0)[0]
            # the single cube's block of this kind starts where its earlier kinds end
            assert a_first == a_base
            ends = [one.layout(L, kind, p)[0] + one.layout(L, kind, p)[1] for p in range(n)]
            block = (one.layout(L, KINDS[KINDS.index(kind) + 1], 0)[0] if kind != hg.VERTEX else one.level_size(L)) - a_first
            assert block >= max(ends) - a_first
            for i in range(copies):
                for p in range(n):
                    ao, asz = one.layout(L, kind, p)
                    uo, usz = uni.layout(L, kind, i * n + p)
                    assert usz == asz
                    assert uo == u_first + i * block + (ao - a_first)
            a_base += block
        assert a_base == one.level_size(L)
        assert uni.level_size(L) == copies * one.level_size(L)
    for kind in KINDS:
        for i in range(copies):
            for p in range(c1[kind]):
                v1, x1, f1 = one.primitive(kind, p)
                vu, xu, fu = uni.primitive(kind, i * c1[kind] + p)
                assert list(vu) == [v + i * nv for v in v1]
                assert f1 == fu
                if kind != hg.VERTEX:
                    continue
                assert np.allclose(np.asarray(xu) - np.asarray(x1), [2.0 * i, 0, 0])

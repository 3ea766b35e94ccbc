"""Macro-mesh construction and the Gmsh wire format, on the host (no GPU).

- meshCubedDomain (MeshGenCubedDomain.cpp:115-383), cube type 0, over a full block of cubes is
  the meshCuboid mesh of that block: same vertices, primitives, order, flags and layouts.
- Cube type 1 has 14 vertices and 24 tetrahedra per cube; every domain of face-connected cubes
  has Euler characteristic V - E + F - C = 1.
- A written Gmsh 2.2 file reads back to the same storage: with flags from the geometry exactly;
  with the file's flags, edges and faces keep theirs and vertices get 0 (points are not read, as
  in the reference's reader). Also with node IDs renumbered and elements shuffled as other
  writers do.
- The reader's failure modes (MeshGenFromGmshFile.cpp:38-160) are errors, not crashes.
- The reference's own 3-D mesh files (when the reference tree is present in this container) all
  parse, with the expected counts for the ones the reference's tests name."""
import os

import numpy as np
import pytest

import hyteg_b200 as hg

REF_MESHES = os.path.join(os.environ.get("HYTEG_REFERENCE", ""), "data", "meshes", "3D") \
    if os.environ.get("HYTEG_REFERENCE") else ""


def describe(m, L):
    """Every primitive's vertex list, coordinates and flag, neighbours, and the level layout."""
    out = []
    counts = m.counts()
    for kind in range(4):
        for p in range(counts[kind]):
            ids, xyz, flag = m.primitive(kind, p)
            nb = [tuple(m.neighbours(kind, p, w)) for w in range(kind + 1, 4)]
            out.append((kind, p, tuple(ids), tuple(np.round(xyz, 12)), flag, tuple(nb), m.layout(L, kind, p)))
    return tuple(counts), out


def test_cubed_domain_type0_is_the_cuboid():
    L = 2
    a = hg.HostMesh.cuboid((0, 0, 0), (2, 2, 2), 2, 2, 2, L)
    cubes = [(x, y, z) for z in range(2) for y in range(2) for x in range(2)]
    b = hg.HostMesh.cubed_domain(cubes[::-1] + cubes[:3], 0, L)  # order and duplicates do not matter
    assert describe(a, L) == describe(b, L)


@pytest.mark.parametrize("cubes", [[(0, 0, 0)], [(0, 0, 0), (1, 0, 0), (0, 1, 0)],
                                   [(x, y, z) for x in range(2) for y in range(2) for z in range(2)]])
def test_cubed_domain_type1_counts(cubes):
    m = hg.HostMesh.cubed_domain(cubes, 1, 1)
    v, e, f, c = m.counts()
    assert c == 24 * len(cubes)
    assert v - e + f - c == 1
    if len(cubes) == 1:
        assert (v, e, f, c) == (14, 49, 60, 24)
    # every cell has positive volume, and the cells fill the cubes
    vol = 0.0
    for k in range(c):
        ids, _, _ = m.primitive(hg.CELL, k)
        p = np.array([m.primitive(hg.VERTEX, i)[1] for i in ids])
        vol += abs(np.linalg.det(p[1:] - p[0])) / 6
    assert abs(vol - len(cubes)) < 1e-12


@pytest.mark.parametrize("which", ["cuboid", "cubed1"])
@pytest.mark.parametrize("file_flags", [True, False])
def test_gmsh_round_trip(tmp_path, which, file_flags):
    L = 2
    if which == "cuboid":
        a = hg.HostMesh.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    else:
        a = hg.HostMesh.cubed_domain([(0, 0, 0), (1, 0, 0), (0, 1, 0)], 1, L)
    path = tmp_path / "m.msh"
    a.write_gmsh(path)
    b = hg.HostMesh.from_gmsh(path, L, flags_from_file=file_flags)
    da, db = describe(a, L), describe(b, L)
    if file_flags:
        # the reader ignores point elements, as the reference's does: vertex flags are 0
        assert all(x[4] == 0 for x in db[1] if x[0] == hg.VERTEX)
        strip = lambda d: [x[:4] + x[5:] if x[0] == hg.VERTEX else x for x in d[1]]  # noqa: E731
        assert da[0] == db[0] and strip(da) == strip(db)
    else:
        assert da == db


def write_shuffled(path, coords, tets, boundary, seed):
    """A Gmsh 2.2 file as other writers produce it: node IDs not contiguous, elements in random
    order, points and lines among them, a duplicate triangle."""
    rng = np.random.default_rng(seed)
    ids = np.sort(rng.choice(np.arange(1, 10 * len(coords)), len(coords), replace=False))
    elems = [("15 2 7 7 %d" % ids[i]) for i in range(len(coords))]
    for t in boundary:
        elems.append("2 2 5 5 %d %d %d" % tuple(ids[list(t)]))
        elems.append("1 2 5 5 %d %d" % (ids[t[0]], ids[t[1]]))
    elems.append("2 2 5 5 %d %d %d" % tuple(ids[list(boundary[0])]))
    for t in tets:
        elems.append("4 2 0 1 %d %d %d %d" % tuple(ids[list(t)]))
    order = rng.permutation(len(elems))
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(coords))
        perm = rng.permutation(len(coords))
        for i in perm:
            f.write("%d %.17g %.17g %.17g\n" % (ids[i], *coords[i]))
        f.write("$EndNodes\n$Elements\n%d\n" % len(elems))
        for n, k in enumerate(order):
            f.write("%d %s\n" % (n + 1, elems[k]))
        f.write("$EndElements\n")


def test_gmsh_foreign_numbering(tmp_path):
    L = 2
    from oracle import oracle
    coords, tets = oracle.cuboid_mesh((0, 0, 0), (1, 1, 1), 2, 2, 2)
    ref = hg.HostMesh.from_tets(coords, tets, L)
    bnd = [tuple(ref.primitive(hg.FACE, f)[0]) for f in range(ref.counts()[2]) if ref.primitive(hg.FACE, f)[2] == 1]
    path = tmp_path / "foreign.msh"
    write_shuffled(path, np.asarray(coords), np.asarray(tets), bnd, 3)
    got = hg.HostMesh.from_gmsh(path, L)
    assert describe(ref, L) == describe(got, L)
    # with the file's flags: boundary triangles and lines carry tag 5, everything else 0
    tagged = hg.HostMesh.from_gmsh(path, L, flags_from_file=True)
    for f in range(tagged.counts()[2]):
        assert tagged.primitive(hg.FACE, f)[2] == (5 if ref.primitive(hg.FACE, f)[2] == 1 else 0)
    for v in range(tagged.counts()[0]):
        assert tagged.primitive(hg.VERTEX, v)[2] == 0


BAD = {
    "version": "$MeshFormat\n4.1 0 8\n$EndMeshFormat\n",
    "binary": "$MeshFormat\n2.2 1 8\n$EndMeshFormat\n",
    "quad": ("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n4\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n$EndNodes\n"
             "$Elements\n2\n1 3 2 0 0 1 2 3 4\n2 4 2 0 0 1 2 3 4\n$EndElements\n"),
    "unknown node": ("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n4\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n"
                     "$EndNodes\n$Elements\n1\n1 4 2 0 0 1 2 3 9\n$EndElements\n"),
    "lonely node": ("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n5\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n"
                    "5 3 3 3\n$EndNodes\n$Elements\n1\n1 4 2 0 0 1 2 3 4\n$EndElements\n"),
    "truncated": "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n4\n1 0 0 0\n2 1 0",
}


@pytest.mark.parametrize("case", sorted(BAD))
def test_gmsh_errors(tmp_path, case):
    path = tmp_path / "bad.msh"
    path.write_text(BAD[case])
    with pytest.raises(hg.HygError) as e:
        hg.HostMesh.from_gmsh(path, 1)
    assert e.value.code == 1
    with pytest.raises(hg.HygError):
        hg.HostMesh.from_gmsh(tmp_path / "missing.msh", 1)


@pytest.mark.skipif(not os.path.isdir(REF_MESHES), reason="reference tree not given (HYTEG_REFERENCE)")
def test_reference_mesh_files_parse():
    expect = {"tet_1el.msh": (4, 6, 4, 1), "cube_6el.msh": (8, 19, 18, 6), "cube_48el.msh": (27, 98, 120, 48)}
    for name in sorted(os.listdir(REF_MESHES)):
        if not name.endswith(".msh"):
            continue
        m = hg.HostMesh.from_gmsh(os.path.join(REF_MESHES, name), 1)
        v, e, f, c = m.counts()
        assert c > 0 and v - e + f - c == 1, name
        if name in expect:
            assert (v, e, f, c) == expect[name], name

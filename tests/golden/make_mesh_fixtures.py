"""Generates tests/golden/meshes.json from the reference's Gmsh fixtures
(data/meshes/3D/*.msh of wagnandr/hyteg): vertex coordinates and tetrahedra (0-based vertex
IDs in the file's vertex order, cells in the file's vertex order, as MeshInfo::fromGmshFile
reads them, src/hyteg/mesh/MeshGenFromGmshFile.cpp:55-199). Run once where the reference
tree is available:  python tests/golden/make_mesh_fixtures.py /path/to/reference
"""
import json
import os
import sys

NAMES = ["tet_1el", "tet_tilted_1el", "pyramid_2el", "pyramid_4el", "pyramid_tilted_4el", "regular_octahedron_8el", "cube_6el",
         "cube_24el"]


def read_msh(path):
    tok = open(path).read().split()
    i = tok.index("$Nodes") + 1
    n = int(tok[i])
    i += 1
    ids, coords = [], []
    for _ in range(n):
        ids.append(int(tok[i]))
        coords.append([float(tok[i + 1]), float(tok[i + 2]), float(tok[i + 3])])
        i += 4
    index = {v: k for k, v in enumerate(sorted(ids))}
    coords = [c for _, c in sorted(zip(ids, coords))]
    i = tok.index("$Elements") + 1
    m = int(tok[i])
    i += 1
    tets = []
    for _ in range(m):
        typ, ntags = int(tok[i + 1]), int(tok[i + 2])
        nodes = {1: 2, 2: 3, 4: 4, 15: 1}[typ]
        vals = [int(t) for t in tok[i + 3 + ntags:i + 3 + ntags + nodes]]
        if typ == 4:
            tets.append([index[v] for v in vals])
        i += 3 + ntags + nodes
    return coords, tets


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HYTEG_REFERENCE")
    if not ref:
        sys.exit("usage: make_mesh_fixtures.py <reference root>  (or set HYTEG_REFERENCE)")
    out = {}
    for name in NAMES:
        p = os.path.join(ref, "data", "meshes", "3D", name + ".msh")
        if os.path.exists(p):
            c, t = read_msh(p)
            out[name] = {"coords": c, "tets": t}
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "meshes.json"), "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", sorted(out))


if __name__ == "__main__":
    main()

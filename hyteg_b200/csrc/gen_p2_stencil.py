"""Writes p2_stencil.h: the offsets of the constant P2 stencil of an interior node, per parity class.

A P2 function of level L lives on the vertex lattice of level L + 1. A node (X, Y, Z) of a
macro-cell has the parity class pc = (X & 1) | (Y & 1) << 1 | (Z & 1) << 2: 0 for the
micro-vertices of level L, 1..7 for the midpoints of the micro-edges of orientation X, Y, XY,
Z, XZ, YZ, XYZ. The level-L micro-cells around an interior node of a class form the same pattern
at every node of that class, so its matrix row couples it to a fixed set of lattice offsets. They
are the union, over the micro-cells (type t, local node j) of the class, of the offsets of the
ten nodes of the micro-cell from node j. The weights depend on the macro-cell and are assembled
on the host in the order written here.

The micro-cell table is the refinement of a macro-cell into six micro-cell types
(`MacroCellIndexing` in the reference); the edge order of the ten local P2 nodes follows the
element matrices (vertices 0-3, then edges 01, 02, 03, 12, 13, 23).

Run: python hyteg_b200/csrc/gen_p2_stencil.py  (rewrites hyteg_b200/csrc/p2_stencil.h)
"""
import os

MICRO_CELLS = [
    [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)],
    [(1, 0, 0), (1, 1, 0), (0, 1, 0), (1, 0, 1)],
    [(1, 0, 0), (0, 1, 0), (1, 0, 1), (0, 0, 1)],
    [(1, 1, 0), (1, 1, 1), (0, 1, 1), (1, 0, 1)],
    [(1, 0, 1), (0, 1, 1), (0, 0, 1), (0, 1, 0)],
    [(0, 1, 0), (1, 1, 0), (1, 0, 1), (0, 1, 1)],
]
EDGES = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]


def node_offsets():
    """Lattice offset (level L + 1 units) of local P2 node j of micro-cell type t from 2 * anchor."""
    off = []
    for cell in MICRO_CELLS:
        o = [tuple(2 * c for c in v) for v in cell]
        o += [tuple(cell[a][d] + cell[b][d] for d in range(3)) for a, b in EDGES]
        off.append(o)
    return off


def stencils():
    off = node_offsets()
    out = []
    for pc in range(8):
        cand = [(t, j) for t in range(6) for j in range(10)
                if (off[t][j][0] & 1) | ((off[t][j][1] & 1) << 1) | ((off[t][j][2] & 1) << 2) == pc]
        s = set()
        for t, j in cand:
            for m in range(10):
                s.add(tuple(off[t][m][d] - off[t][j][d] for d in range(3)))
        out.append(sorted(s, key=lambda o: (o[2], o[1], o[0])))
    return out


WIDTH_REDUCTION = [0, 1, 1, 2, 1, 1]  # micro-cells of type t: a_x + a_y + a_z < N - reduction[t]
FACES = ["Z = 0", "Y = 0", "X = 0", "X + Y + Z = M"]


def face_node(face, pc, M=16):
    """A node of class pc inside face `face` of a macro-cell of lattice M (away from its edges)."""
    X, Y, Z = 4 + (pc & 1), 4 + ((pc >> 1) & 1), 4 + ((pc >> 2) & 1)
    if face == 0:
        Z = 0
    elif face == 1:
        Y = 0
    elif face == 2:
        X = 0
    else:
        Z = M - X - Y
    return X, Y, Z


def face_classes(face):
    return [pc for pc in range(8) if all(c % 2 == b for c, b in zip(face_node(face, pc),
                                                                    (pc & 1, (pc >> 1) & 1, (pc >> 2) & 1)))]


def face_stencils(M=16):
    """Per face and parity class present on it: the micro-cells inside the macro-cell that hold
    a face-interior node (the same at every such node) and the offsets of their nodes."""
    off = node_offsets()
    N = M // 2
    out = []
    for face in range(4):
        for pc in face_classes(face):
            X, Y, Z = face_node(face, pc, M)
            cand = []
            for t in range(6):
                for j in range(10):
                    if (off[t][j][0] & 1) | ((off[t][j][1] & 1) << 1) | ((off[t][j][2] & 1) << 2) != pc:
                        continue
                    a = [(q - o) >> 1 for q, o in zip((X, Y, Z), off[t][j])]
                    if min(a) < 0 or sum(a) >= N - WIDTH_REDUCTION[t]:
                        continue
                    cand.append((t, j))
            s = set()
            for t, j in cand:
                for m in range(10):
                    s.add(tuple(off[t][m][d] - off[t][j][d] for d in range(3)))
            out.append((face, pc, cand, sorted(s, key=lambda o: (o[2], o[1], o[0]))))
    return out


def divt_stencils():
    """Per velocity class: the pressure-lattice offsets (relative to (X >> 1, Y >> 1, Z >> 1)) of
    the vertices of the micro-cells around an interior velocity node, with the (type, local node j,
    vertex i) triples that contribute to each."""
    off = node_offsets()
    out = []
    for pc in range(8):
        par = (pc & 1, (pc >> 1) & 1, (pc >> 2) & 1)
        contrib = {}
        for t in range(6):
            for j in range(10):
                if tuple(c & 1 for c in off[t][j]) != par:
                    continue
                for i in range(4):
                    e = tuple((off[t][i][d] - off[t][j][d] + par[d]) // 2 for d in range(3))
                    contrib.setdefault(e, []).append((t, j, i))
        keys = sorted(contrib, key=lambda o: (o[2], o[1], o[0]))
        out.append(keys)
    return out


def render():
    st = stencils()
    n = max(len(s) for s in st)
    lines = [
        "// Generated by gen_p2_stencil.py (do not edit): the lattice offsets (dx, dy, dz) of the constant",
        "// P2 stencil of an interior node of the level L + 1 vertex lattice, per parity class",
        "// pc = (X & 1) | (Y & 1) << 1 | (Z & 1) << 2, ordered by (dz, dy, dx). The weights of a macro-cell",
        "// are assembled on the host in this order (Storage::createP2Operator).",
        "#pragma once",
        "",
        "namespace hg {",
        "namespace p2s {",
        "",
        "constexpr int kMaxLen = %d;" % n,
        "constexpr int kLen[8] = {%s};" % ", ".join(str(len(s)) for s in st),
        "constexpr int kTotal = %d;" % sum(len(s) for s in st),
        "constexpr int kFirst[8] = {%s};" % ", ".join(str(sum(len(s) for s in st[:k])) for k in range(8)),
        "constexpr int kCentre[8] = {%s};" % ", ".join(str(s.index((0, 0, 0))) for s in st),
        "",
        "// host table, indexed [class][entry][axis]",
        "constexpr signed char kOff[8][kMaxLen][3] = {",
    ]
    for s in st:
        lines.append("    {" + ", ".join("{%d, %d, %d}" % o for o in s) + "},")
    lines += [
        "};",
        "",
        "// device type lists: one O<dx, dy, dz> per entry, in the same order",
        "template <int DX, int DY, int DZ>",
        "struct O {};",
        "template <class... E>",
        "struct List {};",
    ]
    for pc, s in enumerate(st):
        lines.append("using S%d = List<%s>;" % (pc, ", ".join("O<%d, %d, %d>" % o for o in s)))
    fs = face_stencils()
    fmax = max(len(f[3]) for f in fs)
    cmax = max(len(f[2]) for f in fs)
    lines += [
        "",
        "// Face-interior nodes (a node on exactly one face of the macro-cell) couple to the nodes of",
        "// the micro-cells inside the cell that hold them, the same ones at every node of a (face, class):",
        "// faces 0: Z = 0, 1: Y = 0, 2: X = 0, 3: X + Y + Z = M; four classes per face. Entry k of the",
        "// tables below is face k / 4, class kFaceClass[k]; kFaceCand lists its micro-cells (type, local node).",
        "constexpr int kFaceStencils = %d;" % len(fs),
        "constexpr int kFaceMaxLen = %d;" % fmax,
        "constexpr int kFaceClass[%d] = {%s};" % (len(fs), ", ".join(str(f[1]) for f in fs)),
        "constexpr int kFaceLen[%d] = {%s};" % (len(fs), ", ".join(str(len(f[3])) for f in fs)),
        "constexpr int kFaceTotal = %d;" % sum(len(f[3]) for f in fs),
        "constexpr int kFaceFirst[%d] = {%s};" % (len(fs), ", ".join(str(sum(len(g[3]) for g in fs[:k])) for k in range(len(fs)))),
        "constexpr int kFaceNCand[%d] = {%s};" % (len(fs), ", ".join(str(len(f[2])) for f in fs)),
        "constexpr signed char kFaceCand[%d][%d][2] = {" % (len(fs), cmax),
    ]
    for f in fs:
        lines.append("    {" + ", ".join("{%d, %d}" % c for c in f[2]) + "},")
    lines += ["};", "constexpr signed char kFaceOff[%d][kFaceMaxLen][3] = {" % len(fs)]
    for f in fs:
        lines.append("    {" + ", ".join("{%d, %d, %d}" % o for o in f[3]) + "},")
    lines.append("};")
    for k, f in enumerate(fs):
        lines.append("using F%d = List<%s>;  // face %d (%s), class %d" % (k, ", ".join("O<%d, %d, %d>" % o for o in f[3]),
                                                                        f[0], FACES[f[0]], f[1]))
    dt = divt_stencils()
    lines += [
        "",
        "// Taylor-Hood coupling at interior velocity nodes (divT): per velocity class, the offsets",
        "// (ex, ey, ez) of the pressure nodes on the pressure lattice, relative to (X >> 1, Y >> 1, Z >> 1).",
        "// The divergence at an interior pressure node (x, y, z) reads the velocity nodes (2x, 2y, 2z) + S0.",
        "constexpr int kDivTMaxLen = %d;" % max(len(d) for d in dt),
        "constexpr int kDivTLen[8] = {%s};" % ", ".join(str(len(d)) for d in dt),
        "constexpr int kDivTTotal = %d;" % sum(len(d) for d in dt),
        "constexpr int kDivTFirst[8] = {%s};" % ", ".join(str(sum(len(x) for x in dt[:k])) for k in range(8)),
        "constexpr signed char kDivTOff[8][kDivTMaxLen][3] = {",
    ]
    for d in dt:
        lines.append("    {" + ", ".join("{%d, %d, %d}" % o for o in d) + "},")
    lines.append("};")
    for pc, d in enumerate(dt):
        lines.append("using T%d = List<%s>;" % (pc, ", ".join("O<%d, %d, %d>" % o for o in d)))
    lines += ["", "template <int PC>", "struct DivTList;"]
    for pc in range(8):
        lines += ["template <>", "struct DivTList<%d> {" % pc, "  using type = T%d;" % pc, "};"]
    lines += ["", "template <int PC>", "struct Class;"]
    for pc in range(8):
        lines.append("template <>")
        lines.append("struct Class<%d> {" % pc)
        lines.append("  using type = S%d;" % pc)
        lines.append("};")
    lines += ["", "template <int K>", "struct FaceList;"]
    for k in range(len(fs)):
        lines += ["template <>", "struct FaceList<%d> {" % k, "  using type = F%d;" % k, "};"]
    lines += ["", "}  // namespace p2s", "}  // namespace hg", ""]
    return "\n".join(lines)


def main():
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "p2_stencil.h")
    with open(path, "w") as f:
        f.write(render())


if __name__ == "__main__":
    main()

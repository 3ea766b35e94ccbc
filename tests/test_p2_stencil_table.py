"""The committed P2 stencil offset header equals its generator's output, and the offsets have the
properties the in-place multicolour SOR relies on: an edge class couples to no node of its own
class, and the vertex class only to its P1 neighbours (which the four vertex colours separate)."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "hyteg_b200", "csrc")


def load_generator():
    spec = importlib.util.spec_from_file_location("gen_p2_stencil", os.path.join(CSRC, "gen_p2_stencil.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_header_is_generated():
    gen = load_generator()
    with open(os.path.join(CSRC, "p2_stencil.h")) as f:
        assert f.read() == gen.render()


def test_offsets_and_colour_independence():
    gen = load_generator()
    st = gen.stencils()
    p1 = {(1, 0, 0), (0, 1, 0), (0, 0, 1), (-1, 0, 1), (-1, 1, 0), (0, -1, 1), (-1, 1, -1)}
    p1 |= {tuple(-c for c in o) for o in p1}
    for pc, offs in enumerate(st):
        assert (0, 0, 0) in offs
        assert all(max(abs(c) for c in o) <= 2 for o in offs)
        same = [o for o in offs if o != (0, 0, 0) and all(c % 2 == 0 for c in o)]
        if pc == 0:
            assert {tuple(c // 2 for c in o) for o in same} == p1
            # colour (x + 2y + 3z) mod 4 of the coarse lattice differs across every P1 offset
            assert all((a + 2 * b + 3 * c) % 4 != 0 for a, b, c in p1)
        else:
            assert same == []
    assert [len(s) for s in st] == [65, 27, 19, 27, 27, 19, 27, 19]


def test_face_stencils_are_constant_per_face_and_class():
    # at every node inside one face of a macro-cell (lattices 4..16), the micro-cells inside the
    # cell that hold the node are the generated candidates, and the stencil reads stay in the cell
    gen = load_generator()
    off = gen.node_offsets()
    fs = gen.face_stencils()
    assert [f[1] for f in fs] == [0, 1, 2, 3, 0, 1, 4, 5, 0, 2, 4, 6, 0, 3, 5, 6]  # the kernels' entry map
    for M in (4, 8, 16):
        N = M // 2
        on = [lambda X, Y, Z: Z == 0, lambda X, Y, Z: Y == 0, lambda X, Y, Z: X == 0,
              lambda X, Y, Z: X + Y + Z == M]
        for f, pc, cand, offs in fs:
            for Z in range(M + 1):
                for Y in range(M + 1 - Z):
                    for X in range(M + 1 - Z - Y):
                        if not on[f](X, Y, Z) or sum(o(X, Y, Z) for o in on) != 1:
                            continue
                        if (X & 1) | ((Y & 1) << 1) | ((Z & 1) << 2) != pc:
                            continue
                        valid = []
                        for t in range(6):
                            for j in range(10):
                                if tuple(c & 1 for c in off[t][j]) != (pc & 1, (pc >> 1) & 1, (pc >> 2) & 1):
                                    continue
                                a = [(q - o) >> 1 for q, o in zip((X, Y, Z), off[t][j])]
                                if min(a) >= 0 and sum(a) < N - gen.WIDTH_REDUCTION[t]:
                                    valid.append((t, j))
                        assert valid == cand
                        assert all(X + dx >= 0 and Y + dy >= 0 and Z + dz >= 0 and X + Y + Z + dx + dy + dz <= M
                                   for dx, dy, dz in offs)

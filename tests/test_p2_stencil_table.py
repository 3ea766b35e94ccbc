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

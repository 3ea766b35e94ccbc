"""The term lists behind the device re-assembly of stencils (hg_operator_reassemble) on the host:
every stencil entry summed from its terms in order equals the assembled table bit for bit, for
the diffusion and mass forms, on the 48-tet cube and an L-shaped 24-tet-per-cube domain, levels
0-4, with non-uniform macro-cell coefficients."""
import numpy as np
import pytest

import hyteg_b200 as hg


@pytest.mark.parametrize("mesh", ["cube", "cubed1"])
@pytest.mark.parametrize("form", [0, 1])
def test_terms_reproduce_the_tables(mesh, form):
    L = 4
    if mesh == "cube":
        m = hg.HostMesh.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    else:
        m = hg.HostMesh.cubed_domain([(0, 0, 0), (1, 0, 0), (0, 1, 0)], 1, L)
    nc = m.counts()[3]
    m.set_cell_coefficients(np.exp(np.random.default_rng(5).uniform(-2, 2, nc)))
    for lev in range(L + 1):
        targets, terms, bad = m.assembly_plan_check(lev, form)
        assert bad == 0
        assert targets >= 16 * nc
        if lev >= 2:
            assert terms > targets // 2


def test_colour_split_tables():
    """The per-colour point and row tables of the colour-split SOR (schedule 3): every interior
    point once, in order, with its 15 slots equal to the split positions of its neighbours
    recomputed from their coordinates (levels 2-6)."""
    for level in range(2, 7):
        n = 2 ** level
        points, bad = hg.split_tables_check(level)
        assert bad == 0, level
        assert points == (n - 3) * (n - 2) * (n - 1) // 6  # interior points of a macro-cell

"""The packed owned-DoF order of hg_function_*_owned_async, on the CPU: hg_mesh_owned_slots lists
exactly the slots that slot_info marks as owned (every DoF of the level once), in level-buffer
order, on cube, cubed-domain and Gmsh meshes of several levels."""
import json
import os

import numpy as np
import pytest

import hyteg_b200 as hg

HERE = os.path.dirname(os.path.abspath(__file__))


def meshes():
    yield "cube 2x2x2", hg.HostMesh.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, 4)
    yield "cube 3x1x2", hg.HostMesh.cuboid((0, 0, 0), (3, 1, 2), 3, 1, 2, 3)
    with open(os.path.join(HERE, "golden", "meshes.json")) as f:
        m = json.load(f)["regular_octahedron_8el"]
    yield "octahedron", hg.HostMesh.from_tets(np.array(m["coords"], dtype=np.float64),
                                              np.array(m["tets"], dtype=np.int32), 4)


@pytest.mark.parametrize("name,mesh", list(meshes()))
def test_owned_slots_are_the_owned_dofs_in_buffer_order(name, mesh):
    for L in range(mesh.max_level + 1):
        _, owned = mesh.slot_info(L)
        slots = mesh.owned_slots(L)
        assert np.array_equal(slots, np.flatnonzero(owned == 1)), (name, L)

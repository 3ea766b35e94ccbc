"""Device re-assembly of the stencils for new macro-cell coefficients (hg_operator_reassemble):
an operator re-assembled on the device applies bit for bit like an operator assembled on the host
from the same coefficients, in FP64 and FP32, on every level; so does the host re-assembly; and the
operator's diagonal (read from the host copy) follows the new coefficients."""
import numpy as np
import pytest

import hyteg_b200 as hg

pytestmark = pytest.mark.gpu
L = 4


@pytest.fixture(scope="module")
def gpu():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("mesh", ["cube", "cubed1"])
def test_device_reassembly_equals_host_assembly(gpu, dtype, mesh):
    if mesh == "cube":
        st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    else:
        st = hg.PrimitiveStorage.cubed_domain([(0, 0, 0), (1, 0, 0), (0, 1, 0)], 1, L)
    nc = st.counts()[3]
    rng = np.random.default_rng(2)
    st.set_cell_coefficients(np.exp(rng.uniform(-1, 1, nc)))
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    k2 = np.exp(rng.uniform(-2, 2, nc))
    st.set_cell_coefficients(k2)
    A.reassemble(on_device=True)
    B = hg.P1ConstantLaplaceOperator(st, 0, L)  # assembled on the host from k2
    x = hg.P1Function("x", st, 0, L, dtype=dtype)
    ya = hg.P1Function("ya", st, 0, L, dtype=dtype)
    yb = hg.P1Function("yb", st, 0, L, dtype=dtype)
    for lev in range(L + 1):
        x.fill_random(10 + lev, lev, hg.All)
        A.apply(x, ya, lev, hg.All)
        B.apply(x, yb, lev, hg.All)
        assert np.array_equal(ya.to_numpy(lev), yb.to_numpy(lev)), lev
    # a second device re-assembly (term lists reused) and a host re-assembly agree as well
    k3 = np.exp(rng.uniform(-2, 2, nc))
    st.set_cell_coefficients(k3)
    A.reassemble(on_device=True)
    B.reassemble(on_device=False)
    for lev in range(L + 1):
        x.fill_random(20 + lev, lev, hg.All)
        A.apply(x, ya, lev, hg.All)
        B.apply(x, yb, lev, hg.All)
        assert np.array_equal(ya.to_numpy(lev), yb.to_numpy(lev)), lev


def test_mass_form_is_left_alone(gpu):
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, 3)
    M = hg.P1ConstantMassOperator(st, 0, 3)
    x, y0, y1 = (hg.P1Function(n, st, 0, 3) for n in ("x", "y0", "y1"))
    x.fill_random(1, 3, hg.All)
    M.apply(x, y0, 3, hg.All)
    st.set_cell_coefficients(np.full(48, 7.0))
    M.reassemble(on_device=True)
    M.apply(x, y1, 3, hg.All)
    assert np.array_equal(y0.to_numpy(3), y1.to_numpy(3))


def test_sor_and_cycles_after_device_reassembly(gpu):
    # the smoother and the multigrid read the re-assembled stencils: a V-cycle from a device
    # re-assembled operator equals one from a host-assembled operator bit for bit
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    st.set_cell_coefficients(np.exp(np.random.default_rng(9).uniform(-1, 1, 48)))
    A.reassemble(on_device=True)
    B = hg.P1ConstantLaplaceOperator(st, 0, L)
    out = []
    for op in (A, B):
        x, b = hg.P1Function("x", st, 0, L), hg.P1Function("b", st, 0, L)
        b.fill_random(4, L, hg.Inner)
        gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 100, 1e-16),
                                          hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3)
        gmg.set_graphs(op, False)
        for _ in range(2):
            gmg.solve(op, x, b, L)
        out.append(x.to_numpy(L))
    assert np.array_equal(out[0], out[1])

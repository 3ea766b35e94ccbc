"""Size-independent properties at the benchmark's full size: the 48-tet cube at level 8
(133,432,831 inner DoFs, 1.18 GB per FP64 vector), where the oracle cannot follow.

- The constant stencils annihilate constants and linear functions at inner DoFs (the property
  the reference's P1LaplaceOperator3DTest checks).
- An exact solution is a fixed point of the SOR sweep: with b = A x, one sweep (single-pass
  wavefront, four colour passes, and colour passes on colour-split copies; FP64 and FP32) leaves
  x unchanged to rounding.
- On random data, two SOR sweeps (forward and backward, omega = 1.3) of every schedule equal those
  of the four in-place colour passes within 1e-13 at levels 7 and 8: every tile of the wavefront
  pass, including the tiles clipped by the sloped face, and every colour-split row is checked.
- Restriction is the transpose of prolongation on inner DoFs: <R r, c> = <r, P c>.
- apply is linear: A (2 x + 3 y) = 2 A x + 3 A y.

Tolerances are relative to the size of the same operation on random data: 1e-12 in FP64,
1e-5 in FP32."""
import numpy as np
import pytest

import hyteg_b200 as hg

pytestmark = pytest.mark.gpu
L = 8


@pytest.fixture(scope="module")
def l8():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    A = hg.P1ConstantLaplaceOperator(st, L - 1, L)
    return st, A


def inner_max(f, level):
    return float(np.abs(f.to_numpy(level)).max())


def test_stencils_annihilate_constants_and_linears(l8):
    st, A = l8
    x = hg.P1Function("x", st, L, L)
    y = hg.P1Function("y", st, L, L)
    x.fill_random(1, L, hg.All)
    A.apply(x, y, L, hg.Inner)
    scale = inner_max(y, L)
    for setter in (lambda: x.interpolate(2.5, L, hg.All), lambda: x.interpolate_linear(0.3, 1.0, -2.0, 0.5, L, hg.All)):
        setter()
        y.interpolate(0.0, L, hg.All)
        A.apply(x, y, L, hg.Inner)
        assert inner_max(y, L) < 1e-12 * scale


@pytest.mark.parametrize("schedule", [0, 1, 3])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_exact_solution_is_a_fixed_point_of_sor(l8, schedule, dtype, tol):
    st, A = l8
    st.set_sor_schedule(schedule)
    try:
        x = hg.P1Function("x", st, L, L, dtype=dtype)
        x0 = hg.P1Function("x0", st, L, L, dtype=dtype)
        b = hg.P1Function("b", st, L, L, dtype=dtype)
        x.fill_random(7, L, hg.All)
        x0.copy_from(x, L)
        A.apply(x, b, L, hg.Inner | hg.NeumannBoundary)
        A.smooth_sor(x, b, 1.0, L, hg.Inner | hg.NeumannBoundary)
        d = hg.P1Function("d", st, L, L, dtype=dtype)
        d.assign([1.0, -1.0], [x, x0], L, hg.All)
        assert inner_max(d, L) < tol * inner_max(x0, L)
    finally:
        st.set_sor_schedule(0)


@pytest.mark.parametrize("level", [7, 8])
@pytest.mark.parametrize("schedule", [0, 2, 3])
@pytest.mark.parametrize("backwards", [False, True])
def test_sor_schedules_agree_on_random_data(l8, level, schedule, backwards):
    st, A = l8
    x = hg.P1Function("x", st, level, level)
    x1 = hg.P1Function("x1", st, level, level)
    b = hg.P1Function("b", st, level, level)
    x.fill_random(21 + level, level, hg.All)
    b.fill_random(31 + level, level, hg.All)
    x1.copy_from(x, level)
    flag = hg.Inner | hg.NeumannBoundary
    smooth = A.smooth_sor_backwards if backwards else A.smooth_sor
    try:
        for sched, f in ((schedule, x), (1, x1)):
            st.set_sor_schedule(sched)
            for _ in range(2):
                smooth(f, b, 1.3, level, flag)
    finally:
        st.set_sor_schedule(0)
    for f in (x, x1):
        f.communicate(level)
    d = hg.P1Function("d", st, level, level)
    d.assign([1.0, -1.0], [x, x1], level, hg.All)
    assert inner_max(d, level) < 1e-13 * inner_max(x1, level)


def test_restriction_is_the_transpose_of_prolongation(l8):
    st, _ = l8
    r = hg.P1Function("r", st, L - 1, L)
    c = hg.P1Function("c", st, L - 1, L)
    r.fill_random(3, L, hg.Inner)
    c.fill_random(4, L - 1, hg.Inner)
    r.interpolate(0.0, L - 1, hg.All)
    c.interpolate(0.0, L, hg.All)
    hg.P1toP1LinearRestriction().restrict(r, L, hg.Inner)
    hg.P1toP1LinearProlongation().prolongate(c, L - 1, hg.Inner)
    lhs = r.dotGlobal(c, L - 1, hg.Inner)  # <R r, c>
    r2 = hg.P1Function("r2", st, L, L)
    r2.fill_random(3, L, hg.Inner)
    rhs = r2.dotGlobal(c, L, hg.Inner)  # <r, P c>
    assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + abs(rhs))


def test_apply_is_linear(l8):
    st, A = l8
    x, y, z = (hg.P1Function(n, st, L, L) for n in ("x", "y", "z"))
    ax, ay, az = (hg.P1Function(n, st, L, L) for n in ("ax", "ay", "az"))
    x.fill_random(11, L, hg.All)
    y.fill_random(12, L, hg.All)
    z.assign([2.0, 3.0], [x, y], L, hg.All)
    for src, dst in ((x, ax), (y, ay), (z, az)):
        A.apply(src, dst, L, hg.Inner)
    ax.assign([2.0, 3.0, -1.0], [ax, ay, az], L, hg.Inner)
    assert inner_max(ax, L) < 1e-12 * inner_max(az, L)

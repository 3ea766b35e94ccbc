"""The C++ drop-in classes (include/hyteg_b200.hpp) through a compiled C++ caller,
tests/cpp/dropin_check (built by __graft_entry__.build()): storage, P1 functions, the constant
Laplace operator's apply and smooth_sor, a GeometricMultigridSolver V(3,3) cycle, and the
reference's error behaviour (a bad level throws std::runtime_error).

CPU: the header and program compile and link against the library, and without a GPU the program
fails cleanly (status 1, the library's "no CUDA device" message), never by a crash.
GPU: the program's results equal, bit for bit, the same sequence run through the Python mirror
of the same C-ABI."""
import os
import subprocess
import sys

import numpy as np
import pytest

import hyteg_b200 as hg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cpp", "dropin_check")


@pytest.fixture(scope="module")
def binary():
    sys.path.insert(0, ROOT)
    import __graft_entry__

    return __graft_entry__.build_dropin_check()


def test_program_builds_and_fails_cleanly_without_a_gpu(binary, tmp_path):
    if hg.device_count() > 0:
        pytest.skip("a GPU is visible: the GPU test covers the program")
    r = subprocess.run([binary, "3", str(tmp_path / "out.bin")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1, (r.returncode, r.stdout, r.stderr)
    assert "no CUDA device" in r.stderr


def test_program_rejects_bad_arguments(binary):
    r = subprocess.run([binary], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("L", [3, 5])
def test_cpp_caller_equals_python_path_bit_for_bit(binary, tmp_path, L):
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")
    out = tmp_path / "out.bin"
    r = subprocess.run([binary, str(L), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout, r.stderr)
    got = np.fromfile(out, dtype=np.float64)

    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, L)
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    x, b, y = (hg.P1Function(n, st, 0, L) for n in ("x", "b", "y"))
    x.fill_random(1, L, hg.All)
    b.fill_random(2, L, hg.All)
    A.apply(x, y, L, hg.Inner)
    ay = y.to_numpy(L)
    A.smooth_sor(x, b, 1.0, L, hg.Inner | hg.NeumannBoundary)
    sx = x.to_numpy(L)
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 50, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3)
    gmg.solve(A, x, b, L)
    gx = x.to_numpy(L)
    n = st.level_size(L)
    assert got.size == 3 * n
    for k, ref in enumerate((ay, sx, gx)):
        assert np.array_equal(got[k * n:(k + 1) * n], ref), k

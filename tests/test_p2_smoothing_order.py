"""Why the reference's P23DSmoothConvergenceTest (tests/hyteg/convergence/P23DSmoothConvergenceTest.cpp)
is not reproduced by the GPU's P2 smoother, shown on the CPU with the oracle (test
infrastructure): 50 Gauss-Seidel sweeps (omega 1, zero right-hand side, zero Dirichlet data,
random inner start in [0, 1)) on P2 level 2 of pyramid_4el and of the octahedron. A sequential
sweep in node order stays below the test's thresholds (1.6e-3 and 7.7e-2 for the discrete L2
norm over all DoFs). The multicolour order that the GPU runs (11 colours, the oracle's
restatement of it, which the GPU matches to 1e-13) stays above them: the thresholds hold for a
sequential order, not for the multicolour one."""
import json
import os

import numpy as np
import pytest

from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name,bound", [("pyramid_4el", 1.6e-3), ("regular_octahedron_8el", 7.7e-2)])
def test_sequential_order_meets_the_threshold_and_multicolour_does_not(name, bound):
    with open(os.path.join(HERE, "golden", "meshes.json")) as f:
        m = json.load(f)[name]
    L = 2
    orc = oracle.Oracle(np.array(m["coords"], dtype=np.float64), np.array(m["tets"], dtype=np.int32), L + 1)
    n = orc.n(L + 1)
    inner = np.flatnonzero(~orc.dirichlet(L + 1))
    A = np.zeros((n, n))
    for j in range(n):  # the assembled P2 operator, column by column
        e = np.zeros(n)
        e[j] = 1.0
        A[:, j] = orc.p2_apply(L, e)
    A = A[np.ix_(inner, inner)]
    u0 = np.zeros(n)
    u0[inner] = np.random.default_rng(0).uniform(0.0, 1.0, len(inner))
    multicolour = np.linalg.norm(orc.p2_sor(L, u0, np.zeros(n), 1.0, sweeps=50))
    v = u0[inner].copy()
    for _ in range(50):
        for i in range(len(inner)):
            v[i] -= (A[i] @ v) / A[i, i]
    sequential = np.linalg.norm(v)
    assert sequential < bound < multicolour, (sequential, bound, multicolour)

"""Generates tests/golden/convergence_cube.json: the oracle's V(3,3) multigrid on the 48-tet cube
(meshCuboid((0,0,0),(1,1,1),2,2,2), levels 3..6, CG on level 0) for the manufactured problem
-Lap u = 3 pi^2 u, u = sin(pi x) sin(pi y) sin(pi z), b = M I(3 pi^2 u), x0 = 0
(MultigridStudies.cpp:488-495 of the reference), 20 cycles each with

  lexicographic SOR in the reference's order (P1Operator.hpp:350-420, the reference's own
                generated kernels' sweep order; omega = 1), and
  multicolour SOR (the GPU's colouring, restated in the oracle).

Stored per level and ordering: the residual 2-norm over the inner DoFs before and after each
cycle, and the discrete L2 error sqrt(e.e / #inner) against u after 10 cycles
(MultigridStudies.cpp:229-256). The GPU tests compare their cycle factors and errors with these.

  python tests/golden/make_convergence_factors.py       (about four minutes on one core)
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle  # noqa: E402

LEVELS = (3, 4, 5, 6)
CYCLES = 20


def main():
    coords, tets = oracle.cuboid_mesh((0, 0, 0), (1, 1, 1), 2, 2, 2)
    orc = oracle.Oracle(coords, tets, max(LEVELS))
    out = {"mesh": "meshCuboid((0,0,0),(1,1,1),2,2,2), 48 macro-tets", "cycle": "V(3,3), CG on level 0, omega = 1",
           "problem": "b = M I(3 pi^2 u), u = sin(pi x) sin(pi y) sin(pi z), x0 = 0", "levels": {}}
    for L in LEVELS:
        nodes = orc.nodes(L)[0]
        inner = ~orc.dirichlet(L)
        exact = np.sin(np.pi * nodes[:, 0]) * np.sin(np.pi * nodes[:, 1]) * np.sin(np.pi * nodes[:, 2])
        b = orc.apply(L, 3 * np.pi ** 2 * exact, form=1)
        rec = {"inner_dofs": int(inner.sum())}
        for name, mc in (("lexicographic", False), ("multicolour", True)):
            u = np.zeros(len(nodes))
            res = [float(np.sqrt(((b - orc.apply(L, u))[inner] ** 2).sum()))]
            err10 = None
            for c in range(CYCLES):
                u, _ = orc.gmg(L, 0, u, b, 1, 3, 3, 1.0, multicolour=mc, cg_iter=1000, cg_tol=1e-16)
                res.append(float(np.sqrt(((b - orc.apply(L, u))[inner] ** 2).sum())))
                if c == 9:
                    err10 = float(np.sqrt(((u - exact)[inner] ** 2).mean()))
            rec[name] = {"residuals": res, "l2_error_after_10": err10}
            print(L, name, " ".join("%.3f" % (res[i + 1] / res[i]) for i in range(CYCLES)), flush=True)
        out["levels"][str(L)] = rec
    with open(os.path.join(ROOT, "tests", "golden", "convergence_cube.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()

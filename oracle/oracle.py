"""ctypes loader of the CPU oracle (oracle/liboracle.so) and of the reference's own kernels
(oracle/_ref/libhyteg_ref.so). TEST INFRASTRUCTURE ONLY: imported by tests/, by
__graft_entry__.smoke() as the checker and by bench.py's CPU-baseline leg; never by the product.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libhyteg_ref.so")

P = ctypes.POINTER
c_double, c_int, c_int64, c_void_p = ctypes.c_double, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p


def build():
    """make -C oracle (builds _ref only where the reference tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load_oracle():
    if not os.path.exists(ORACLE_LIB):
        build()
    lib = ctypes.CDLL(ORACLE_LIB)
    sig = {
        "orc_create": (c_void_p, [c_int, P(c_double), c_int, P(c_int), P(c_double), c_int]),
        "orc_destroy": (None, [c_void_p]),
        "orc_num_nodes": (c_int64, [c_void_p, c_int]),
        "orc_nodes": (None, [c_void_p, c_int, P(c_double), P(c_int)]),
        "orc_apply": (None, [c_void_p, c_int, c_int, P(c_double), P(c_double)]),
        "orc_sor": (None, [c_void_p, c_int, P(c_double), P(c_double), c_double, c_int, c_int, c_int]),
        "orc_sor_phases": (None, [c_void_p, c_int, P(c_double), P(c_double), c_double, c_int, c_int, c_int]),
        "orc_restrict": (None, [c_void_p, c_int, P(c_double), P(c_double)]),
        "orc_prolongate": (None, [c_void_p, c_int, P(c_double), P(c_double), c_int]),
        "orc_dot": (c_double, [c_void_p, c_int, P(c_double), P(c_double)]),
        "orc_cg": (c_int, [c_void_p, c_int, P(c_double), P(c_double), c_int, c_double, P(c_double)]),
        "orc_gmg": (None, [c_void_p, c_int, c_int, P(c_double), P(c_double), c_int, c_int, c_int, c_double, c_int,
                           c_int, c_double, P(c_double)]),
        "orc_element_laplace": (None, [P(c_double), P(c_double)]),
        "orc_element_mass": (None, [P(c_double), P(c_double)]),
        "orc_p2_apply": (None, [c_void_p, c_int, P(c_double), P(c_double)]),
        "orc_p2_element_laplace": (None, [P(c_double), P(c_double)]),
        "orc_p2_sor": (None, [c_void_p, c_int, P(c_double), P(c_double), c_double, c_int, c_int]),
        "orc_p2_prolongate": (None, [c_void_p, c_int, P(c_double), P(c_double), c_int]),
        "orc_p2_restrict": (None, [c_void_p, c_int, P(c_double), P(c_double)]),
        "orc_p2_cg": (c_int, [c_void_p, c_int, P(c_double), P(c_double), c_int, c_double]),
        "orc_stokes_apply": (None, [c_void_p, c_int] + [P(c_double)] * 8),
        "orc_p2p1_div_element": (None, [P(c_double), P(c_double)]),
        "orc_element_pspg": (None, [P(c_double), P(c_double)]),
        "orc_pspg_diag": (None, [c_void_p, c_int, P(c_double)]),
        "orc_lumped_mass": (None, [c_void_p, c_int, P(c_double)]),
        "orc_restrict_all": (None, [c_void_p, c_int, P(c_double), P(c_double)]),
        "orc_prolongate_all": (None, [c_void_p, c_int, P(c_double), P(c_double), c_int]),
        "orc_cell_local_stencil": (None, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_int, P(c_double)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load_oracle()
    return _lib


def ref_lib():
    """The reference's own kernels, or None when oracle/_ref was not built."""
    if not os.path.exists(REF_LIB):
        return None
    r = ctypes.CDLL(REF_LIB)
    d = P(c_double)
    r.ref_apply_cell.argtypes = [d, d, c_int, d, c_int]
    r.ref_sor_cell.argtypes = [d, d, c_int, d, c_double]
    r.ref_apply_face.argtypes = [d, d, d, c_int, c_int64, c_int64, c_int64, d, P(c_int), c_int]
    r.ref_restrict_cell.argtypes = [d, d, c_int, d, d, d]
    r.ref_prolongate_cell.argtypes = [d, d, c_int, d, d, d]
    r.ref_p1_tet_diffusion.argtypes = [d, d]
    r.ref_p1_tet_mass.argtypes = [d, d]
    r.ref_p2_tet_diffusion.argtypes = [d, d]
    r.ref_p1_tet_pspg.argtypes = [d, d]
    r.ref_p2_to_p1_div.argtypes = [d, c_int, d]
    r.ref_p1_to_p2_divt.argtypes = [d, c_int, d]
    for f in (r.ref_apply_cell, r.ref_sor_cell, r.ref_apply_face, r.ref_restrict_cell, r.ref_prolongate_cell,
              r.ref_p1_tet_diffusion, r.ref_p1_tet_mass, r.ref_p2_tet_diffusion, r.ref_p2_to_p1_div,
              r.ref_p1_to_p2_divt, r.ref_p1_tet_pspg):
        f.restype = None
    return r


def dp(a):
    return a.ctypes.data_as(P(c_double))


class Oracle:
    """Global-vector CPU restatement on one tetrahedral macro-mesh, levels 0..max_level."""

    def __init__(self, coords, tets, max_level, k=None):
        self.coords = np.ascontiguousarray(coords, dtype=np.float64)
        self.tets = np.ascontiguousarray(tets, dtype=np.int32)
        kk = None if k is None else np.ascontiguousarray(k, dtype=np.float64)
        self._k = kk
        self.max_level = max_level
        self.h = lib().orc_create(len(self.coords), dp(self.coords), len(self.tets),
                                  self.tets.ctypes.data_as(P(c_int)), None if kk is None else dp(kk), max_level)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def n(self, L):
        return int(lib().orc_num_nodes(self.h, L))

    def nodes(self, L):
        n = self.n(L)
        xyz = np.zeros((n, 3))
        info = np.zeros((n, 4), dtype=np.int32)
        lib().orc_nodes(self.h, L, dp(xyz), info.ctypes.data_as(P(c_int)))
        return xyz, info

    def dirichlet(self, L):
        return self.nodes(L)[1][:, 2].astype(bool)

    def apply(self, L, u, y=None, form=0):
        u = np.ascontiguousarray(u, dtype=np.float64)
        y = np.zeros_like(u) if y is None else np.ascontiguousarray(y, dtype=np.float64).copy()
        lib().orc_apply(self.h, L, form, dp(u), dp(y))
        return y

    def sor(self, L, u, f, omega, sweeps=1, multicolour=False, backwards=False):
        u = np.ascontiguousarray(u, dtype=np.float64).copy()
        f = np.ascontiguousarray(f, dtype=np.float64)
        lib().orc_sor(self.h, L, dp(u), dp(f), omega, sweeps, 1 if multicolour else 0, 1 if backwards else 0)
        return u

    def sor_phases(self, L, u, f, omega, kind_mask, multicolour=False, backwards=False):
        u = np.ascontiguousarray(u, dtype=np.float64).copy()
        f = np.ascontiguousarray(f, dtype=np.float64)
        lib().orc_sor_phases(self.h, L, dp(u), dp(f), omega, 1 if multicolour else 0, 1 if backwards else 0, kind_mask)
        return u

    def restrict(self, Lf, fine, coarse=None):
        fine = np.ascontiguousarray(fine, dtype=np.float64)
        coarse = np.zeros(self.n(Lf - 1)) if coarse is None else np.ascontiguousarray(coarse, dtype=np.float64).copy()
        lib().orc_restrict(self.h, Lf, dp(fine), dp(coarse))
        return coarse

    def prolongate(self, Lc, coarse, fine=None, add=False):
        coarse = np.ascontiguousarray(coarse, dtype=np.float64)
        fine = np.zeros(self.n(Lc + 1)) if fine is None else np.ascontiguousarray(fine, dtype=np.float64).copy()
        lib().orc_prolongate(self.h, Lc, dp(coarse), dp(fine), 1 if add else 0)
        return fine

    def dot(self, L, a, b):
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        return lib().orc_dot(self.h, L, dp(a), dp(b))

    def cg(self, L, x, b, max_iter, tol):
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        b = np.ascontiguousarray(b, dtype=np.float64)
        res = c_double()
        it = lib().orc_cg(self.h, L, dp(x), dp(b), max_iter, tol, ctypes.byref(res))
        return x, it, res.value

    def gmg(self, L, minL, x, b, cycles, pre=3, post=3, omega=1.0, multicolour=False, cg_iter=10000, cg_tol=1e-16):
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        b = np.ascontiguousarray(b, dtype=np.float64)
        res = np.zeros(cycles)
        lib().orc_gmg(self.h, L, minL, dp(x), dp(b), cycles, pre, post, omega, 1 if multicolour else 0, cg_iter, cg_tol,
                      dp(res))
        return x, res

    def p2_apply(self, L, u):
        """P2 Laplace of level L applied to u; u and the result are indexed by the nodes of level
        L + 1 (the oracle must hold level L + 1)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        y = np.zeros(self.n(L + 1))
        lib().orc_p2_apply(self.h, L, dp(u), dp(y))
        return y

    def p2_sor(self, L, u, f, omega, sweeps=1, backwards=False):
        """Multicolour SOR on P2 level L (nodes of level L + 1), the GPU's colour order."""
        u = np.ascontiguousarray(u, dtype=np.float64).copy()
        f = np.ascontiguousarray(f, dtype=np.float64)
        lib().orc_p2_sor(self.h, L, dp(u), dp(f), omega, sweeps, 1 if backwards else 0)
        return u

    def p2_prolongate(self, Lc, coarse, fine=None, add=False):
        """P2 quadratic prolongation from P2 level Lc (nodes of level Lc + 1) to Lc + 1."""
        coarse = np.ascontiguousarray(coarse, dtype=np.float64)
        fine = np.zeros(self.n(Lc + 2)) if fine is None else np.ascontiguousarray(fine, dtype=np.float64).copy()
        lib().orc_p2_prolongate(self.h, Lc, dp(coarse), dp(fine), 1 if add else 0)
        return fine

    def p2_restrict(self, Lf, fine):
        """Transpose of the P2 prolongation: P2 level Lf (nodes of Lf + 1) to Lf - 1 (nodes of Lf)."""
        fine = np.ascontiguousarray(fine, dtype=np.float64)
        coarse = np.zeros(self.n(Lf))
        lib().orc_p2_restrict(self.h, Lf, dp(fine), dp(coarse))
        return coarse

    def p2_cg(self, L, x, b, max_iter=10000, tol=1e-13):
        """CG solution of the P2 Laplace system of level L (Dirichlet values of x kept)."""
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        b = np.ascontiguousarray(b, dtype=np.float64)
        lib().orc_p2_cg(self.h, L, dp(x), dp(b), max_iter, tol)
        return x

    def stokes_apply(self, L, u, p):
        """Taylor-Hood Stokes of P2 level L: u = three velocity vectors (nodes of level L + 1), p the
        pressure (nodes of level L); returns (v, q) with v_k = A u_k + D_k^T p, q = sum_k D_k u_k."""
        u = [np.ascontiguousarray(x, dtype=np.float64) for x in u]
        p = np.ascontiguousarray(p, dtype=np.float64)
        v = [np.zeros(self.n(L + 1)) for _ in range(3)]
        q = np.zeros(self.n(L))
        lib().orc_stokes_apply(self.h, L, dp(u[0]), dp(u[1]), dp(u[2]), dp(p), dp(v[0]), dp(v[1]), dp(v[2]), dp(q))
        return v, q

    def restrict_all(self, Lf, fine):
        """P1 linear restriction P^T on every node (all-inner functions such as the pressure)."""
        fine = np.ascontiguousarray(fine, dtype=np.float64)
        coarse = np.zeros(self.n(Lf - 1))
        lib().orc_restrict_all(self.h, Lf, dp(fine), dp(coarse))
        return coarse

    def prolongate_all(self, Lc, coarse, fine=None, add=False):
        coarse = np.ascontiguousarray(coarse, dtype=np.float64)
        fine = np.zeros(self.n(Lc + 1)) if fine is None else np.ascontiguousarray(fine, dtype=np.float64).copy()
        lib().orc_prolongate_all(self.h, Lc, dp(coarse), dp(fine), 1 if add else 0)
        return fine

    def pspg_diag(self, L):
        """Diagonal of the assembled P1 PSPG matrix (-tau grad.grad, tau = |T|^(2/3) / 12)."""
        d = np.zeros(self.n(L))
        lib().orc_pspg_diag(self.h, L, dp(d))
        return d

    def uzawa_smooth(self, L, u, p, f, g, omega, velocity_sweeps=2):
        """UzawaSmoother::uzawaSmooth (solvers/UzawaSmoother.hpp:287-423, block-Laplace variant
        without stabilisation) on P2 level L: r_u = f - D^T p; velocity_sweeps times one forward
        multicolour P2 SOR sweep (omega 1) per component; r_p = g - D u; p += omega r_p / diag(PSPG).
        Velocity Dirichlet values are kept; every pressure node is an unknown."""
        nv, npr = self.n(L + 1), self.n(L)
        u = [np.array(x, dtype=np.float64) for x in u]
        p = np.array(p, dtype=np.float64)
        dt, _ = self.stokes_apply(L, [np.zeros(nv)] * 3, p)
        r = [f[k] - dt[k] for k in range(3)]
        for _ in range(velocity_sweeps):
            for k in range(3):
                u[k] = self.p2_sor(L, u[k], r[k], 1.0)
        _, q = self.stokes_apply(L, u, np.zeros(npr))
        p = p + omega * (g - q) / self.pspg_diag(L)
        return u, p

    def uzawa_estimate(self, L, start, iterations, velocity_sweeps=2):
        """estimateUzawaRelaxationParameter (solvers/UzawaSmoother.hpp:52-68): power iterations
        (numerictools/SpectrumEstimation.hpp:57-81) on E = M_lumped^-1 D S D^T from `start`, S the
        velocity sweeps of the Uzawa smoother from zero; 2-norms over every pressure node."""
        nv, npr = self.n(L + 1), self.n(L)
        lumped = np.zeros(npr)
        lib().orc_lumped_mass(self.h, L, dp(lumped))

        def E(v):
            dt, _ = self.stokes_apply(L, [np.zeros(nv)] * 3, v)
            u = [np.zeros(nv) for _ in range(3)]
            for _ in range(velocity_sweeps):
                for k in range(3):
                    u[k] = self.p2_sor(L, u[k], dt[k], 1.0)
            _, q = self.stokes_apply(L, u, np.zeros(npr))
            return q / lumped

        it = np.asarray(start, dtype=np.float64) / np.linalg.norm(start)
        aux = E(it)
        radius = 0.0
        for _ in range(iterations):
            it = aux / np.linalg.norm(aux)
            aux = E(it)
            radius = float(it @ aux)
        return radius

    def stokes_residual(self, L, u, p, f, g):
        v, q = self.stokes_apply(L, u, p)
        dv = self.dirichlet(L + 1)
        return [np.where(dv, 0.0, f[k] - v[k]) for k in range(3)], g - q

    def stokes_coarse_solve(self, L, u, p, f, g):
        """u, p += K^+ (b - K x) on the unknowns of level L (inner velocity DoFs, every pressure
        DoF); K^+ the pseudo-inverse of the assembled block operator (numpy)."""
        dv = self.dirichlet(L + 1)
        free = np.where(~dv)[0]
        nf, npr = len(free), self.n(L)
        n = 3 * nf + npr
        K = np.zeros((n, n))
        for c in range(n):
            e = np.zeros(n)
            e[c] = 1.0
            uu = [np.zeros(self.n(L + 1)) for _ in range(3)]
            for k in range(3):
                uu[k][free] = e[k * nf:(k + 1) * nf]
            v, q = self.stokes_apply(L, uu, e[3 * nf:])
            K[:, c] = np.concatenate([v[0][free], v[1][free], v[2][free], q])
        K = 0.5 * (K + K.T)
        ru, rp = self.stokes_residual(L, u, p, f, g)
        x = np.linalg.pinv(K, rcond=1e-10, hermitian=True) @ np.concatenate([ru[0][free], ru[1][free], ru[2][free], rp])
        u = [np.array(x_, dtype=np.float64) for x_ in u]
        for k in range(3):
            u[k][free] += x[k * nf:(k + 1) * nf]
        return u, p + x[3 * nf:]

    def stokes_uzawa_cycle(self, L, minL, u, p, f, g, pre, post, omega, velocity_sweeps=2):
        """One V-cycle of GeometricMultigridSolver (GeometricMultigridSolver.hpp:136-235) on the
        Taylor-Hood system with the Uzawa smoother and the composite transfers (quadratic on the
        velocity, linear on the pressure), the pseudo-inverse on level minL."""
        if L == minL:
            return self.stokes_coarse_solve(L, u, p, f, g)
        for _ in range(pre):
            u, p = self.uzawa_smooth(L, u, p, f, g, omega, velocity_sweeps)
        ru, rp = self.stokes_residual(L, u, p, f, g)
        dc = self.dirichlet(L)
        fc = [np.where(dc, 0.0, self.p2_restrict(L, ru[k])) for k in range(3)]
        gc = self.restrict_all(L, rp)
        uc, pc = self.stokes_uzawa_cycle(L - 1, minL, [np.zeros(self.n(L))] * 3, np.zeros(self.n(L - 1)), fc, gc, pre,
                                         post, omega, velocity_sweeps)
        dv = self.dirichlet(L + 1)
        u = [np.where(dv, u[k], self.p2_prolongate(L - 1, uc[k], u[k], add=True)) for k in range(3)]
        p = self.prolongate_all(L - 1, pc, p, add=True)
        for _ in range(post):
            u, p = self.uzawa_smooth(L, u, p, f, g, omega, velocity_sweeps)
        return u, p

    def cell_local_stencil(self, L, cell, x, y, z, form=0):
        out = np.zeros(15)
        lib().orc_cell_local_stencil(self.h, L, cell, x, y, z, form, dp(out))
        return out


def p2_element_laplace(coords4x3):
    """P2 Laplace element matrix (vertices, then edges (0,1),(0,2),(0,3),(1,2),(1,3),(2,3))."""
    c = np.ascontiguousarray(coords4x3, dtype=np.float64).reshape(12)
    K = np.zeros(100)
    lib().orc_p2_element_laplace(dp(c), dp(K))
    return K.reshape(10, 10)


def p2p1_div_element(coords4x3):
    """Taylor-Hood divergence element [3][4][10] (P1 vertex, P2 node in the oracle's order)."""
    c = np.ascontiguousarray(coords4x3, dtype=np.float64).reshape(12)
    D = np.zeros(120)
    lib().orc_p2p1_div_element(dp(c), dp(D))
    return D.reshape(3, 4, 10)


def element_laplace(coords4x3):
    c = np.ascontiguousarray(coords4x3, dtype=np.float64).reshape(12)
    K = np.zeros(16)
    lib().orc_element_laplace(dp(c), dp(K))
    return K.reshape(4, 4)


def element_mass(coords4x3):
    c = np.ascontiguousarray(coords4x3, dtype=np.float64).reshape(12)
    K = np.zeros(16)
    lib().orc_element_mass(dp(c), dp(K))
    return K.reshape(4, 4)


def cuboid_mesh(lo, hi, nx, ny, nz):
    """Restatement of MeshInfo::meshCuboid (src/hyteg/mesh/MeshGenCuboid.cpp:32-171): vertex
    coordinates and the six tetrahedra per sub-cube in their frame order."""
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    h = (hi - lo) / np.array([nx, ny, nz])
    coords = []
    for iz in range(nz + 1):
        for iy in range(ny + 1):
            for ix in range(nx + 1):
                coords.append(lo + h * np.array([ix, iy, iz]))
    tnode = [[4, 5, 7, 3], [0, 3, 1, 4], [4, 1, 5, 3], [5, 6, 7, 2], [1, 3, 2, 5], [7, 2, 3, 5]]
    off = [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]]

    def vid(i, j, k):
        return k * (nx + 1) * (ny + 1) + j * (nx + 1) + i

    tets = []
    for iz in range(nz):
        for iy in range(ny):
            for ix in range(nx):
                for t in range(6):
                    tets.append([vid(ix + off[m][0], iy + off[m][1], iz + off[m][2]) for m in tnode[t]])
    return np.array(coords), np.array(tets, dtype=np.int32)


class RefCycle:
    """One V(pre, post) cycle of the reference's P1 multigrid in the reference's own layout,
    through the reference's generated kernels (oracle/ref_cycle.cpp in oracle/_ref): the timed
    CPU baseline. Everything it needs comes from the oracle: the macro-mesh (`coords`, `tets`,
    e.g. `cuboid_mesh`), each cell's 15-point stencil and its one-sided face stencil on level 2
    (`Oracle.cell_local_stencil`; level l uses them scaled by 2^(2 - l)), each face's neighbour
    cells with their cell-local vertex IDs, and the neighbour-cell counts of every cell's edges,
    faces and vertices (the scaling of the transfer kernels, P1toP1LinearRestriction.cpp:186-233).
    The right-hand side and initial guess are seeded values in [-1, 1)."""

    EDGES = [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (2, 3)]
    FACES = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]

    def __init__(self, coords, tets, L, pre=3, post=3, seed=1):
        r = ref_lib()
        if r is None:
            raise RuntimeError("oracle/_ref (the reference's kernels) was not built")
        self._r = r
        r.ref_cycle_create.restype = c_void_p
        r.ref_cycle_create.argtypes = [c_int, c_int, c_int, P(c_double), P(c_double), P(c_int), P(c_int), P(c_int),
                                       P(c_double), c_int, c_int, ctypes.c_uint]
        r.ref_cycle_destroy.argtypes = [c_void_p]
        r.ref_cycle_destroy.restype = None
        r.ref_cycle_run.argtypes = [c_void_p, c_int, c_double]
        r.ref_cycle_run.restype = c_int
        r.ref_cycle_checksum.argtypes = [c_void_p]
        r.ref_cycle_checksum.restype = c_double
        tets = [list(map(int, t)) for t in tets]
        nc = len(tets)
        orc = Oracle(coords, np.array(tets, dtype=np.int32), 2)
        cellW = np.array([orc.cell_local_stencil(2, c, 1, 1, 1) for c in range(nc)])
        del orc
        faces = {}
        for c, t in enumerate(tets):
            for fl in self.FACES:
                key = tuple(sorted(t[i] for i in fl))
                faces.setdefault(key, []).append(c)
        keys = sorted(faces)
        nf = len(keys)
        faceNc = np.zeros(nf, dtype=np.int32)
        faceCell = np.zeros((nf, 2), dtype=np.int32)
        faceLid = np.zeros((nf, 2, 3), dtype=np.int32)
        faceW = np.zeros((nf, 2, 15))
        # one-sided face stencil of each (face, neighbour cell) in the face-local frame (x along
        # the face's vertices 0 -> 1, y along 0 -> 2, z into the cell): the stencil at a face point
        # of the cell re-ordered as (face vertices, opposite vertex)
        sides = []
        for f, key in enumerate(keys):
            cells = sorted(faces[key])
            faceNc[f] = len(cells)
            for k, c in enumerate(cells):
                faceCell[f, k] = c
                faceLid[f, k] = [tets[c].index(v) for v in key]
                sides.append(list(key) + [v for v in tets[c] if v not in key])
        so = Oracle(coords, np.array(sides, dtype=np.int32), 2)
        i = 0
        for f in range(nf):
            for k in range(faceNc[f]):
                faceW[f, k] = so.cell_local_stencil(2, i, 1, 1, 0)
                i += 1
        del so
        vcount, ecount = {}, {}
        for t in tets:
            for v in t:
                vcount[v] = vcount.get(v, 0) + 1
            for a, b in self.EDGES:
                e = tuple(sorted((t[a], t[b])))
                ecount[e] = ecount.get(e, 0) + 1
        counts = np.zeros((nc, 14))
        for c, t in enumerate(tets):
            counts[c, :6] = [ecount[tuple(sorted((t[a], t[b])))] for a, b in self.EDGES]
            counts[c, 6:10] = [len(faces[tuple(sorted(t[i] for i in fl))]) for fl in self.FACES]
            counts[c, 10:] = [vcount[v] for v in t]
        self.L, self.nc, self.nf = L, nc, nf
        self.interior_faces = int((faceNc == 2).sum())
        self._keep = [np.ascontiguousarray(a) for a in (cellW, counts, faceNc, faceCell, faceLid, faceW)]
        cw, cn, fn, fc, fl, fw = self._keep
        self.h = r.ref_cycle_create(L, nc, nf, dp(cw), dp(cn), fn.ctypes.data_as(P(c_int)), fc.ctypes.data_as(P(c_int)),
                                    fl.ctypes.data_as(P(c_int)), dp(fw), pre, post, seed)

    def timed_dofs(self):
        """Inner DoFs whose work one cycle runs on the finest level: the cell interiors and the
        interiors of faces shared by two cells (edges and vertices are not run)."""
        N = 2 ** self.L
        return self.nc * (N - 1) * (N - 2) * (N - 3) // 6 + self.interior_faces * (N - 1) * (N - 2) // 2

    def run(self, threads, relax=1.0):
        """One cycle on `threads` host threads; returns the threads used."""
        return self._r.ref_cycle_run(self.h, threads, relax)

    def checksum(self):
        return self._r.ref_cycle_checksum(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self._r.ref_cycle_destroy(self.h)
            self.h = None

"""Shared test utilities: slot <-> oracle-node matching and a numpy evaluation of the
product's exported halo and stencil tables (independent of the device kernels)."""
import numpy as np
from scipy.spatial import cKDTree

import hyteg_b200 as hg


def tri(w):
    return w * (w + 1) // 2


def tet(w):
    return w * (w + 1) * (w + 2) // 6


def face_idx(w, x, y):
    return y * (w + 1) - y * (y + 1) // 2 + x


def cell_idx(w, x, y, z):
    W = w - z
    return tet(w) - tet(W) + y * (W + 1) - y * (y + 1) // 2 + x


CELL_OFF = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [-1, 1, 0], [1, -1, 0], [0, 0, 1],
                     [-1, 0, 1], [0, -1, 1], [1, -1, 1], [0, 0, -1], [1, 0, -1], [0, 1, -1], [-1, 1, -1]])


def match_slots(slot_xyz, node_xyz, tol=1e-9):
    """Index of the oracle node at each slot's coordinates (-1 for padding slots)."""
    tree = cKDTree(node_xyz)
    d, i = tree.query(slot_xyz)
    i = np.where(d < tol, i, -1)
    return i


def bc_type(mesh, kind, prim):
    if kind == hg.CELL:
        return hg.Inner
    _, _, flag = mesh.primitive(kind, prim)
    return {1: hg.DirichletBoundary, 2: hg.NeumannBoundary, 3: hg.FreeslipBoundary}.get(flag, hg.Inner)


def interior_cell_points(N):
    pts = [(x, y, z) for z in range(1, N) for y in range(1, N) for x in range(1, N) if x + y + z <= N - 1]
    return np.array(pts, dtype=np.int64).reshape(-1, 3)


def interior_face_points(N):
    pts = [(x, y) for y in range(1, N) for x in range(1, N) if x + y <= N - 1]
    return np.array(pts, dtype=np.int64).reshape(-1, 2)


def tables_apply(mesh, L, form, u, flag=hg.Inner):
    """y = A u evaluated from the product's exported stencil tables on a level buffer u whose
    copy slots are consistent; only owned slots of flagged primitives are written (others 0)."""
    N = 2 ** L
    w = N + 1
    nv, ne, nf, nc = mesh.counts()
    y = np.zeros_like(u)
    pts = interior_cell_points(N)
    for c in range(nc):
        if not (bc_type(mesh, hg.CELL, c) & flag) or len(pts) == 0:
            continue
        off, _ = mesh.layout(L, hg.CELL, c)
        wt = mesh.cell_stencil(L, form, c)
        ctr = off + cell_idx(w, pts[:, 0], pts[:, 1], pts[:, 2])
        acc = np.zeros(len(pts))
        for k in range(15):
            q = pts + CELL_OFF[k]
            acc += wt[k] * u[off + cell_idx(w, q[:, 0], q[:, 1], q[:, 2])]
        y[ctr] = acc
    fp = interior_face_points(N)
    for f in range(nf):
        if not (bc_type(mesh, hg.FACE, f) & flag) or len(fp) == 0:
            continue
        off, _ = mesh.layout(L, hg.FACE, f)
        layer, dx, dy, wt = mesh.face_stencil(L, form, f)
        acc = np.zeros(len(fp))
        for k in range(len(wt)):
            x = fp[:, 0] + dx[k]
            yy = fp[:, 1] + dy[k]
            if layer[k] == 0:
                s = face_idx(w, x, yy)
            else:
                s = tri(w) + (layer[k] - 1) * tri(w - 1) + face_idx(w - 1, x, yy)
            acc += wt[k] * u[off + s]
        y[off + face_idx(w, fp[:, 0], fp[:, 1])] = acc
    for kind, count, xs in ((hg.EDGE, ne, np.arange(1, N)), (hg.VERTEX, nv, np.arange(0, 1))):
        for p in range(count):
            if not (bc_type(mesh, kind, p) & flag) or len(xs) == 0:
                continue
            off, _ = mesh.layout(L, kind, p)
            rel, wt = mesh.low_stencil(L, form, kind, p)
            acc = np.zeros(len(xs))
            for k in range(len(wt)):
                acc += wt[k] * u[off + xs + rel[k]]
            y[off + xs] = acc
    return y


def scatter(node_of_slot, g):
    """Level buffer with every slot holding its DoF's value from the global vector g."""
    u = np.zeros(len(node_of_slot))
    m = node_of_slot >= 0
    u[m] = g[node_of_slot[m]]
    return u


def gather_owned(u, node_of_slot, owned, n_nodes):
    """Global vector from the owned slots of a level buffer (NaN where no slot owns the node)."""
    g = np.full(n_nodes, np.nan)
    m = owned == 1
    g[node_of_slot[m]] = u[m]
    return g


def cube(max_level, nx=2):
    from oracle import oracle
    coords, tets = oracle.cuboid_mesh((0, 0, 0), (1, 1, 1), nx, nx, nx)
    mesh = hg.HostMesh.cuboid((0, 0, 0), (1, 1, 1), nx, nx, nx, max_level)
    orc = oracle.Oracle(coords, tets, max_level)
    return coords, tets, mesh, orc


def cell_coefficients(mesh, coords, tets, kfun):
    """Per-macro-cell coefficient kfun(centroid) in the storage's cell order and in the order of
    the oracle's tetrahedron list (the two orders differ; cells are matched by centroid)."""
    nc = mesh.counts()[3]
    cs = np.array([np.mean([mesh.primitive(hg.VERTEX, v)[1] for v in mesh.primitive(hg.CELL, c)[0]], axis=0)
                   for c in range(nc)])
    co = np.array([coords[t].mean(axis=0) for t in tets])
    return kfun(cs), kfun(co)

"""B200-native matrix-free P1 geometric multigrid with HyTeG's operator API.

The classes mirror the reference's host interface (names, argument meaning and error
behaviour) and forward to the C-ABI of libhyteg_b200.so (include/hyteg_b200.h):

  PrimitiveStorage.cuboid(...)      MeshInfo::meshCuboid + SetupPrimitiveStorage
  P1Function(name, storage, lmin, lmax)                 VertexDoFFunction.hpp:66-77
    .interpolate / .assign / .add / .dotGlobal / .communicate
  P1ConstantLaplaceOperator(storage, lmin, lmax)       P1ConstantOperator.hpp:165-166
    .apply(src, dst, level, flag, updateType)           Operator.hpp:73-80
    .smooth_sor / .smooth_gs / *_backwards              Smoothables.hpp:30-102
  P1toP1LinearRestriction().restrict(f, srcLevel, flag)
  P1toP1LinearProlongation().prolongate / prolongateAndAdd
  SORSmoother(relax), CGSolver(...), GeometricMultigridSolver(...)

Every computation runs on the GPU; importing the package without the built library raises.
"""
import ctypes
import os

import numpy as np

from . import _capi
from ._capi import HygError, call, dptr, iptr, i64ptr

# DoFType (src/hyteg/types/types.hpp:35-44)
Inner = 1
DirichletBoundary = 2
NeumannBoundary = 4
FreeslipBoundary = 8
All = 15
# UpdateType
Replace = 0
Add = 1
# primitive kinds
VERTEX, EDGE, FACE, CELL = 0, 1, 2, 3
VCYCLE, WCYCLE = 0, 1


def split_tables_check(level):
    """(points, mismatches) of the colour-split SOR tables of a level, checked on the host."""
    a, b = ctypes.c_int64(), ctypes.c_int64()
    call("hg_split_tables_check", level, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def device_count():
    return _capi.lib.hg_device_count()


class HostMesh:
    """Host-only view of a discretization: topology, reference layout, halo and stencil tables."""

    def __init__(self, handle, max_level):
        self._h = handle
        self.max_level = max_level

    @classmethod
    def cuboid(cls, lo, hi, nx, ny, nz, max_level):
        h = ctypes.c_void_p()
        lo_ = np.asarray(lo, dtype=np.float64)
        hi_ = np.asarray(hi, dtype=np.float64)
        call("hg_mesh_create_cuboid", dptr(lo_), dptr(hi_), nx, ny, nz, max_level, ctypes.byref(h))
        return cls(h, max_level)

    @classmethod
    def from_tets(cls, coords, tets, max_level):
        h = ctypes.c_void_p()
        c = np.ascontiguousarray(coords, dtype=np.float64)
        t = np.ascontiguousarray(tets, dtype=np.int32)
        call("hg_mesh_create_tets", len(c), dptr(c), len(t), iptr(t), max_level, ctypes.byref(h))
        return cls(h, max_level)

    @classmethod
    def cuboid_copies(cls, k, copies, max_level):
        """The solve server's union macro-mesh: `copies` disjoint copies of the k^3 cube."""
        h = ctypes.c_void_p()
        call("hg_mesh_create_cuboid_copies", int(k), int(copies), max_level, ctypes.byref(h))
        return cls(h, max_level)

    @classmethod
    def cubed_domain(cls, cubes, cube_type, max_level):
        """MeshInfo::meshCubedDomain(cubeCoordinates, cubeType) (MeshGenCubedDomain.cpp:115-383)."""
        h = ctypes.c_void_p()
        c = np.ascontiguousarray(cubes, dtype=np.int32).reshape(-1, 3)
        call("hg_mesh_create_cubed_domain", len(c), iptr(c), int(cube_type), max_level, ctypes.byref(h))
        return cls(h, max_level)

    @classmethod
    def from_gmsh(cls, path, max_level, flags_from_file=False):
        """MeshInfo::fromGmshFile (MeshGenFromGmshFile.cpp:31-206), Gmsh 2.2 ASCII."""
        h = ctypes.c_void_p()
        call("hg_mesh_create_gmsh", os.fsencode(path), max_level, 1 if flags_from_file else 0, ctypes.byref(h))
        return cls(h, max_level)

    def write_gmsh(self, path):
        call("hg_mesh_write_gmsh", self._h, os.fsencode(path))

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                _capi.lib.hg_mesh_destroy(self._h)
                self._h = None
        except (AttributeError, TypeError):  # interpreter shutdown
            pass

    def counts(self):
        c = np.zeros(4, dtype=np.int32)
        call("hg_mesh_counts", self._h, iptr(c))
        return tuple(int(v) for v in c)

    def set_cell_coefficients(self, k):
        k = np.ascontiguousarray(k, dtype=np.float64)
        call("hg_mesh_set_cell_coefficients", self._h, dptr(k), len(k))

    def primitive(self, kind, prim):
        ids = np.zeros(4, dtype=np.int32)
        xyz = np.zeros(3)
        flag = ctypes.c_int()
        call("hg_mesh_primitive_vertices", self._h, kind, prim, iptr(ids), dptr(xyz), ctypes.byref(flag))
        return [int(i) for i in ids if i >= 0], xyz, flag.value

    def neighbours(self, kind, prim, which):
        ids = np.zeros(64, dtype=np.int32)
        n = ctypes.c_int()
        call("hg_mesh_primitive_neighbours", self._h, kind, prim, which, iptr(ids), 64, ctypes.byref(n))
        return [int(i) for i in ids[: n.value]]

    def layout(self, level, kind, prim):
        off = ctypes.c_int64()
        size = ctypes.c_int64()
        call("hg_mesh_primitive_layout", self._h, level, kind, prim, ctypes.byref(off), ctypes.byref(size))
        return off.value, size.value

    def level_size(self, level):
        n = ctypes.c_int64()
        call("hg_mesh_level_size", self._h, level, ctypes.byref(n))
        return n.value

    def slot_info(self, level):
        n = self.level_size(level)
        xyz = np.zeros((n, 3))
        owned = np.zeros(n, dtype=np.int8)
        call("hg_mesh_slot_info", self._h, level, dptr(xyz), owned.ctypes.data_as(ctypes.POINTER(ctypes.c_byte)), n)
        return xyz, owned

    def owned_slots(self, level):
        """The level-buffer slot of each entry of the packed owned-DoF order (every DoF of the
        level once, in level-buffer order), as used by P1Function.upload_owned_async."""
        n = ctypes.c_int64()
        call("hg_mesh_owned_slots", self._h, level, None, ctypes.byref(n))
        slots = np.zeros(n.value, dtype=np.int64)
        call("hg_mesh_owned_slots", self._h, level, slots.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(n))
        return slots

    def halo_table(self, level, group):
        n = ctypes.c_int64()
        call("hg_mesh_halo_table", self._h, level, group, None, None, ctypes.byref(n))
        dst = np.zeros(n.value, dtype=np.int64)
        src = np.zeros(n.value, dtype=np.int64)
        call("hg_mesh_halo_table", self._h, level, group, i64ptr(dst), i64ptr(src), ctypes.byref(n))
        return dst, src

    def assembly_plan_check(self, level, form):
        """(targets, terms, mismatches) of the device re-assembly's term lists against the tables."""
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        call("hg_mesh_assembly_plan_check", self._h, level, form, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    def cell_stencil(self, level, form, cell):
        w = np.zeros(15)
        call("hg_mesh_cell_stencil", self._h, level, form, cell, dptr(w))
        return w

    def face_stencil(self, level, form, face):
        layer = np.zeros(32, dtype=np.int32)
        dx = np.zeros(32, dtype=np.int32)
        dy = np.zeros(32, dtype=np.int32)
        w = np.zeros(32)
        n = ctypes.c_int()
        call("hg_mesh_face_stencil", self._h, level, form, face, iptr(layer), iptr(dx), iptr(dy), dptr(w), 32,
             ctypes.byref(n))
        k = n.value
        return layer[:k].copy(), dx[:k].copy(), dy[:k].copy(), w[:k].copy()

    def low_stencil(self, level, form, kind, prim):
        rel = np.zeros(128, dtype=np.int64)
        w = np.zeros(128)
        n = ctypes.c_int()
        call("hg_mesh_low_stencil", self._h, level, form, kind, prim, i64ptr(rel), dptr(w), 128, ctypes.byref(n))
        return rel[: n.value].copy(), w[: n.value].copy()


class PrimitiveStorage:
    """Macro-mesh, device arena and stream of one problem (PrimitiveStorage.hpp:111-521)."""

    def __init__(self, handle, max_level, mesh_args):
        self._h = handle
        self.max_level = max_level
        self._mesh_args = mesh_args
        self._host = None

    @classmethod
    def cuboid(cls, lo, hi, nx, ny, nz, max_level):
        h = ctypes.c_void_p()
        lo_ = np.asarray(lo, dtype=np.float64)
        hi_ = np.asarray(hi, dtype=np.float64)
        call("hg_storage_create_cuboid", dptr(lo_), dptr(hi_), nx, ny, nz, max_level, ctypes.byref(h))
        return cls(h, max_level, ("cuboid", (tuple(lo), tuple(hi), nx, ny, nz)))

    @classmethod
    def from_tets(cls, coords, tets, max_level):
        h = ctypes.c_void_p()
        c = np.ascontiguousarray(coords, dtype=np.float64)
        t = np.ascontiguousarray(tets, dtype=np.int32)
        call("hg_storage_create_tets", len(c), dptr(c), len(t), iptr(t), max_level, ctypes.byref(h))
        return cls(h, max_level, ("tets", (c, t)))

    @classmethod
    def cubed_domain(cls, cubes, cube_type, max_level):
        """MeshInfo::meshCubedDomain + SetupPrimitiveStorage + setMeshBoundaryFlagsOnBoundary(1, 0, true)."""
        h = ctypes.c_void_p()
        c = np.ascontiguousarray(cubes, dtype=np.int32).reshape(-1, 3)
        call("hg_storage_create_cubed_domain", len(c), iptr(c), int(cube_type), max_level, ctypes.byref(h))
        return cls(h, max_level, ("cubed", (c, int(cube_type))))

    @classmethod
    def from_gmsh(cls, path, max_level, flags_from_file=False):
        """MeshInfo::fromGmshFile + SetupPrimitiveStorage; boundary flags from the geometry (as
        setMeshBoundaryFlagsOnBoundary(1, 0, true)) unless flags_from_file."""
        h = ctypes.c_void_p()
        call("hg_storage_create_gmsh", os.fsencode(path), max_level, 1 if flags_from_file else 0, ctypes.byref(h))
        return cls(h, max_level, ("gmsh", (os.fspath(path), bool(flags_from_file))))

    def write_gmsh(self, path):
        """The macro-mesh as a Gmsh 2.2 file; from_gmsh(path, flags_from_file=True) restores it."""
        call("hg_storage_write_gmsh", self._h, os.fsencode(path))

    def close(self):
        if getattr(self, "_h", None):
            _capi.lib.hg_storage_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except (AttributeError, TypeError):  # interpreter shutdown
            pass

    @property
    def handle(self):
        return self._h

    def host(self):
        """HostMesh of the same topology (built lazily; used for coordinates of interpolation)."""
        if self._host is None:
            kind, a = self._mesh_args
            if kind == "cuboid":
                self._host = HostMesh.cuboid(a[0], a[1], a[2], a[3], a[4], self.max_level)
            elif kind == "cubed":
                self._host = HostMesh.cubed_domain(a[0], a[1], self.max_level)
            elif kind == "gmsh":
                self._host = HostMesh.from_gmsh(a[0], self.max_level, a[1])
            else:
                self._host = HostMesh.from_tets(a[0], a[1], self.max_level)
            if getattr(self, "_k", None) is not None:
                self._host.set_cell_coefficients(self._k)
        return self._host

    def counts(self):
        c = np.zeros(4, dtype=np.int32)
        call("hg_storage_counts", self._h, iptr(c))
        return tuple(int(v) for v in c)

    def set_cell_coefficients(self, k):
        k = np.ascontiguousarray(k, dtype=np.float64)
        call("hg_storage_set_cell_coefficients", self._h, dptr(k), len(k))
        self._k = k
        if self._host is not None:
            self._host.set_cell_coefficients(k)

    def set_sor_schedule(self, schedule):
        """0: single-pass wavefront SOR (level buffers double-buffered), 1: in-place colour passes,
        2: the single pass with shorter tiles, 3: colour passes on colour-split copies of the cell
        arrays (converted once per group of sweeps)."""
        call("hg_storage_set_sor_schedule", self._h, int(schedule))

    def set_concurrent_components(self, on):
        """Stokes MINRES: the three velocity V-cycles of a preconditioner application on three
        CUDA streams at once (True, default) or one after another (False); same iterates."""
        call("hg_storage_set_concurrent_components", self.handle, 1 if on else 0)

    def set_sor_fused_phases(self, on):
        """Face, edge and vertex phases of the SOR as one launch per phase (True, default) or one
        launch per colour and halo refresh (False); the sweep is the same bit for bit."""
        call("hg_storage_set_sor_fused_phases", self.handle, 1 if on else 0)

    def set_sor_schedule_level(self, level, schedule, dtype=np.float64):
        """One level's SOR schedule for one precision (-1: the storage-wide schedule)."""
        prec = {np.dtype(np.float64): 8, np.dtype(np.float32): 4}[np.dtype(dtype)]
        call("hg_storage_set_sor_schedule_level", self._h, int(level), prec, int(schedule))

    def autotune_sor(self, minLevel, maxLevel, dtype=np.float64, reps=3):
        """Times the four SOR schedules per level (groups of three sweeps) and keeps the fastest;
        returns {level: (chosen schedule, ms per sweep of schedules 0, 1, 2, 3)}."""
        n = maxLevel - minLevel + 1
        ms = np.zeros(4 * n)
        ch = np.zeros(n, dtype=np.int32)
        prec = {np.dtype(np.float64): 8, np.dtype(np.float32): 4}[np.dtype(dtype)]
        call("hg_storage_autotune_sor", self._h, minLevel, maxLevel, prec, int(reps), dptr(ms), iptr(ch))
        return {minLevel + i: (int(ch[i]),) + tuple(float(ms[4 * i + k]) for k in range(4)) for i in range(n)}

    def set_stream(self, stream_ptr):
        call("hg_storage_set_stream", self._h, ctypes.c_void_p(stream_ptr))

    def owned_count(self, level):
        """Number of DoFs of a level (each once): the size of the packed owned-DoF transfers."""
        n = ctypes.c_int64()
        call("hg_owned_count", self._h, level, ctypes.byref(n))
        return n.value

    def synchronize(self):
        call("hg_storage_synchronize", self._h)

    def set_l2_budget(self, nbytes):
        call("hg_storage_set_l2_budget", self._h, int(nbytes))

    def launch_count(self):
        n = ctypes.c_ulonglong()
        call("hg_storage_launch_count", self._h, ctypes.byref(n))
        return n.value

    def level_size(self, level):
        n = ctypes.c_int64()
        call("hg_level_size", self._h, level, ctypes.byref(n))
        return n.value

    def layout(self, level, kind, prim):
        off = ctypes.c_int64()
        size = ctypes.c_int64()
        call("hg_primitive_layout", self._h, level, kind, prim, ctypes.byref(off), ctypes.byref(size))
        return off.value, size.value


class P1Function:
    """P1 (vertex-DoF) function on levels [minLevel, maxLevel], FP64 or FP32 on the device."""

    def __init__(self, name, storage, minLevel, maxLevel, dtype=np.float64):
        self.name = name
        self.storage = storage
        self.minLevel = minLevel
        self.maxLevel = maxLevel
        self.dtype = np.dtype(dtype)
        prec = {np.dtype(np.float64): 8, np.dtype(np.float32): 4}[self.dtype]
        h = ctypes.c_int()
        call("hg_function_create", storage.handle, minLevel, maxLevel, prec, ctypes.byref(h))
        self.id = h.value

    def __del__(self):
        try:
            st = getattr(self, "storage", None)
            if st is not None and st.handle:
                _capi.lib.hg_function_destroy(st.handle, self.id)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass

    def device_ptr(self, level):
        p = ctypes.c_void_p()
        call("hg_function_device_ptr", self.storage.handle, self.id, level, ctypes.byref(p))
        return p.value

    def to_numpy(self, level):
        n = self.storage.level_size(level)
        a = np.empty(n, dtype=self.dtype)
        call("hg_function_download", self.storage.handle, self.id, level, a.ctypes.data_as(ctypes.c_void_p), n)
        return a

    def from_numpy(self, level, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        call("hg_function_upload", self.storage.handle, self.id, level, a.ctypes.data_as(ctypes.c_void_p), a.size)

    def upload_async(self, level, a, stream):
        """Enqueue the upload of the contiguous host array `a` (pinned memory for an asynchronous
        copy; kept alive by the caller) on the CUDA stream handle `stream`, without waiting."""
        if a.dtype != self.dtype or not a.flags["C_CONTIGUOUS"]:
            raise ValueError("upload_async: a contiguous array of the function's precision is required")
        call("hg_function_upload_async", self.storage.handle, self.id, level, a.ctypes.data_as(ctypes.c_void_p), a.size,
             ctypes.c_void_p(stream))

    def download_async(self, level, a, stream):
        """Enqueue the download of the level buffer into the contiguous host array `a` (pinned
        memory for an asynchronous copy) on the CUDA stream handle `stream`, without waiting; `a`
        holds the values once the stream has passed the copy."""
        if a.dtype != self.dtype or not a.flags["C_CONTIGUOUS"] or not a.flags["WRITEABLE"]:
            raise ValueError("download_async: a writeable contiguous array of the function's precision is required")
        call("hg_function_download_async", self.storage.handle, self.id, level, a.ctypes.data_as(ctypes.c_void_p),
             a.size, ctypes.c_void_p(stream))

    def upload_owned_async(self, level, a, stream):
        """Enqueue the upload of the owned DoFs (packed, level-buffer order, PrimitiveStorage.
        owned_count elements) from the contiguous host array `a` on the CUDA stream handle
        `stream`; the scatter into the level buffer and the halo refresh follow on the storage's
        stream. `a` (pinned for an asynchronous copy) must stay alive until the copy is done."""
        if a.dtype != self.dtype or not a.flags["C_CONTIGUOUS"]:
            raise ValueError("upload_owned_async: a contiguous array of the function's precision is required")
        call("hg_function_upload_owned_async", self.storage.handle, self.id, level,
             a.ctypes.data_as(ctypes.c_void_p), a.size, ctypes.c_void_p(stream))

    def download_owned_async(self, level, a, stream):
        """Enqueue the download of the owned DoFs (packed, level-buffer order) into the contiguous
        host array `a`: packed on the storage's stream, copied on the CUDA stream handle `stream`;
        `a` holds the values once `stream` has passed the copy."""
        if a.dtype != self.dtype or not a.flags["C_CONTIGUOUS"] or not a.flags["WRITEABLE"]:
            raise ValueError("download_owned_async: a writeable contiguous array of the function's precision is required")
        call("hg_function_download_owned_async", self.storage.handle, self.id, level,
             a.ctypes.data_as(ctypes.c_void_p), a.size, ctypes.c_void_p(stream))

    def communicate(self, level):
        call("hg_communicate", self.storage.handle, self.id, level)

    def interpolate(self, value, level, flag=All):
        """Constant (on the device) or callable f(x, y, z) evaluated at every slot's coordinates."""
        if callable(value):
            xyz, owned = self.storage.host().slot_info(level)
            cur = self.to_numpy(level)
            vals = np.asarray(value(xyz[:, 0], xyz[:, 1], xyz[:, 2]), dtype=np.float64)
            mask = _flag_mask(self.storage, level, flag)
            cur[mask] = vals[mask]
            self.from_numpy(level, cur)
        else:
            call("hg_interpolate_const", self.storage.handle, self.id, float(value), level, flag)

    def interpolate_sines(self, amplitude, k, level, flag=All):
        """amplitude * sin(k pi x) sin(k pi y) sin(k pi z), evaluated on the device."""
        p = np.array([amplitude, k, 0.0, 0.0])
        call("hg_interpolate_expr", self.storage.handle, self.id, level, flag, 0, dptr(p))

    def interpolate_linear(self, a, b, c, d, level, flag=All):
        """a + b x + c y + d z, evaluated on the device."""
        p = np.array([a, b, c, d], dtype=np.float64)
        call("hg_interpolate_expr", self.storage.handle, self.id, level, flag, 1, dptr(p))

    def fill_random(self, seed, level, flag=All, lo=-1.0, hi=1.0):
        """Seeded uniform [lo, hi) values at the flagged DoFs (reproducible per topology)."""
        call("hg_function_fill_random", self.storage.handle, self.id, level, flag, ctypes.c_uint64(seed), float(lo),
             float(hi))

    def assign(self, scalars, functions, level, flag=All):
        s = np.ascontiguousarray(scalars, dtype=np.float64)
        f = np.ascontiguousarray([g.id for g in functions], dtype=np.int32)
        call("hg_assign", self.storage.handle, self.id, level, flag, len(f), dptr(s), iptr(f))

    def add(self, scalars, functions, level, flag=All):
        s = np.ascontiguousarray(scalars, dtype=np.float64)
        f = np.ascontiguousarray([g.id for g in functions], dtype=np.int32)
        call("hg_add", self.storage.handle, self.id, level, flag, len(f), dptr(s), iptr(f))

    def copy_from(self, other, level, flag=All, add=False):
        """Copy (with precision conversion) from another function: the FP64 <-> FP32 bridge."""
        call("hg_copy_cast", self.storage.handle, self.id, other.id, level, flag, 1 if add else 0)

    def dotGlobal(self, other, level, flag=All):
        out = ctypes.c_double()
        call("hg_dot", self.storage.handle, self.id, other.id, level, flag, ctypes.byref(out))
        return out.value


def _flag_mask(storage, level, flag):
    """Boolean mask over a level buffer: slots of primitives whose DoFType matches flag."""
    host = storage.host()
    n = host.level_size(level)
    mask = np.zeros(n, dtype=bool)
    counts = host.counts()
    bc = {0: Inner, 1: DirichletBoundary, 2: NeumannBoundary, 3: FreeslipBoundary}
    for kind in range(4):
        for p in range(counts[kind]):
            _, _, mflag = host.primitive(kind, p)
            t = Inner if kind == CELL else bc.get(mflag, Inner)
            if t & flag:
                off, size = host.layout(level, kind, p)
                mask[off:off + size] = True
    return mask


class _P1ConstantOperator:
    FORM = 0

    def __init__(self, storage, minLevel, maxLevel):
        self.storage = storage
        self.minLevel = minLevel
        self.maxLevel = maxLevel
        h = ctypes.c_int()
        call("hg_operator_create", storage.handle, self.FORM, minLevel, maxLevel, ctypes.byref(h))
        self.id = h.value

    def __del__(self):
        try:
            st = getattr(self, "storage", None)
            if st is not None and st.handle:
                _capi.lib.hg_operator_destroy(st.handle, self.id)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass

    def apply(self, src, dst, level, flag, updateType=Replace):
        if src is dst:
            raise ValueError("apply: src and dst must be different functions")
        call("hg_apply", self.storage.handle, self.id, src.id, dst.id, level, flag, updateType)

    def reassemble(self, on_device=True):
        """Stencils from the storage's current cell coefficients, on the device (bit-identical to
        the host assembly) or on the host."""
        call("hg_operator_reassemble", self.storage.handle, self.id, 1 if on_device else 0)

    def apply_primitives(self, src, dst, level, flag, updateType=Replace, kinds=15, refresh=True):
        """Only the kernels of the selected primitive kinds (bit set over VERTEX..CELL)."""
        call("hg_apply_primitives", self.storage.handle, self.id, src.id, dst.id, level, flag, updateType, kinds,
             1 if refresh else 0)

    def residual(self, x, b, r, level, flag):
        """r = b - A x (fused apply + assign of GeometricMultigridSolver.hpp:185-186)."""
        call("hg_residual", self.storage.handle, self.id, x.id, b.id, r.id, level, flag)

    def smooth_sor(self, dst, rhs, relax, level, flag):
        call("hg_smooth_sor", self.storage.handle, self.id, dst.id, rhs.id, float(relax), level, flag, 0)

    def smooth_sor_backwards(self, dst, rhs, relax, level, flag):
        call("hg_smooth_sor", self.storage.handle, self.id, dst.id, rhs.id, float(relax), level, flag, 1)

    def smooth_sor_primitives(self, dst, rhs, relax, level, flag, kinds=15, refresh=True, backwards=False):
        """The SOR phases of the selected primitive kinds only (bit set over VERTEX..CELL)."""
        call("hg_smooth_sor_primitives", self.storage.handle, self.id, dst.id, rhs.id, float(relax), level, flag,
             1 if backwards else 0, kinds, 1 if refresh else 0)

    def smooth_gs(self, dst, rhs, level, flag):
        self.smooth_sor(dst, rhs, 1.0, level, flag)

    def smooth_gs_backwards(self, dst, rhs, level, flag):
        self.smooth_sor_backwards(dst, rhs, 1.0, level, flag)


class P1ConstantLaplaceOperator(_P1ConstantOperator):
    """-div(k grad u) with k piecewise constant per macro-cell (k = 1 unless set on the storage)."""
    FORM = 0


class P1ConstantMassOperator(_P1ConstantOperator):
    FORM = 1


class P1PSPGOperator(_P1ConstantOperator):
    """-tau grad p . grad q with tau = |T|^(2/3) / 12 per micro-cell (pressure stabilisation)."""
    FORM = 2


class P1toP1LinearRestriction:
    def restrict(self, function, sourceLevel, flag):
        call("hg_restrict", function.storage.handle, function.id, sourceLevel, flag)


class P1toP1LinearProlongation:
    def prolongate(self, function, sourceLevel, flag):
        call("hg_prolongate", function.storage.handle, function.id, sourceLevel, flag, 0)

    def prolongateAndAdd(self, function, sourceLevel, flag):
        call("hg_prolongate", function.storage.handle, function.id, sourceLevel, flag, 1)


class SORSmoother:
    def __init__(self, relax):
        self.relax = relax

    def solve(self, A, x, b, level):
        A.smooth_sor(x, b, self.relax, level, Inner | NeumannBoundary)


class CGSolver:
    def __init__(self, storage, minLevel, maxLevel, maxIter=2 ** 31 - 1, tolerance=1e-16):
        self.storage = storage
        self.maxIter = maxIter
        self.tolerance = tolerance
        self.iterations = 0
        self.residual = 0.0

    def solve(self, A, x, b, level):
        it = ctypes.c_int()
        res = ctypes.c_double()
        call("hg_cg_solve", self.storage.handle, A.id, x.id, b.id, level, int(min(self.maxIter, 2 ** 31 - 1)),
             float(self.tolerance), ctypes.byref(it), ctypes.byref(res))
        self.iterations = it.value
        self.residual = res.value


class GeometricMultigridSolver:
    """GeometricMultigridSolver.hpp:42-116. The smoother must be an SORSmoother and the coarse
    solver a CGSolver; transfers are the linear P1 restriction/prolongation."""

    def __init__(self, storage, smoother, coarseSolver, restrictionOperator, prolongationOperator, minLevel, maxLevel,
                 preSmoothSteps=3, postSmoothSteps=3, smoothIncrementOnCoarserGrids=0, cycleType=VCYCLE,
                 A=None, dtype=np.float64):
        if not isinstance(smoother, SORSmoother):
            raise TypeError("The SOR-Smoother requires the SORSmoothable interface.")
        if not isinstance(coarseSolver, CGSolver):
            raise TypeError("coarse solver must be a CGSolver")
        if smoothIncrementOnCoarserGrids != 0:
            raise ValueError("smoothIncrementOnCoarserGrids != 0 is not supported")
        self.storage = storage
        self.args = (minLevel, maxLevel, preSmoothSteps, postSmoothSteps, float(smoother.relax), cycleType,
                     int(min(coarseSolver.maxIter, 2 ** 31 - 1)), float(coarseSolver.tolerance),
                     {np.dtype(np.float64): 8, np.dtype(np.float32): 4}[np.dtype(dtype)])
        self._cache = {}

    def _handle(self, A):
        if A.id not in self._cache:
            h = ctypes.c_int()
            a = self.args
            call("hg_gmg_create", self.storage.handle, A.id, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8],
                 ctypes.byref(h))
            self._cache[A.id] = h.value
        return self._cache[A.id]

    def solve(self, A, x, b, level):
        call("hg_gmg_solve", self.storage.handle, self._handle(A), x.id, b.id, level)

    def set_graphs(self, A, enable):
        """Replay cycles from captured CUDA graphs (default on; identical results)."""
        call("hg_gmg_set_graphs", self.storage.handle, self._handle(A), 1 if enable else 0)

    def set_compact(self, A, max_dofs, cluster_blocks=1):
        """Run the coarse levels with at most max_dofs unknowns per group as one launch per cycle
        (0: off; default 6000 unknowns, one block per group)."""
        call("hg_gmg_set_compact", self.storage.handle, self._handle(A), int(max_dofs), int(cluster_blocks))

    def compact_top(self, A):
        """Highest level of the compact coarse cycle (-1: none)."""
        t = ctypes.c_int()
        call("hg_gmg_compact_top", self.storage.handle, self._handle(A), ctypes.byref(t))
        return t.value

    def set_timing(self, A, enable):
        """Device-timed phases in a timing tree (the reference's WcTimingTree nodes); cycles run
        eagerly while on."""
        call("hg_gmg_set_timing", self.storage.handle, self._handle(A), 1 if enable else 0)

    def timing_tree(self, A):
        """The timing tree as a dict (waLBerla TimingTree JSON layout, seconds)."""
        import json
        n = ctypes.c_int64()
        call("hg_gmg_timing_json", self.storage.handle, self._handle(A), None, 0, ctypes.byref(n))
        buf = ctypes.create_string_buffer(n.value + 1)
        call("hg_gmg_timing_json", self.storage.handle, self._handle(A), buf, n.value + 1, ctypes.byref(n))
        return json.loads(buf.value.decode())

    def solve_to(self, A, x, b, level, tol, max_iter=100):
        """Iterate to a relative residual tol (FP64 x, b). An FP32 solver runs FP64 defect
        correction around FP32 cycles. Returns (iterations, relative residual, history)."""
        it = ctypes.c_int()
        rel = ctypes.c_double()
        hist = np.zeros(max_iter)
        call("hg_gmg_solve_to", self.storage.handle, self._handle(A), x.id, b.id, level, float(tol), int(max_iter),
             ctypes.byref(it), ctypes.byref(rel), dptr(hist), int(max_iter))
        return it.value, rel.value, hist[: it.value].copy()

    def __del__(self):
        try:
            st = getattr(self, "storage", None)
            if st is not None and st.handle:
                for h in self._cache.values():
                    _capi.lib.hg_gmg_destroy(st.handle, h)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass


class P2Function:
    """P2 (quadratic) function on levels [minLevel, maxLevel] (P2Function.hpp of the reference).
    Its DoFs on level L are the vertex DoFs of level L + 1 (micro-vertices at even lattice
    coordinates, micro-edge midpoints at the others), held by a vertex-DoF function `v` of
    levels [minLevel + 1, maxLevel + 1]; level arguments here are P2 levels."""

    def __init__(self, name, storage, minLevel, maxLevel, dtype=np.float64):
        self.name = name
        self.storage = storage
        self.minLevel, self.maxLevel = minLevel, maxLevel
        self.v = P1Function(name, storage, minLevel + 1, maxLevel + 1, dtype=dtype)
        self.id = self.v.id
        self.dtype = self.v.dtype

    def to_numpy(self, level):
        return self.v.to_numpy(level + 1)

    def from_numpy(self, level, a):
        self.v.from_numpy(level + 1, a)

    def communicate(self, level):
        self.v.communicate(level + 1)

    def fill_random(self, seed, level, flag=All, lo=-1.0, hi=1.0):
        self.v.fill_random(seed, level + 1, flag, lo, hi)

    def interpolate(self, value, level, flag=All):
        self.v.interpolate(value, level + 1, flag)

    def assign(self, scalars, functions, level, flag=All):
        self.v.assign(scalars, [f.v for f in functions], level + 1, flag)

    def dotGlobal(self, other, level, flag=All):
        return self.v.dotGlobal(other.v, level + 1, flag)


class P2ConstantLaplaceOperator:
    """P2ConstantLaplaceOperator (P2ConstantOperator.hpp:154-157): element-wise P2 Laplace with
    the per-macro-cell coefficient, on levels [minLevel, maxLevel] (the storage needs
    maxLevel + 1)."""

    def __init__(self, storage, minLevel, maxLevel):
        self.storage = storage
        h = ctypes.c_int()
        call("hg_p2_operator_create", storage.handle, 0, minLevel, maxLevel, ctypes.byref(h))
        self.id = h.value

    def apply(self, src, dst, level, flag=Inner):
        call("hg_p2_apply", self.storage.handle, self.id, src.id, dst.id, level, flag)

    def residual(self, x, b, r, level, flag=Inner):
        call("hg_p2_residual", self.storage.handle, self.id, x.id, b.id, r.id, level, flag)

    def smooth_sor(self, dst, rhs, relax, level, flag=Inner | NeumannBoundary):
        call("hg_p2_smooth_sor", self.storage.handle, self.id, dst.id, rhs.id, float(relax), level, flag, 0)

    def smooth_sor_backwards(self, dst, rhs, relax, level, flag=Inner | NeumannBoundary):
        call("hg_p2_smooth_sor", self.storage.handle, self.id, dst.id, rhs.id, float(relax), level, flag, 1)

    def __del__(self):
        try:
            st = getattr(self, "storage", None)
            if st is not None and st.handle:
                _capi.lib.hg_p2_operator_destroy(st.handle, self.id)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass


class P2toP2QuadraticProlongation:
    """P2toP2QuadraticProlongation: quadratic interpolation from P2 level `level` to level + 1."""

    def prolongate(self, f, level, flag=All):
        call("hg_p2_prolongate", f.storage.handle, f.id, level, flag, 0)

    def prolongateAndAdd(self, f, level, flag=All):
        call("hg_p2_prolongate", f.storage.handle, f.id, level, flag, 1)


class P2toP2QuadraticRestriction:
    """P2toP2QuadraticRestriction: transpose of the quadratic prolongation, from P2 level
    `level` to level - 1."""

    def restrict(self, f, level, flag=All):
        call("hg_p2_restrict", f.storage.handle, f.id, level, flag)


class P2GeometricMultigridSolver:
    """GeometricMultigridSolver for P2ConstantLaplaceOperator: multicolour P2 SOR, quadratic
    transfers, an exact solve on the coarsest level (CG when it has more than 1024 unknowns);
    FP64. Cycles are replayed from captured CUDA graphs unless set_graphs(False)."""

    def __init__(self, storage, A, minLevel, maxLevel, preSmoothSteps=3, postSmoothSteps=3, relax=1.0,
                 coarseMaxIter=1000, coarseTolerance=1e-16):
        self.storage = storage
        h = ctypes.c_int()
        call("hg_p2_gmg_create", storage.handle, A.id, minLevel, maxLevel, preSmoothSteps, postSmoothSteps,
             float(relax), int(coarseMaxIter), float(coarseTolerance), ctypes.byref(h))
        self.id = h.value

    def solve(self, x, b, level):
        call("hg_p2_gmg_solve", self.storage.handle, self.id, x.id, b.id, level)

    def set_graphs(self, enable):
        call("hg_p2_gmg_set_graphs", self.storage.handle, self.id, 1 if enable else 0)

    def solve_to(self, x, b, level, tol, max_iter=100):
        it = ctypes.c_int()
        rel = ctypes.c_double()
        hist = np.zeros(max_iter)
        call("hg_p2_gmg_solve_to", self.storage.handle, self.id, x.id, b.id, level, float(tol), int(max_iter),
             ctypes.byref(it), ctypes.byref(rel), dptr(hist), int(max_iter))
        return it.value, rel.value, hist[: it.value].copy()

    def __del__(self):
        try:
            st = getattr(self, "storage", None)
            if st is not None and st.handle:
                _capi.lib.hg_p2_gmg_destroy(st.handle, self.id)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass


class P2P1TaylorHoodStokesOperator:
    """P2P1TaylorHoodStokesOperator: velocity = three P2Functions, pressure = a P1Function whose
    level L is the pressure of P2 level L. apply(u, p, v, q, level): v = A u + D^T p, q = D u."""

    def __init__(self, storage, minLevel, maxLevel):
        self.storage = storage
        h = ctypes.c_int()
        call("hg_p2p1_stokes_create", storage.handle, minLevel, maxLevel, ctypes.byref(h))
        self.id = h.value

    def apply(self, u, p, v, q, level, flagVelocity=Inner | NeumannBoundary, flagPressure=All):
        ui = (ctypes.c_int * 3)(*[f.id for f in u])
        vi = (ctypes.c_int * 3)(*[f.id for f in v])
        call("hg_p2p1_stokes_apply", self.storage.handle, self.id, ui, p.id, vi, q.id, level, flagVelocity,
             flagPressure)

    def minres(self, u, p, f, g, level, nu=2, max_iter=500, tol=1e-8, precondition_dtype=np.float64):
        """MinResSolver with the block-diagonal preconditioner (symmetric P2 V(nu, nu) per velocity
        component, lumped P1 mass on the pressure); precondition_dtype float32 runs the V-cycles in
        FP32 inside the FP64 iteration. Returns (iterations, relative residual, history)."""
        ui = (ctypes.c_int * 3)(*[x.id for x in u])
        fi = (ctypes.c_int * 3)(*[x.id for x in f])
        it = ctypes.c_int()
        rel = ctypes.c_double()
        hist = np.zeros(max_iter)
        prec = {np.dtype(np.float64): 8, np.dtype(np.float32): 4}[np.dtype(precondition_dtype)]
        call("hg_p2p1_stokes_minres_mixed", self.storage.handle, self.id, ui, p.id, fi, g.id, level, int(nu),
             int(max_iter), float(tol), prec, ctypes.byref(it), ctypes.byref(rel), dptr(hist), int(max_iter))
        return it.value, rel.value, hist[: it.value].copy()

    def __del__(self):
        try:
            st = getattr(self, "storage", None)
            if st is not None and st.handle:
                _capi.lib.hg_p2_operator_destroy(st.handle, self.id)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass


class UzawaSmoother:
    """UzawaSmoother for P2P1TaylorHoodStokesOperator (block-Laplace variant without stabilisation):
    r_u = f - D^T p; numGSIterationsVelocity forward P2 SOR sweeps (omega 1) per velocity
    component; p += relaxParam (g - D u) / diag(PSPG). Velocity DoFs flagged Inner | Neumann are
    unknowns, every pressure DoF is one. solve(u, p, f, g, level) is one smoothing step."""

    def __init__(self, storage, S, minLevel, maxLevel, relaxParam, numGSIterationsVelocity=2):
        self.storage, self.S = storage, S
        self.minLevel, self.maxLevel = minLevel, maxLevel
        self.relax, self.sweeps = float(relaxParam), int(numGSIterationsVelocity)
        self._native = _StokesUzawaGmg(storage, S, minLevel, maxLevel, 0, 0, self.relax, self.sweeps)

    def solve(self, u, p, f, g, level):
        ui = (ctypes.c_int * 3)(*[x.id for x in u])
        fi = (ctypes.c_int * 3)(*[x.id for x in f])
        call("hg_p2p1_stokes_uzawa_smooth", self.storage.handle, self._native.id, ui, p.id, fi, g.id, level)


def estimateUzawaRelaxationParameter(storage, S, level, numPowerIterations=20, numGSIterationsVelocity=2, seed=42):
    """estimateUzawaRelaxationParameter: the spectral radius of M_lumped^-1 D S D^T (S: the Uzawa
    smoother's velocity sweeps from zero) by power iterations from seeded uniform [0, 1) values."""
    native = _StokesUzawaGmg(storage, S, level, level, 0, 0, 1.0, numGSIterationsVelocity)
    w = ctypes.c_double()
    call("hg_p2p1_stokes_uzawa_estimate_omega", storage.handle, native.id, level, int(numPowerIterations),
         ctypes.c_uint64(seed), ctypes.byref(w))
    return w.value


class _StokesUzawaGmg:
    def __init__(self, storage, S, minLevel, maxLevel, pre, post, relax, sweeps):
        self.storage = storage
        h = ctypes.c_int()
        call("hg_p2p1_stokes_uzawa_gmg_create", storage.handle, S.id, minLevel, maxLevel, int(pre), int(post),
             float(relax), int(sweeps), ctypes.byref(h))
        self.id = h.value

    def __del__(self):
        try:
            st = getattr(self, "storage", None)
            if st is not None and st.handle:
                _capi.lib.hg_p2p1_stokes_uzawa_gmg_destroy(st.handle, self.id)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass


class StokesGeometricMultigridSolver:
    """GeometricMultigridSolver for P2P1TaylorHoodStokesOperator with an UzawaSmoother and the
    P2P1StokesToP2P1Stokes restriction / prolongation (quadratic velocity, linear pressure); the
    coarsest level is solved by the pseudo-inverse of the operator on its unknowns (up to 1024 of
    them), a larger one by preconditioned MINRES to a relative residual of 1e-11."""

    def __init__(self, storage, S, smoother, minLevel, maxLevel, preSmoothSteps=2, postSmoothSteps=2):
        self.storage = storage
        self._native = _StokesUzawaGmg(storage, S, minLevel, maxLevel, preSmoothSteps, postSmoothSteps,
                                       smoother.relax, smoother.sweeps)

    def solve(self, u, p, f, g, level):
        ui = (ctypes.c_int * 3)(*[x.id for x in u])
        fi = (ctypes.c_int * 3)(*[x.id for x in f])
        call("hg_p2p1_stokes_uzawa_gmg_solve", self.storage.handle, self._native.id, ui, p.id, fi, g.id, level)

    def solve_to(self, u, p, f, g, level, tol, max_iter=100):
        ui = (ctypes.c_int * 3)(*[x.id for x in u])
        fi = (ctypes.c_int * 3)(*[x.id for x in f])
        it = ctypes.c_int()
        rel = ctypes.c_double()
        hist = np.zeros(max_iter)
        call("hg_p2p1_stokes_uzawa_gmg_solve_to", self.storage.handle, self._native.id, ui, p.id, fi, g.id, level,
             float(tol), int(max_iter), ctypes.byref(it), ctypes.byref(rel), dptr(hist), int(max_iter))
        return it.value, rel.value, hist[: it.value].copy()


class SolveServer:
    """Continuous-batching server of P1 Poisson solves (hg_server_*): requests on the unit cube
    split into k^3 sub-cubes of 6 tetrahedra at a refinement level, constant coefficient, seeded
    uniform[-1,1] right-hand side, solved to a relative residual. precision 4 runs FP64 defect
    correction around FP32 V(3,3) cycles, precision 8 plain FP64 V(3,3) cycles."""

    def __init__(self, workers=8, hbm_budget_bytes=64 << 30, precision=4):
        h = ctypes.c_void_p()
        call("hg_server_create", int(workers), int(hbm_budget_bytes), int(precision), ctypes.byref(h))
        self._h = h

    def prewarm(self, k, level):
        call("hg_server_prewarm", self._h, int(k), int(level))

    def set_batching(self, max_level):
        """Solve queued requests of levels up to max_level (-1: none) together, several in one
        union hierarchy of their shape (see prewarm_batch), when at least two of a shape wait."""
        call("hg_server_set_batching", self._h, int(max_level))

    def prewarm_batch(self, k, level, copies):
        """Build one resident union hierarchy: `copies` disjoint copies of shape (k, level) in one
        storage, which solves up to `copies` requests of that shape at once."""
        call("hg_server_prewarm_batch", self._h, int(k), int(level), int(copies))

    def submit(self, k, level, coefficient=1.0, seed=0, tol=1e-8, max_iter=100, keep_solution=False):
        i = ctypes.c_int64()
        call("hg_server_submit", self._h, int(k), int(level), float(coefficient), ctypes.c_uint64(seed), float(tol),
             int(max_iter), 1 if keep_solution else 0, ctypes.byref(i))
        return i.value

    def wait(self, rid, timeout=-1.0):
        d = ctypes.c_int()
        call("hg_server_wait", self._h, int(rid), float(timeout), ctypes.byref(d))
        return bool(d.value)

    def result(self, rid):
        """dict(status, iterations, rel_residual, t_submit, t_start, t_solve, t_end, inner_dofs,
        built_hierarchy, batch_size); raises for a failed request. batch_size: the requests solved
        together with it in one union hierarchy (1: solved alone). built_hierarchy: the request's
        shape had no resident hierarchy when it was admitted, so one was built for it (its setup
        time, t_solve - t_start, includes that)."""
        st, it = ctypes.c_int(), ctypes.c_int()
        rel = ctypes.c_double()
        t = np.zeros(4)
        n = ctypes.c_int64()
        built = ctypes.c_int()
        call("hg_server_result", self._h, int(rid), ctypes.byref(st), ctypes.byref(it), ctypes.byref(rel), dptr(t),
             ctypes.byref(n))
        call("hg_server_request_setup", self._h, int(rid), ctypes.byref(built))
        batch = ctypes.c_int()
        call("hg_server_request_batch", self._h, int(rid), ctypes.byref(batch))
        return {"status": st.value, "iterations": it.value, "rel_residual": rel.value, "t_submit": t[0],
                "t_start": t[1], "t_solve": t[2], "t_end": t[3], "inner_dofs": n.value,
                "built_hierarchy": bool(built.value), "batch_size": batch.value}

    def solution(self, rid):
        n = ctypes.c_int64()
        call("hg_server_solution", self._h, int(rid), None, 0, ctypes.byref(n))
        out = np.empty(n.value)
        call("hg_server_solution", self._h, int(rid), dptr(out), n.value, ctypes.byref(n))
        return out

    def stats(self):
        s = np.zeros(6, dtype=np.int64)
        call("hg_server_stats", self._h, s.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        keys = ("admitted", "completed", "failed", "resident_hierarchies", "resident_bytes", "peak_bytes")
        return dict(zip(keys, (int(v) for v in s)))

    def close(self):
        if getattr(self, "_h", None):
            call("hg_server_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except (AttributeError, TypeError):  # interpreter shutdown
            pass

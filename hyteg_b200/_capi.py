"""ctypes binding of include/hyteg_b200.h (the library is built in-tree by hyteg_b200.build).

Importing this module fails loudly when libhyteg_b200.so is missing: there is no fallback.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhyteg_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        "hyteg_b200: %s is missing; build it with `python -m hyteg_b200.build` (nvcc, sm_100a)" % LIB_PATH
    )

lib = ctypes.CDLL(LIB_PATH)

c_int = ctypes.c_int
c_uint = ctypes.c_uint
c_double = ctypes.c_double
c_int64 = ctypes.c_int64
c_void_p = ctypes.c_void_p
c_char_p = ctypes.c_char_p
P = ctypes.POINTER

HG_OK, HG_ERR_ARG, HG_ERR_CUDA, HG_ERR_OOM, HG_ERR_STATE, HG_ERR_NUMERIC, HG_ERR_INTERNAL = range(7)


class HygError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("hyteg_b200 error %d: %s" % (code, msg))
        self.code = code


_SIGS = {
    "hg_last_error": (ctypes.c_char_p, []),
    "hg_device_count": (c_int, []),
    "hg_storage_create_cuboid": (c_int, [P(c_double), P(c_double), c_int, c_int, c_int, c_int, P(c_void_p)]),
    "hg_storage_create_tets": (c_int, [c_int, P(c_double), c_int, P(c_int), c_int, P(c_void_p)]),
    "hg_storage_create_cubed_domain": (c_int, [c_int, P(c_int), c_int, c_int, P(c_void_p)]),
    "hg_storage_create_gmsh": (c_int, [c_char_p, c_int, c_int, P(c_void_p)]),
    "hg_storage_write_gmsh": (c_int, [c_void_p, c_char_p]),
    "hg_storage_destroy": (c_int, [c_void_p]),
    "hg_storage_counts": (c_int, [c_void_p, P(c_int)]),
    "hg_storage_set_stream": (c_int, [c_void_p, c_void_p]),
    "hg_storage_synchronize": (c_int, [c_void_p]),
    "hg_storage_set_l2_budget": (c_int, [c_void_p, c_int64]),
    "hg_storage_launch_count": (c_int, [c_void_p, P(ctypes.c_ulonglong)]),
    "hg_storage_set_cell_coefficients": (c_int, [c_void_p, P(c_double), c_int]),
    "hg_primitive_vertices": (c_int, [c_void_p, c_int, c_int, P(c_int), P(c_double), P(c_int)]),
    "hg_primitive_neighbours": (c_int, [c_void_p, c_int, c_int, c_int, P(c_int), c_int, P(c_int)]),
    "hg_primitive_layout": (c_int, [c_void_p, c_int, c_int, c_int, P(c_int64), P(c_int64)]),
    "hg_level_size": (c_int, [c_void_p, c_int, P(c_int64)]),
    "hg_mesh_create_cuboid": (c_int, [P(c_double), P(c_double), c_int, c_int, c_int, c_int, P(c_void_p)]),
    "hg_mesh_create_tets": (c_int, [c_int, P(c_double), c_int, P(c_int), c_int, P(c_void_p)]),
    "hg_mesh_create_cuboid_copies": (c_int, [c_int, c_int, c_int, P(c_void_p)]),
    "hg_mesh_create_cubed_domain": (c_int, [c_int, P(c_int), c_int, c_int, P(c_void_p)]),
    "hg_mesh_create_gmsh": (c_int, [c_char_p, c_int, c_int, P(c_void_p)]),
    "hg_mesh_write_gmsh": (c_int, [c_void_p, c_char_p]),
    "hg_mesh_destroy": (c_int, [c_void_p]),
    "hg_mesh_counts": (c_int, [c_void_p, P(c_int)]),
    "hg_mesh_set_cell_coefficients": (c_int, [c_void_p, P(c_double), c_int]),
    "hg_mesh_primitive_vertices": (c_int, [c_void_p, c_int, c_int, P(c_int), P(c_double), P(c_int)]),
    "hg_mesh_primitive_neighbours": (c_int, [c_void_p, c_int, c_int, c_int, P(c_int), c_int, P(c_int)]),
    "hg_mesh_primitive_layout": (c_int, [c_void_p, c_int, c_int, c_int, P(c_int64), P(c_int64)]),
    "hg_mesh_level_size": (c_int, [c_void_p, c_int, P(c_int64)]),
    "hg_mesh_slot_info": (c_int, [c_void_p, c_int, P(c_double), P(ctypes.c_byte), c_int64]),
    "hg_mesh_owned_slots": (c_int, [c_void_p, c_int, P(c_int64), P(c_int64)]),
    "hg_mesh_halo_table": (c_int, [c_void_p, c_int, c_int, P(c_int64), P(c_int64), P(c_int64)]),
    "hg_split_tables_check": (c_int, [c_int, P(c_int64), P(c_int64)]),
    "hg_mesh_assembly_plan_check": (c_int, [c_void_p, c_int, c_int, P(c_int64), P(c_int64), P(c_int64)]),
    "hg_mesh_cell_stencil": (c_int, [c_void_p, c_int, c_int, c_int, P(c_double)]),
    "hg_mesh_face_stencil": (c_int, [c_void_p, c_int, c_int, c_int, P(c_int), P(c_int), P(c_int), P(c_double), c_int, P(c_int)]),
    "hg_mesh_low_stencil": (c_int, [c_void_p, c_int, c_int, c_int, c_int, P(c_int64), P(c_double), c_int, P(c_int)]),
    "hg_function_create": (c_int, [c_void_p, c_int, c_int, c_int, P(c_int)]),
    "hg_function_destroy": (c_int, [c_void_p, c_int]),
    "hg_storage_set_sor_schedule": (c_int, [c_void_p, c_int]),
    "hg_storage_set_sor_fused_phases": (c_int, [c_void_p, c_int]),
    "hg_storage_set_concurrent_components": (c_int, [c_void_p, c_int]),
    "hg_storage_set_sor_schedule_level": (c_int, [c_void_p, c_int, c_int, c_int]),
    "hg_storage_autotune_sor": (c_int, [c_void_p, c_int, c_int, c_int, c_int, P(c_double), P(c_int)]),
    "hg_function_device_ptr": (c_int, [c_void_p, c_int, c_int, P(c_void_p)]),
    "hg_function_upload": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int64]),
    "hg_function_upload_async": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_void_p]),
    "hg_function_download_async": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_void_p]),
    "hg_owned_count": (c_int, [c_void_p, c_int, P(c_int64)]),
    "hg_function_upload_owned_async": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_void_p]),
    "hg_function_download_owned_async": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_void_p]),
    "hg_function_download": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int64]),
    "hg_communicate": (c_int, [c_void_p, c_int, c_int]),
    "hg_interpolate_const": (c_int, [c_void_p, c_int, c_double, c_int, c_uint]),
    "hg_interpolate_expr": (c_int, [c_void_p, c_int, c_int, c_uint, c_int, P(c_double)]),
    "hg_assign": (c_int, [c_void_p, c_int, c_int, c_uint, c_int, P(c_double), P(c_int)]),
    "hg_add": (c_int, [c_void_p, c_int, c_int, c_uint, c_int, P(c_double), P(c_int)]),
    "hg_copy_cast": (c_int, [c_void_p, c_int, c_int, c_int, c_uint, c_int]),
    "hg_dot": (c_int, [c_void_p, c_int, c_int, c_int, c_uint, P(c_double)]),
    "hg_dot_noalloc": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_uint, c_void_p]),
    "hg_operator_create": (c_int, [c_void_p, c_int, c_int, c_int, P(c_int)]),
    "hg_operator_reassemble": (c_int, [c_void_p, c_int, c_int]),
    "hg_operator_destroy": (c_int, [c_void_p, c_int]),
    "hg_apply": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_uint, c_int]),
    "hg_apply_primitives": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_uint, c_int, c_int, c_int]),
    "hg_residual": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_uint]),
    "hg_smooth_sor": (c_int, [c_void_p, c_int, c_int, c_int, c_double, c_int, c_uint, c_int]),
    "hg_smooth_sor_primitives": (c_int, [c_void_p, c_int, c_int, c_int, c_double, c_int, c_uint, c_int, c_int, c_int]),
    "hg_restrict": (c_int, [c_void_p, c_int, c_int, c_uint]),
    "hg_prolongate": (c_int, [c_void_p, c_int, c_int, c_uint, c_int]),
    "hg_cg_solve": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_double, P(c_int), P(c_double)]),
    "hg_gmg_create": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_double, c_int, c_int, c_double, c_int, P(c_int)]),
    "hg_gmg_destroy": (c_int, [c_void_p, c_int]),
    "hg_gmg_solve": (c_int, [c_void_p, c_int, c_int, c_int, c_int]),
    "hg_p2_operator_create": (c_int, [c_void_p, c_int, c_int, c_int, P(c_int)]),
    "hg_p2_operator_destroy": (c_int, [c_void_p, c_int]),
    "hg_p2_apply": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_uint]),
    "hg_p2_residual": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_uint]),
    "hg_p2_smooth_sor": (c_int, [c_void_p, c_int, c_int, c_int, c_double, c_int, c_uint, c_int]),
    "hg_p2_prolongate": (c_int, [c_void_p, c_int, c_int, c_uint, c_int]),
    "hg_p2_restrict": (c_int, [c_void_p, c_int, c_int, c_uint]),
    "hg_p2_gmg_create": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_double, c_int, c_double, P(c_int)]),
    "hg_p2_gmg_destroy": (c_int, [c_void_p, c_int]),
    "hg_p2_gmg_solve": (c_int, [c_void_p, c_int, c_int, c_int, c_int]),
    "hg_p2_gmg_set_graphs": (c_int, [c_void_p, c_int, c_int]),
    "hg_p2p1_stokes_uzawa_gmg_create": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_double, c_int,
                                                 P(c_int)]),
    "hg_p2p1_stokes_uzawa_gmg_destroy": (c_int, [c_void_p, c_int]),
    "hg_p2p1_stokes_uzawa_smooth": (c_int, [c_void_p, c_int, P(c_int), c_int, P(c_int), c_int, c_int]),
    "hg_p2p1_stokes_uzawa_estimate_omega": (c_int, [c_void_p, c_int, c_int, c_int, ctypes.c_uint64, P(c_double)]),
    "hg_p2p1_stokes_uzawa_gmg_solve": (c_int, [c_void_p, c_int, P(c_int), c_int, P(c_int), c_int, c_int]),
    "hg_p2p1_stokes_uzawa_gmg_solve_to": (c_int, [c_void_p, c_int, P(c_int), c_int, P(c_int), c_int, c_int, c_double,
                                                   c_int, P(c_int), P(c_double), P(c_double), c_int]),
    "hg_p2_gmg_solve_to": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_double, c_int, P(c_int), P(c_double),
                                   P(c_double), c_int]),
    "hg_p2p1_stokes_create": (c_int, [c_void_p, c_int, c_int, P(c_int)]),
    "hg_p2p1_stokes_apply": (c_int, [c_void_p, c_int, P(c_int), c_int, P(c_int), c_int, c_int, c_uint, c_uint]),
    "hg_p2p1_stokes_minres": (c_int, [c_void_p, c_int, P(c_int), c_int, P(c_int), c_int, c_int, c_int, c_int, c_double,
                                      P(c_int), P(c_double), P(c_double), c_int]),
    "hg_p2p1_stokes_minres_mixed": (c_int, [c_void_p, c_int, P(c_int), c_int, P(c_int), c_int, c_int, c_int, c_int,
                                            c_double, c_int, P(c_int), P(c_double), P(c_double), c_int]),
    "hg_server_create": (c_int, [c_int, c_int64, c_int, P(c_void_p)]),
    "hg_server_destroy": (c_int, [c_void_p]),
    "hg_server_prewarm": (c_int, [c_void_p, c_int, c_int]),
    "hg_server_submit": (c_int, [c_void_p, c_int, c_int, c_double, ctypes.c_uint64, c_double, c_int, c_int, P(c_int64)]),
    "hg_server_wait": (c_int, [c_void_p, c_int64, c_double, P(c_int)]),
    "hg_server_result": (c_int, [c_void_p, c_int64, P(c_int), P(c_int), P(c_double), P(c_double), P(c_int64)]),
    "hg_server_request_setup": (c_int, [c_void_p, c_int64, P(c_int)]),
    "hg_server_set_batching": (c_int, [c_void_p, c_int]),
    "hg_server_prewarm_batch": (c_int, [c_void_p, c_int, c_int, c_int]),
    "hg_server_request_batch": (c_int, [c_void_p, c_int64, P(c_int)]),
    "hg_server_solution": (c_int, [c_void_p, c_int64, P(c_double), c_int64, P(c_int64)]),
    "hg_server_stats": (c_int, [c_void_p, P(c_int64)]),
    "hg_function_fill_random": (c_int, [c_void_p, c_int, c_int, c_uint, ctypes.c_uint64, c_double, c_double]),
    "hg_gmg_set_timing": (c_int, [c_void_p, c_int, c_int]),
    "hg_gmg_timing_json": (c_int, [c_void_p, c_int, c_char_p, c_int64, P(c_int64)]),
    "hg_gmg_set_graphs": (c_int, [c_void_p, c_int, c_int]),
    "hg_gmg_set_compact": (c_int, [c_void_p, c_int, c_int, c_int]),
    "hg_gmg_compact_top": (c_int, [c_void_p, c_int, P(c_int)]),
    "hg_gmg_solve_to": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_double, c_int, P(c_int), P(c_double), P(c_double),
                                c_int]),
}


def _declare():
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


_declare()

DECLARED = sorted(_SIGS)


def check(code):
    if code != HG_OK:
        raise HygError(code, lib.hg_last_error().decode())
    return code


def call(name, *args):
    return check(getattr(lib, name)(*args))


def dptr(a):
    return a.ctypes.data_as(P(c_double))


def iptr(a):
    return a.ctypes.data_as(P(c_int))


def i64ptr(a):
    return a.ctypes.data_as(P(c_int64))

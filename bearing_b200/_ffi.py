"""ctypes bindings for the two native libraries of this package.

``libbearing_gpu.so`` is the CUDA solve stage behind the C ABI in ``include/bearing_gpu.h``;
``libbearing_host.so`` is the host side of ``World.step`` in ``include/bearing_world.h``.
Both are built in-tree by ``bearing_b200/build.py``.  The structures below mirror the headers
field for field.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))

BG_POINTS = 4
BG_COLOURS = 32
BG_OVERFLOW = 32
BG_RESTING = 33
BG_STARTS = 35

BG_OK = 0
BG_EINVAL = -1
BG_ECUDA = -2
BG_ETIMEOUT = -3
BG_ENOMEM = -4
BG_EUNSUPPORTED = -5
BG_EFAULT = -6

BG_FLAG_PIN_HOST, BG_FLAG_GRID, BG_FLAG_BLOCK = 1, 2, 4
BG_BATCH_ON_GRID = 1
BG_MAX_BATCH_GROUPS = 8
BG_STATIC_MAX_BODIES, BG_STATIC_MAX_ROWS = 512, 2048

BG_DYNAMIC, BG_STATIC, BG_KINEMATIC = 0, 1, 2
BG_BOX, BG_SPHERE, BG_CAPSULE = 0, 1, 2

_d = C.POINTER(C.c_double)
_u8 = C.POINTER(C.c_uint8)
_i32 = C.POINTER(C.c_int32)


class Bodies(C.Structure):
    """bg_bodies: per-slot columns, as World keeps them (src/world.js:228-311)."""

    _fields_ = [
        ("capacity", C.c_int32),
        ("awake_count", C.c_int32),
        ("awake_list", _i32),
        ("awake", _u8),
        ("position", _d),
        ("rotation", _d),
        ("velocity", _d),
        ("angular", _d),
        ("tumbled", _d),
        ("ceiling", _d),
        ("start", _d),
        ("start_q", _d),
        ("inv_i", _d),
        ("inv_mass", _d),
        ("inertia", _d),
        ("inv_inertia", _d),
        ("dims", _d),
        ("damping", _d),
        ("angular_damping", _d),
        ("gravity_scale", _d),
        ("type", _u8),
        ("shape", _u8),
        ("frozen", _u8),
        ("framed", _u8),
        ("lock", _u8),
        ("joint_head", _i32),
    ]


class Rows(C.Structure):
    """bg_rows: one step's manifolds in colour order (src/contact.js Contacts)."""

    _fields_ = [
        ("count", C.c_int32),
        ("solved", C.c_int32),
        ("starts", C.c_int32 * BG_STARTS),
        ("row", _i32),
        ("a", _i32),
        ("b", _i32),
        ("points", _u8),
        ("normal", _d),
        ("t1", _d),
        ("t2", _d),
        ("friction", _d),
        ("restitution", _d),
        ("tolerance", _d),
        ("patch", _d),
        ("separation", _d),
        ("point", _d),
        ("shift", _d),
        ("normal_impulse", _d),
        ("tangent_impulse1", _d),
        ("tangent_impulse2", _d),
        ("roll_impulse1", _d),
        ("roll_impulse2", _d),
        ("spin_impulse", _d),
        ("drift1", _d),
        ("drift2", _d),
        ("gap", _d),
        ("max_normal_impulse", _d),
        ("relative_velocity", _d),
        ("sliding", _u8),
        ("anchor_a", _d),
        ("anchor_b", _d),
    ]


class Step(C.Structure):
    _fields_ = [("dt", C.c_double), ("substeps", C.c_int32), ("gravity", C.c_double * 3)]


class Worlds(C.Structure):
    _fields_ = [
        ("count", C.c_int32),
        ("body_offset", _i32),
        ("awake_offset", _i32),
        ("row_offset", _i32),
        ("starts", _i32),
        ("gravity", _d),
    ]


class BodyGrads(C.Structure):
    """bg_body_grads: adjoints of the body columns a step reads and writes."""

    _fields_ = [(f, _d) for f in ("position", "rotation", "velocity", "angular", "tumbled", "ceiling")]


class RowGrads(C.Structure):
    """bg_row_grads: adjoints of the row columns a step reads and writes."""

    _fields_ = [(f, _d) for f in ("normal_impulse", "tangent_impulse1", "tangent_impulse2", "roll_impulse1",
                                  "roll_impulse2", "spin_impulse", "drift1", "drift2", "normal", "t1", "t2",
                                  "friction", "restitution", "separation", "point")]


class RowMemory(C.Structure):
    """bw_row_memory: per row, what narrow() used besides the row's columns."""

    _fields_ = [
        ("pid", C.POINTER(C.c_uint32)),
        ("margin", _d),
        ("remembered", _u8),
        ("memory_pid", C.POINTER(C.c_uint32)),
        ("memory", _d),
    ]


BW_MEMORY = 16


class Pairs(C.Structure):
    """bg_pairs: the pairs narrow() hands to collide(), with their margins and tolerances."""

    _fields_ = [("count", C.c_int32), ("a", _i32), ("b", _i32), ("margin", _d), ("tolerance", _d)]


class Manifolds(C.Structure):
    """bg_manifolds: one manifold a pair (points 0..BG_POINTS)."""

    _fields_ = [("points", _u8), ("normal", _d), ("point", _d), ("separation", _d),
                ("pid", C.POINTER(C.c_uint32))]


class Materials(C.Structure):
    """bg_materials: per-slot friction, restitution and size, what emit() reads."""

    _fields_ = [("friction", _d), ("restitution", _d), ("size", _d), ("reach", _d)]


class ContactPairs(C.Structure):
    """bg_contact_pairs: the step's pair list with each pair's contact record (or -1)."""

    _fields_ = [("list", Pairs), ("memory", _i32), ("reuse", C.c_int32)]


class ContactResult(C.Structure):
    """bg_contact_result: per-pair point counts and touching flags, and the step's row counts."""

    _fields_ = [("points", _u8), ("touching", _u8), ("rows", C.c_int32), ("solved", C.c_int32),
                ("points_solved", C.c_int32), ("starts", C.c_int32 * 35)]


class Options(C.Structure):
    _fields_ = [("gravity", C.c_double * 3), ("substeps", C.c_int32), ("reuse", C.c_int32)]


class BodySpec(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("shape", C.c_int32),
        ("size", C.c_double * 3),
        ("radius", C.c_double),
        ("height", C.c_double),
        ("density", C.c_double),
        ("mass", C.c_double),
        ("friction", C.c_double),
        ("restitution", C.c_double),
        ("damping", C.c_double),
        ("angular_damping", C.c_double),
        ("gravity_scale", C.c_double),
        ("position", C.c_double * 3),
        ("rotation", C.c_double * 4),
        ("velocity", C.c_double * 3),
        ("angular", C.c_double * 3),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("bodies", C.c_int32),
        ("awake", C.c_int32),
        ("pairs", C.c_int32),
        ("rows", C.c_int32),
        ("solved", C.c_int32),
        ("points", C.c_int32),
        ("colours", C.c_int32),
        ("overflow", C.c_int32),
        ("step", C.c_int64),
    ]


SOLVER = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.POINTER(Bodies), C.POINTER(Rows), C.POINTER(Step))

_host = None
_gpu = None


def lib_path(name: str) -> str:
    return os.path.join(HERE, name)


def host() -> C.CDLL:
    """libbearing_host.so, loaded once."""
    global _host
    if _host is None:
        path = lib_path("libbearing_host.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run bearing_b200.build.build() first")
        lib = C.CDLL(path)
        lib.bw_create.restype = C.c_void_p
        lib.bw_create.argtypes = [C.POINTER(Options)]
        lib.bw_destroy.argtypes = [C.c_void_p]
        lib.bw_last_error.restype = C.c_char_p
        lib.bw_last_error.argtypes = [C.c_void_p]
        lib.bw_add_body.argtypes = [C.c_void_p, C.POINTER(BodySpec)]
        lib.bw_set_solver.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.bw_step.argtypes = [C.c_void_p, C.c_double]
        lib.bw_begin_step.argtypes = [C.c_void_p, C.c_double]
        lib.bw_end_step.argtypes = [C.c_void_p]
        lib.bw_bodies_view.argtypes = [C.c_void_p, C.POINTER(Bodies)]
        lib.bw_rows_view.argtypes = [C.c_void_p, C.POINTER(Rows)]
        lib.bw_step_params.argtypes = [C.c_void_p, C.POINTER(Step)]
        lib.bw_transforms.restype = C.POINTER(C.c_float)
        lib.bw_transforms.argtypes = [C.c_void_p]
        lib.bw_stats_get.argtypes = [C.c_void_p, C.POINTER(Stats)]
        lib.bw_batch_create.restype = C.c_void_p
        lib.bw_batch_create.argtypes = [C.POINTER(C.c_void_p), C.c_int32]
        lib.bw_batch_destroy.argtypes = [C.c_void_p]
        lib.bw_batch_begin_step.argtypes = [C.c_void_p, C.c_double, C.c_int32]
        lib.bw_batch_views.argtypes = [C.c_void_p, C.POINTER(Bodies), C.POINTER(Rows), C.POINTER(Worlds), C.POINTER(Step)]
        lib.bw_batch_end_step.argtypes = [C.c_void_p, C.c_int32]
        lib.bw_materials.argtypes = [C.c_void_p, _d, _d]
        lib.bw_keep_backward.argtypes = [C.POINTER(Rows), C.POINTER(Worlds), _d, C.POINTER(RowGrads)]
        lib.bw_narrow_backward.argtypes = [C.POINTER(Bodies), C.POINTER(Rows), C.POINTER(Worlds), C.POINTER(RowMemory),
                                           _d, _d, _d, C.POINTER(RowGrads), _d, _d, _d, _d, _d, C.c_int32]
        lib.bw_row_memory_get.argtypes = [C.c_void_p, C.POINTER(RowMemory)]
        lib.bw_batch_row_memory.argtypes = [C.c_void_p, C.POINTER(RowMemory)]
        lib.bw_clone.restype = C.c_void_p
        lib.bw_clone.argtypes = [C.c_void_p]
        lib.bw_copy.argtypes = [C.c_void_p, C.c_void_p]
        lib.bw_narrow_pairs.argtypes = [C.c_void_p, C.POINTER(Pairs)]
        lib.bw_set_narrowphase.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.bw_set_workers.argtypes = [C.c_void_p, C.c_int32]
        lib.bw_set_contact_step.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.bw_colour_rows.argtypes = [C.POINTER(Bodies), C.c_int32, _i32, _i32, _i32, _i32, _i32, _i32]
        lib.bw_collide_pairs.argtypes = [C.POINTER(Bodies), _d, C.POINTER(Pairs), C.POINTER(Manifolds), C.c_int32]
        for f in ("bw_add_body", "bw_set_solver", "bw_step", "bw_begin_step", "bw_end_step",
                  "bw_bodies_view", "bw_rows_view", "bw_step_params", "bw_stats_get", "bw_batch_begin_step",
                  "bw_batch_views", "bw_batch_end_step", "bw_row_memory_get", "bw_batch_row_memory", "bw_copy",
                  "bw_keep_backward", "bw_narrow_backward", "bw_materials", "bw_narrow_pairs", "bw_collide_pairs",
                  "bw_set_narrowphase", "bw_set_workers", "bw_colour_rows", "bw_set_contact_step"):
            getattr(lib, f).restype = C.c_int32
        _host = lib
    return _host


def gpu() -> C.CDLL:
    """libbearing_gpu.so, loaded once.  Raises if it was not built: there is no fallback."""
    global _gpu
    if _gpu is None:
        path = lib_path("libbearing_gpu.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run bearing_b200.build.build() first")
        lib = C.CDLL(path)
        lib.bg_create.restype = C.c_void_p
        lib.bg_create.argtypes = [C.c_int32, C.c_uint32]
        lib.bg_destroy.argtypes = [C.c_void_p]
        lib.bg_last_error.restype = C.c_char_p
        lib.bg_last_error.argtypes = [C.c_void_p]
        lib.bg_version.restype = C.c_uint32
        lib.bg_version.argtypes = []
        three = [C.c_void_p, C.POINTER(Bodies), C.POINTER(Rows)]
        lib.bg_solve_step.argtypes = three + [C.POINTER(Step)]
        lib.bg_upload.argtypes = three
        lib.bg_restore.argtypes = [C.c_void_p]
        lib.bg_solve.argtypes = [C.c_void_p, C.POINTER(Step)]
        lib.bg_download.argtypes = three
        lib.bg_batch_solve_step.argtypes = three + [C.POINTER(Worlds), C.POINTER(Step)]
        lib.bg_batch_upload.argtypes = three + [C.POINTER(Worlds)]
        lib.bg_batch_solve.argtypes = [C.c_void_p, C.POINTER(Step)]
        lib.bg_batch_download.argtypes = three
        lib.bg_stream.restype = C.c_void_p
        lib.bg_stream.argtypes = [C.c_void_p]
        lib.bg_register_host.argtypes = three + [C.c_int32]
        lib.bg_register_host.restype = C.c_int32
        lib.bg_unregister_host.argtypes = [C.c_void_p]
        lib.bg_unregister_host.restype = C.c_int32
        lib.bg_registered_bytes.argtypes = [C.c_void_p]
        lib.bg_registered_bytes.restype = C.c_int64
        lib.bg_backward_bytes.argtypes = [C.c_void_p]
        lib.bg_backward_bytes.restype = C.c_int64
        lib.bg_collide.argtypes = [C.c_void_p, C.POINTER(Bodies), _d, C.POINTER(Pairs), C.POINTER(Manifolds)]
        lib.bg_collide.restype = C.c_int32
        lib.bg_colour.argtypes = [C.c_void_p, C.POINTER(Bodies), C.c_int32, _i32, _i32, _i32, _i32, _i32, _i32]
        lib.bg_colour.restype = C.c_int32
        lib.bg_last_colour_ms.argtypes = [C.c_void_p]
        lib.bg_contact_step.argtypes = [C.c_void_p, C.POINTER(Bodies), C.POINTER(Materials), C.POINTER(ContactPairs),
                                        C.POINTER(Step), C.POINTER(ContactResult)]
        lib.bg_contact_step.restype = C.c_int32
        lib.bg_last_contact_ms.argtypes = [C.c_void_p, _d]
        lib.bg_last_contact_ms.restype = C.c_int32
        lib.bg_contact_records.argtypes = [C.c_void_p]
        lib.bg_contact_records.restype = C.c_int32
        lib.bg_contact_forget.argtypes = [C.c_void_p]
        lib.bg_contact_forget.restype = C.c_int32
        lib.bg_last_colour_ms.restype = C.c_double
        lib.bg_last_collide_ms.argtypes = [C.c_void_p]
        lib.bg_last_collide_ms.restype = C.c_double
        lib.bg_last_launches.argtypes = [C.c_void_p]
        lib.bg_set_wait_budget.argtypes = [C.c_void_p, C.c_int64]
        lib.bg_last_stage_ms.argtypes = [C.c_void_p]
        lib.bg_last_stage_ms.restype = C.c_double
        lib.bg_set_block_threads.argtypes = [C.c_void_p, C.c_int32]
        lib.bg_set_block_threads.restype = C.c_int32
        lib.bg_block_threads.argtypes = [C.c_void_p]
        lib.bg_block_threads.restype = C.c_int32
        lib.bg_set_batch_groups.argtypes = [C.c_void_p, C.c_int32]
        lib.bg_set_batch_groups.restype = C.c_int32
        lib.bg_backward.argtypes = three + [C.POINTER(Worlds), C.POINTER(Step), C.POINTER(BodyGrads), C.POINTER(RowGrads),
                                            C.POINTER(BodyGrads), C.POINTER(RowGrads)]
        lib.bg_backward.restype = C.c_int32
        lib.bg_backward_tape_peak.argtypes = [C.c_void_p]
        lib.bg_backward_tape_peak.restype = C.c_int32
        lib.bg_backward_ms.argtypes = [C.c_void_p]
        lib.bg_backward_ms.restype = C.c_double
        lib.bg_solve_step_static.argtypes = [C.POINTER(Bodies), C.POINTER(Rows), C.POINTER(Step), C.c_void_p]
        lib.bg_solve_step_static.restype = C.c_int32
        for f in ("bg_solve_step", "bg_upload", "bg_restore", "bg_solve", "bg_download",
                  "bg_batch_solve_step", "bg_batch_upload", "bg_batch_solve", "bg_batch_download",
                  "bg_last_launches", "bg_set_wait_budget"):
            getattr(lib, f).restype = C.c_int32
        _gpu = lib
    return _gpu


# Every symbol each header declares, for the export checks.
GPU_SYMBOLS = [
    "bg_create", "bg_destroy", "bg_last_error", "bg_version", "bg_solve_step", "bg_upload", "bg_restore",
    "bg_solve", "bg_download", "bg_batch_solve_step", "bg_batch_upload", "bg_batch_solve",
    "bg_batch_download", "bg_stream", "bg_last_launches", "bg_last_stage_ms", "bg_set_wait_budget", "bg_set_block_threads",
    "bg_block_threads", "bg_set_batch_groups", "bg_backward", "bg_backward_tape_peak", "bg_backward_ms",
    "bg_solve_step_static", "bg_register_host", "bg_unregister_host", "bg_registered_bytes", "bg_collide",
    "bg_last_collide_ms", "bg_backward_bytes", "bg_colour", "bg_last_colour_ms", "bg_contact_step",
    "bg_last_contact_ms", "bg_contact_records", "bg_contact_forget",
]
HOST_SYMBOLS = [
    "bw_create", "bw_destroy", "bw_last_error", "bw_add_body", "bw_set_solver", "bw_step", "bw_begin_step",
    "bw_end_step", "bw_bodies_view", "bw_rows_view", "bw_step_params", "bw_transforms", "bw_stats_get",
    "bw_batch_create", "bw_batch_destroy", "bw_batch_begin_step", "bw_batch_views", "bw_batch_end_step",
    "bw_row_memory_get", "bw_batch_row_memory", "bw_clone", "bw_copy", "bw_keep_backward", "bw_narrow_backward",
    "bw_materials", "bw_narrow_pairs", "bw_collide_pairs", "bw_set_narrowphase", "bw_set_workers", "bw_colour_rows",
    "bw_set_contact_step",
]

"""ctypes binding of the C ABI declared in include/dfem.h (libdfem.so, in-tree).

The library must be built (``python -m diff_fem_b200.build``); there is no CPU
fallback: every call goes to the CUDA engine, and loading fails loudly when
the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdfem.so")

DFEM_OK = 0
DFEM_ERR_INVALID = 1
DFEM_ERR_CUDA = 2
DFEM_ERR_FACTOR = 3
DFEM_ERR_NONFINITE = 4
DFEM_ERR_STATE = 5
DFEM_ERR_CAP = 6
DFEM_ERR_NOMEM = 7
DFEM_ERR_UNSUPPORTED = 8
DFEM_JOINT_PRISMATIC, DFEM_JOINT_ROTATIONAL, DFEM_JOINT_ALL = 0, 1, 2
DFEM_MEM_HOST = 0
DFEM_MEM_DEVICE = 1
DFEM_PREC_FP64 = 0
DFEM_PREC_MIXED = 1

STATUS_NAMES = {
    0: "DFEM_OK", 1: "DFEM_ERR_INVALID", 2: "DFEM_ERR_CUDA", 3: "DFEM_ERR_FACTOR",
    4: "DFEM_ERR_NONFINITE", 5: "DFEM_ERR_STATE", 6: "DFEM_ERR_CAP", 7: "DFEM_ERR_NOMEM",
    8: "DFEM_ERR_UNSUPPORTED",
}

_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int32)
_pu8 = C.POINTER(C.c_uint8)


class SceneDescC(C.Structure):
    """Mirror of ``dfem_scene_desc`` (field order and types must match dfem.h)."""
    _fields_ = [
        ("n_vertices", C.c_int32), ("x0", _pd), ("mass", _pd), ("gravity_mask", _pu8),
        ("n_tets", C.c_int32), ("tets", _pi), ("youngs", _pd), ("poisson", _pd),
        ("n_attach", C.c_int32), ("attach_vertex", _pi), ("attach_target", _pd), ("attach_stiffness", _pd),
        ("n_muscle", C.c_int32), ("muscle_tets", _pi), ("muscle_fiber", _pd), ("muscle_stiffness", _pd),
        ("muscle_segment", _pi), ("n_segments", C.c_int32),
        ("n_springs", C.c_int32), ("spring_vertices", _pi), ("spring_rest", _pd), ("spring_weight", _pd),
        ("spring_channel", _pi),
        ("n_bending", C.c_int32), ("bend_offsets", _pi), ("bend_vertices", _pi), ("bend_weight", _pd),
        ("n_contact_vertices", C.c_int32), ("contact_vertices", _pi),
        ("n_contact_faces", C.c_int32), ("contact_faces", _pi),
        ("n_obstacle_vertices", C.c_int32), ("obstacle_x", _pd),
        ("n_obstacle_faces", C.c_int32), ("obstacle_faces", _pi),
        ("time_step", C.c_double), ("max_iterations", C.c_int32), ("damping", C.c_double),
        ("gravity", C.c_double * 3),
        ("handle_collision", C.c_int32), ("self_collision", C.c_int32),
        ("alpha", C.c_double), ("friction", C.c_double), ("obstacle_friction", C.c_double),
        ("precision", C.c_int32), ("checkpoint_every", C.c_int32),
        ("underwater", C.c_int32), ("n_drag_faces", C.c_int32), ("drag_faces", _pi),
        ("n_links", C.c_int32), ("link_parent", _pi), ("link_type", _pi), ("link_joint", _pd),
        ("link_axis", _pd), ("link_offsets", _pi), ("link_vertices", _pi), ("link_channel", _pi),
    ]


class SceneInfoC(C.Structure):
    _fields_ = [
        ("n_vertices", C.c_int32), ("n_tets", C.c_int32), ("n_attach", C.c_int32), ("n_muscle", C.c_int32),
        ("n_springs", C.c_int32), ("n_bending", C.c_int32),
        ("n_supernodes", C.c_int32), ("n_levels", C.c_int32),
        ("nnz_factor", C.c_int64), ("n_slots", C.c_int32), ("device", C.c_int32),
        ("factor_regularisation", C.c_double),
    ]


# (name, restype, argtypes)
_VP = C.c_void_p
SIGNATURES = [
    ("dfem_scene_create", C.c_int, [C.POINTER(SceneDescC), C.c_int, C.POINTER(_VP)]),
    ("dfem_scene_create_batch", C.c_int, [C.POINTER(SceneDescC), C.c_int32, C.c_int, C.POINTER(_VP)]),
    ("dfem_batch_layout", C.c_int, [_VP, _pi, _pi, _pi, _pi]),
    ("dfem_scene_destroy", C.c_int, [_VP]),
    ("dfem_scene_get_info", C.c_int, [_VP, C.POINTER(SceneInfoC)]),
    ("dfem_set_materials", C.c_int, [_VP, _VP, _VP, C.c_int]),
    ("dfem_set_activations", C.c_int, [_VP, _VP, C.c_int]),
    ("dfem_set_joint_state", C.c_int, [_VP, _pd, _pd]),
    ("dfem_get_joint_state", C.c_int, [_VP, _pd, _pd]),
    ("dfem_set_joint_state_grad", C.c_int, [_VP, _pd, _pd]),
    ("dfem_get_joint_state_grad", C.c_int, [_VP, _pd, _pd]),
    ("dfem_step_forward", C.c_int, [_VP, _VP, _VP, _VP, C.c_int32, _VP, _VP, _VP, C.c_int]),
    ("dfem_step_backward", C.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, C.c_int]),
    ("dfem_eval_local", C.c_int, [_VP, _VP, _VP, C.c_int]),
    ("dfem_eval_corotated_noalloc", C.c_int,
     [C.c_int32, C.c_int32, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    ("dfem_get_iterations", C.c_int, [_VP, _pi, C.c_int32]),
    ("dfem_get_contact_passes", C.c_int, [_VP, _pi, C.c_int32]),
    ("dfem_host_factor_solve", C.c_int, [C.POINTER(SceneDescC), _VP, _VP, C.POINTER(SceneInfoC)]),
    ("dfem_solve_mode", C.c_int, [_VP, C.c_int32, _pi, C.POINTER(C.c_double)]),
    ("dfem_solve_split", C.c_int, [_VP, _pi, _pi, C.POINTER(C.c_double)]),
    ("dfem_solve_times", C.c_int, [_VP, C.POINTER(C.c_double), C.c_int32]),
    ("dfem_solve_select", C.c_int, [_VP, _pi, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("dfem_profile_levels", C.c_int, [_VP, C.c_int32, C.c_int32, _pi, C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), _pi, _pi, _pi]),
    ("dfem_set_adjoint_budget", C.c_int, [_VP, C.c_int64]),
    ("dfem_get_launch_count", C.c_int, [_VP, C.POINTER(C.c_int64)]),
    ("dfem_profile_phases", C.c_int, [_VP, C.c_int32, C.POINTER(C.c_double)]),
    ("dfem_synchronize", C.c_int, [_VP]),
    ("dfem_obj_writer_create", C.c_int, [C.c_int32, _pi, _pi, _pi, C.POINTER(C.c_char_p), C.c_int32, C.POINTER(_VP)]),
    ("dfem_obj_writer_enqueue", C.c_int, [_VP, _VP, C.c_char_p, _VP, C.c_int]),
    ("dfem_obj_writer_flush", C.c_int, [_VP]),
    ("dfem_obj_writer_destroy", C.c_int, [_VP]),
    ("dfem_last_error", C.c_char_p, []),
    ("dfem_abi_version", C.c_int, []),
    ("dfem_set_limit", C.c_int, [_VP, C.c_int32, C.c_int64]),
    ("dfem_set_option", C.c_int, [_VP, C.c_int32, C.c_int64]),
    ("dfem_debug_fail_allocations", C.c_int, [C.c_int64]),
]

_lib = None


class DfemError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib() -> C.CDLL:
    """Load libdfem.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m diff_fem_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != DFEM_OK:
        raise DfemError(rc, lib().dfem_last_error().decode(errors="replace"))

"""ctypes binding of libfvedg_b200.so (include/dg_gpu.h). Loading fails loudly if the library
is missing: there is no CPU fallback for any entry point."""
import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libfvedg_b200.so")

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int64_p = ctypes.POINTER(ctypes.c_int64)
c_uint8_p = ctypes.POINTER(ctypes.c_uint8)
c_int8_p = ctypes.POINTER(ctypes.c_int8)
c_int_p = ctypes.POINTER(ctypes.c_int)

DG_OK = 0
DG_E_ARG = -1
DG_E_WATCHDOG = -6
STATUS = {0: "DG_OK", -1: "DG_E_ARG", -2: "DG_E_MESH", -3: "DG_E_CUDA", -4: "DG_E_NOMEM",
          -5: "DG_E_NONPHYSICAL", -6: "DG_E_WATCHDOG", -7: "DG_E_STATE", -8: "DG_E_IO"}


class DGError(RuntimeError):
    def __init__(self, code, what):
        self.code = code
        msg = f"{what}: {STATUS.get(code, code)}"
        if code == -3 and _lib is not None:  # DG_E_CUDA: name the CUDA error behind it
            msg += f" ({_lib.dg_last_cuda_error().decode()})"
        super().__init__(msg)


class MeshDesc(ctypes.Structure):
    _fields_ = [
        ("ncell", ctypes.c_int64), ("nface", ctypes.c_int64),
        ("face_cells", c_int64_p), ("face_bc", c_uint8_p),
        ("face_natural", c_double_p), ("face_normal", c_double_p), ("face_area", c_double_p),
        ("cell_invjac", c_double_p), ("cell_detj", c_double_p),
        ("npts", ctypes.c_int64), ("points", c_double_p), ("cell_nodes", c_int64_p),
        ("face_nodes", c_int64_p), ("face_nodes1", c_int64_p), ("face_periodic", c_uint8_p),
        ("nghost", ctypes.c_int64),
    ]


class Config(ctypes.Structure):
    _fields_ = [("order", ctypes.c_int), ("flux", ctypes.c_int), ("quad_vol", ctypes.c_int),
                ("quad_face", ctypes.c_int), ("gamma", ctypes.c_double), ("precision", ctypes.c_int),
                ("device", ctypes.c_int), ("schedule", ctypes.c_int), ("limiter", ctypes.c_int),
                ("mu", ctypes.c_double), ("prandtl", ctypes.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built; run __graft_entry__.build() or python fve_dg_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    sig = {
        "dg_create": (vp, [ctypes.POINTER(MeshDesc), ctypes.POINTER(Config), c_int_p]),
        "dg_destroy": (None, [vp]),
        "dg_residual": (ctypes.c_int, [vp, c_double_p, c_double_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_int]),
        "dg_residual_device": (ctypes.c_int, [vp, vp, vp, ctypes.c_double, ctypes.c_int, vp]),
        "dg_residual_device_static": (ctypes.c_int, [vp, vp, vp, ctypes.c_int, vp]),
        "dg_watchdog_selftest": (ctypes.c_int, [vp, ctypes.c_int64]),
        "dg_last_cuda_error": (ctypes.c_char_p, []),
        "dg_static_scratch_capacity": (ctypes.c_int64, []),
        "dg_set_state": (ctypes.c_int, [vp, c_double_p, ctypes.c_size_t]),
        "dg_get_state": (ctypes.c_int, [vp, c_double_p, ctypes.c_size_t]),
        "dg_ssprk3": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int]),
        "dg_ssprk3_graph": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int]),
        "dg_mass": (ctypes.c_int, [vp, c_double_p, ctypes.c_size_t]),
        "dg_limit": (ctypes.c_int, [vp, c_double_p, c_double_p, ctypes.c_size_t, ctypes.c_int]),
        "dg_viscous_residual": (ctypes.c_int, [vp, c_double_p, c_double_p, ctypes.c_size_t, ctypes.c_double,
                                               ctypes.c_double]),
        "dg_viscous_residual_device": (ctypes.c_int, [vp, vp, vp, ctypes.c_double, ctypes.c_double, vp]),
        "dg_limit_device": (ctypes.c_int, [vp, vp, vp, ctypes.c_int, vp]),
        "dg_save_checkpoint": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_double, ctypes.c_int64]),
        "dg_load_checkpoint": (ctypes.c_int, [vp, ctypes.c_char_p, c_double_p, c_int64_p]),
        "dg_ssprk3_timed": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int, c_double_p, ctypes.c_int]),
        "dg_stream": (vp, [vp]),
        "dg_state_device": (vp, [vp, ctypes.c_int]),
        "dg_refresh_split": (ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_int64, vp]),
        "dg_ssprk3_stage": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int]),
        "dg_ssprk3_stage_phase": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int, ctypes.c_int]),
        "dg_create_ensemble": (vp, [ctypes.POINTER(MeshDesc), ctypes.c_int, ctypes.POINTER(Config), c_int_p]),
        "dg_ensemble_offsets": (ctypes.c_int, [vp, c_int64_p]),
        "dg_ssprk3_ensemble": (ctypes.c_int, [vp, c_double_p, ctypes.c_int, ctypes.c_int]),
        "dg_autotune": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_char_p, ctypes.c_size_t]),
        "dg_set_element_shape": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
        "dg_partition_create": (vp, [ctypes.POINTER(MeshDesc), ctypes.POINTER(ctypes.c_int32), ctypes.c_int, c_int_p]),
        "dg_partition_destroy": (None, [vp]),
        "dg_partition_local_mesh": (ctypes.c_int, [vp, ctypes.POINTER(MeshDesc)]),
        "dg_partition_counts": (ctypes.c_int, [vp, c_int64_p, c_int64_p, c_int_p, c_int_p]),
        "dg_partition_l2g": (c_int64_p, [vp]),
        "dg_partition_global_faces": (c_int64_p, [vp]),
        "dg_partition_send": (ctypes.c_int, [vp, ctypes.c_int, c_int_p, c_int64_p, ctypes.POINTER(c_int64_p)]),
        "dg_partition_recv": (ctypes.c_int, [vp, ctypes.c_int, c_int_p, c_int64_p, ctypes.POINTER(c_int64_p)]),
        "dg_halo_pack": (ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_int64, vp, vp]),
        "dg_halo_unpack": (ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_int64, vp, vp]),
        "dg_set_dirichlet": (ctypes.c_int, [vp, c_double_p]),
        "dg_conservation": (ctypes.c_int, [vp, c_double_p]),
        "dg_max_wave_speed": (ctypes.c_int, [vp, c_double_p]),
        "dg_check_state": (ctypes.c_int, [vp, c_int64_p]),
        "dg_info": (ctypes.c_int, [vp, c_int_p, c_int_p, c_int_p, c_int_p, c_int_p]),
        "dg_mesh_geometry": (ctypes.c_int, [ctypes.POINTER(MeshDesc), c_double_p, c_double_p, c_double_p,
                                            c_double_p, c_double_p, c_double_p]),
        "dg_face_perms": (ctypes.c_int, [ctypes.POINTER(MeshDesc), c_int8_p]),
        "dg_basis": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, c_double_p, c_double_p, c_double_p]),
        "dg_quad_rule": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, c_double_p, c_double_p]),
        "dg_auto_rules": (ctypes.c_int, [ctypes.c_int, c_int_p, c_int_p]),
        "dg_status_string": (ctypes.c_char_p, [ctypes.c_int]),
        "dg_launch_count": (ctypes.c_int64, []),
        "dg_box_mesh_create": (vp, [ctypes.c_int, c_double_p, c_double_p, ctypes.c_double, ctypes.c_uint64,
                                    c_int_p, ctypes.c_int, c_int_p]),
        "dg_box_mesh_destroy": (None, [vp]),
        "dg_box_mesh_view": (ctypes.c_int, [vp, ctypes.POINTER(MeshDesc), ctypes.POINTER(c_int64_p),
                                            ctypes.POINTER(c_int64_p)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def exported_symbols():
    """Names this binding expects the library to export."""
    return ["dg_create", "dg_destroy", "dg_residual", "dg_residual_device", "dg_residual_device_static",
            "dg_static_scratch_capacity", "dg_set_state", "dg_get_state",
            "dg_ssprk3", "dg_ssprk3_graph", "dg_ssprk3_timed", "dg_stream", "dg_state_device",
            "dg_refresh_split", "dg_ssprk3_stage", "dg_ssprk3_stage_phase", "dg_create_ensemble",
            "dg_ensemble_offsets", "dg_ssprk3_ensemble", "dg_autotune", "dg_set_element_shape", "dg_partition_create", "dg_partition_destroy",
            "dg_partition_local_mesh", "dg_partition_counts", "dg_partition_l2g", "dg_partition_global_faces",
            "dg_partition_send", "dg_partition_recv", "dg_halo_pack", "dg_halo_unpack", "dg_watchdog_selftest", "dg_mass", "dg_limit", "dg_limit_device", "dg_viscous_residual", "dg_viscous_residual_device",
            "dg_save_checkpoint", "dg_load_checkpoint",
            "dg_set_dirichlet", "dg_conservation",
            "dg_max_wave_speed", "dg_check_state", "dg_info", "dg_mesh_geometry", "dg_face_perms", "dg_basis",
            "dg_quad_rule", "dg_auto_rules", "dg_status_string", "dg_last_cuda_error", "dg_launch_count", "dg_box_mesh_create",
            "dg_box_mesh_destroy", "dg_box_mesh_view"]


def check(rc, what):
    if rc != DG_OK:
        raise DGError(rc, what)


def dptr(a):
    return a.ctypes.data_as(c_double_p) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(c_int64_p) if a is not None else None


def u8ptr(a):
    return a.ctypes.data_as(c_uint8_p) if a is not None else None


def as_f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def as_i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def as_u8(a):
    return np.ascontiguousarray(a, dtype=np.uint8)

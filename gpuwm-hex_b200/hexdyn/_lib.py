"""ctypes binding of ``libhexdyn.so`` (declarations: include/hexdyn.h).

Loading fails loudly: there is no CPU fallback for the dycore step.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

LIBRARY = Path(__file__).resolve().parent / "libhexdyn.so"

HEXDYN_ABI_VERSION = 5
HEXDYN_OK = 0
HEXDYN_E_ARG = -1
HEXDYN_E_STATE = -2
HEXDYN_E_NUMERIC = -3
HEXDYN_E_CAPACITY = -4

FIELDS = {
    "rho": 0, "rho_theta": 1, "rho_u": 2, "rho_w": 3, "scalars": 4,
    "theta_m": 5, "exner": 6, "density_perturbation": 7, "rho_theta_perturbation": 8,
    "pressure_perturbation": 9, "normal_velocity": 10, "vertical_velocity": 11,
}
HEXDYN_NUM_FIELDS = len(FIELDS)
STATE_FIELDS = ("rho", "rho_theta", "rho_u", "rho_w", "scalars")
SIDECAR_FIELDS = ("theta_m", "exner", "density_perturbation", "rho_theta_perturbation",
                  "pressure_perturbation", "normal_velocity", "vertical_velocity")

_I32P = C.POINTER(C.c_int32)
_F32P = C.POINTER(C.c_float)


class HexDynFields(C.Structure):
    """Device pointers of one state + sidecar, indexed by FIELDS values."""

    _fields_ = [("field", C.c_void_p * 12)]


class HexDynDesc(C.Structure):
    _fields_ = [
        ("n_cells", C.c_int32), ("n_edges", C.c_int32), ("n_vertices", C.c_int32), ("n_levels", C.c_int32),
        ("max_edges", C.c_int32), ("max_edges2", C.c_int32), ("adv_width", C.c_int32), ("n_scalars", C.c_int32),
        ("cells_on_edge", _I32P), ("edges_on_cell", _I32P), ("cells_on_cell", _I32P),
        ("vertices_on_cell", _I32P), ("n_edges_on_cell", _I32P), ("vertices_on_edge", _I32P),
        ("edges_on_vertex", _I32P), ("cells_on_vertex", _I32P), ("edges_on_edge", _I32P),
        ("n_edges_on_edge", _I32P), ("adv_cells", _I32P), ("n_adv_cells", _I32P),
        ("dc_edge", _F32P), ("dv_edge", _F32P), ("area_cell", _F32P), ("area_triangle", _F32P),
        ("kite_areas", _F32P), ("weights_on_edge", _F32P), ("f_vertex", _F32P), ("f_edge", _F32P),
        ("cos_angle_edge", _F32P), ("sin_angle_edge", _F32P), ("adv_coefs", _F32P), ("adv_coefs_3rd", _F32P),
        ("fzm", _F32P), ("fzp", _F32P), ("rdzw", _F32P), ("rdzu", _F32P),
        ("zz", _F32P), ("zxu", _F32P), ("dss", _F32P), ("zb_cell", _F32P), ("zb3_cell", _F32P),
        ("rho_base", _F32P), ("rho_theta_base", _F32P), ("exner_base", _F32P),
        ("u_init", _F32P), ("v_init", _F32P),
        ("cf1", C.c_float), ("cf2", C.c_float), ("cf3", C.c_float), ("nominal_min_dc", C.c_float),
        ("dt", C.c_double), ("n_sub_steps", C.c_int32), ("split_steps", C.c_int32),
        ("monotonic", C.c_int32), ("moist", C.c_int32), ("numerics", C.c_int32),
        ("coef_3rd_order", C.c_float), ("apvm_upwinding", C.c_float), ("smdiv", C.c_float), ("len_disp", C.c_float),
        ("epssm_minimum", C.c_float), ("epssm_maximum", C.c_float), ("epssm_bottom_z", C.c_float),
        ("epssm_top_z", C.c_float),
        ("rgas", C.c_float), ("cp", C.c_float), ("gravity", C.c_float), ("p0", C.c_float),
        ("acoustic_dts2", C.c_float * 3), ("time_integration_order", C.c_int32),
        ("horiz_mixing", C.c_int32), ("deform_c2", _F32P), ("deform_s2", _F32P), ("deform_cs", _F32P),
        ("mix_del2", _F32P), ("mix_del4", _F32P), ("smag_strain_scale", C.c_float), ("smag_ceiling", C.c_float),
        ("smag_h4", C.c_float), ("smag_div_factor", C.c_float),
        ("rayleigh_levels", C.c_int32), ("rayleigh_inverse", C.c_float), ("cam_levels", C.c_int32),
        ("cam_base", C.c_float), ("clamp_negative_scalars", C.c_int32),
    ]


# Physics stage hook (hexdyn_set_stage_hook): (user, dynamics_substep, rk_step, current fields) -> bit set
STAGE_HOOK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(HexDynFields))
PHYS_RHO_U, PHYS_RHO_THETA, PHYS_RHO, PHYS_DIABATIC_THETA, PHYS_MODIFIED_RATE = 1, 2, 4, 8, 16
# Halo exchange hook (hexdyn_set_exchange_hook): (user, point, nbufs, device buffers, kinds) -> 0 / negative
EXCHANGE_HOOK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_int))
XCH_STATE, XCH_DIAG, XCH_ACOUSTIC, XCH_SCALARS, XCH_FCT = 1, 2, 3, 4, 5
KIND_CELL, KIND_EDGE, KIND_TRACER = 0, 1, 2


class HexDynBatch(C.Structure):
    """Groups of an uneven batch and their step counts (hexdyn_step_batched)."""

    _fields_ = [("n_groups", C.c_int32), ("groups", C.POINTER(C.c_void_p)),
                ("steps", C.POINTER(C.c_int32)), ("flags", C.POINTER(C.c_int32))]


EXPORTS = {
    "hexdyn_abi_version": (C.c_int, []),
    "hexdyn_create": (C.c_int, [C.POINTER(HexDynDesc), C.POINTER(C.c_void_p)]),
    "hexdyn_set_state": (C.c_int, [C.c_void_p, C.c_int, _F32P, C.c_size_t, C.c_void_p]),
    "hexdyn_rebuild_sidecar": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hexdyn_get_state": (C.c_int, [C.c_void_p, C.c_int, _F32P, C.c_size_t, C.c_void_p]),
    "hexdyn_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "hexdyn_step_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "hexdyn_step_host": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_void_p]),
    "hexdyn_read_flag": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    "hexdyn_capture_graph": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hexdyn_profile_steps": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_char_p, C.c_size_t]),
    "hexdyn_device_field": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "hexdyn_acoustic_field": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "hexdyn_level_stride": (C.c_int, [C.c_void_p]),
    "hexdyn_launches_per_step": (C.c_longlong, [C.c_void_p]),
    "hexdyn_device_bytes": (C.c_size_t, [C.c_void_p]),
    "hexdyn_step_noalloc": (C.c_int, [C.c_void_p, C.POINTER(HexDynFields), C.POINTER(HexDynFields),
                                      C.c_void_p, C.POINTER(C.c_int)]),
    "hexdyn_create_ensemble": (C.c_int, [C.POINTER(HexDynDesc), C.c_int, C.POINTER(C.c_void_p)]),
    "hexdyn_member_count": (C.c_int, [C.c_void_p]),
    "hexdyn_set_member_state": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _F32P, C.c_size_t, C.c_void_p]),
    "hexdyn_get_member_state": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _F32P, C.c_size_t, C.c_void_p]),
    "hexdyn_step_batched": (C.c_int, [C.POINTER(HexDynBatch), C.c_void_p]),
    "hexdyn_column_features": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "hexdyn_edge_features": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "hexdyn_apply_increments": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hexdyn_total_energy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hexdyn_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_char_p, C.c_size_t]),
    "hexdyn_bind_state": (C.c_int, [C.c_void_p, C.POINTER(HexDynFields), C.c_void_p]),
    "hexdyn_set_stage_hook": (C.c_int, [C.c_void_p, STAGE_HOOK, C.c_void_p]),
    "hexdyn_physics_buffer": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "hexdyn_set_exchange_hook": (C.c_int, [C.c_void_p, EXCHANGE_HOOK, C.c_void_p]),
    "hexdyn_halo_words": (C.c_size_t, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_int, C.c_int]),
    "hexdyn_halo_pack": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_int), C.c_void_p,
                                   C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "hexdyn_halo_unpack": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_int), C.c_void_p,
                                     C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "hexdyn_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    "hexdyn_destroy": (C.c_int, [C.c_void_p]),
}

_lib: C.CDLL | None = None


class HexDynError(RuntimeError):
    """A refused call or a CUDA error reported by the C ABI."""

    def __init__(self, code: int, message: str):
        self.code = code
        super().__init__(f"hexdyn error {code}: {message}")


def load(path: str | Path | None = None) -> C.CDLL:
    """Load the library (no fallback: a missing library is an error)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    lib_path = Path(path) if path is not None else LIBRARY
    if not lib_path.exists():
        raise ImportError(f"hexdyn CUDA library not found at {lib_path}; build it with "
                          "hexdyn._build.build_library() (nvcc, sm_100a)")
    lib = C.CDLL(str(lib_path))
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.hexdyn_abi_version() != HEXDYN_ABI_VERSION:
        raise ImportError("hexdyn ABI version mismatch")
    if path is None:
        _lib = lib
    return lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().hexdyn_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != HEXDYN_OK:
        raise HexDynError(rc, last_error())

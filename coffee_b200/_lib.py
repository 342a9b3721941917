"""ctypes binding of libcoffee_b200.so (the C ABI in include/coffee_b200.h).

The library is the product: this module only loads it and declares its
signatures.  There is no fallback: if the shared library is missing or has no
CUDA device to run on, calls fail with ``CoffeeError``.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcoffee_b200.so")

COFFEE_OK = 0
COFFEE_E_TIMEOUT = -6
ERRORS = {
    -1: "COFFEE_E_INVALID", -2: "COFFEE_E_CONFIG", -3: "COFFEE_E_CUDA", -4: "COFFEE_E_NOMEM",
    -5: "COFFEE_E_NONFINITE", -6: "COFFEE_E_TIMEOUT", -7: "COFFEE_E_IO",
}

FIELD_IDS = {"Ex": 0, "Ey": 1, "Ez": 2, "Bx": 3, "By": 4, "Bz": 5, "P": 6,
             "Jx": 7, "Jy": 8, "Jz": 9, "divE": 10, "divB": 11,
             "B0x": 12, "B0y": 13, "B0z": 14,
             "dU_EgtB": 15, "dU_Epar": 16, "dU_KO": 17,
             "dU_EgtB_cum": 18, "dU_Epar_cum": 19, "dU_KO_cum": 20}
ENERGY_DIAG_NAMES = ("dU_EgtB", "dU_Epar", "dU_KO", "dU_EgtB_cum", "dU_Epar_cum", "dU_KO_cum")
VARIANT_FLAT = 0
VARIANT_LOGSPH = 1
VARIANT_CYL = 2
VARIANT_GR = 3
VARIANT_YEE = 4
VARIANT_GRYEE = 5
KERNEL_STAGE_FIRST, KERNEL_STAGE, KERNEL_KO = 0, 1, 2
SEM_CPU_REF = 0
SEM_GPU_REF = 1
DIAG = {"energy_E": 0, "energy_B": 1, "divB_l2": 2, "max_edotb": 3, "max_e_over_b": 4}


class CoffeeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_d = ctypes.c_double
_i = ctypes.c_int


class CoffeeParams(ctypes.Structure):
    """Mirror of ``coffee_params`` (same order as Coffee::sim_params)."""

    _fields_ = [
        ("dt", _d), ("max_steps", ctypes.c_uint64), ("data_interval", _i),
        ("snapshot_interval", _i), ("periodic_boundary", _i * 3), ("downsample", _i),
        ("slice_x", _i), ("slice_x_pos", _d), ("slice_y", _i), ("slice_y_pos", _d),
        ("slice_z", _i), ("slice_z_pos", _d), ("slice_xy", _i), ("slice_interval", _i),
        ("downsample_2d", _i), ("N", _i * 3), ("guard", _i * 3), ("lower", _d * 3),
        ("size", _d * 3), ("nodes", _i * 3), ("shift_ghost", _i), ("kn", _i * 3), ("a", _d),
        ("calc_current", _i), ("clean_ep", _i), ("check_egb", _i), ("pml", _i * 3),
        ("pmllen", _i), ("sigpml", _d), ("divB_clean", _i), ("ch2", _d), ("tau", _d),
        ("KOeps", _d), ("KO_geometry", _i), ("use_edotb_damping", _i), ("damp_gamma", _d),
        ("problem", _i), ("radius", _d), ("omega", _d), ("b0", _d),
        ("p1", _d), ("p2", _d), ("p3", _d), ("q11", _d), ("q12", _d), ("q13", _d),
        ("q22", _d), ("q23", _d), ("q_offset_x", _d), ("q_offset_y", _d), ("q_offset_z", _d),
        ("tp_start", _d), ("tp_end", _d), ("rpert1", _d), ("rpert2", _d), ("thp1", _d),
        ("thp2", _d), ("dw0", _d), ("nT", _d), ("shear", _d), ("ph1", _d), ("ph2", _d),
        ("dph", _d), ("theta0", _d), ("drpert", _d),
        ("tp_start1", _d), ("tp_end1", _d), ("rpert11", _d), ("rpert21", _d), ("thp11", _d),
        ("thp21", _d), ("dw1", _d), ("nT1", _d), ("shear1", _d), ("ph11", _d), ("ph21", _d),
        ("dph1", _d), ("pert_type", _i), ("skymap_Nth", _i), ("skymap_Nph", _i),
    ]


class CoffeeGrid(ctypes.Structure):
    _fields_ = [("dims", _i * 3), ("guard", _i * 3), ("delta", _d * 3), ("inv_delta", _d * 3),
                ("lower", _d * 3), ("sizes", _d * 3), ("offset", _i * 3)]


_vp = ctypes.c_void_p
_pp = ctypes.POINTER(ctypes.c_void_p)
_P = ctypes.POINTER

# name -> (restype, argtypes)
SIGNATURES = {
    "coffee_last_error_string": (ctypes.c_char_p, []),
    "coffee_version": (ctypes.c_char_p, []),
    "coffee_params_default": (None, [_P(CoffeeParams)]),
    "coffee_params_parse_toml": (_i, [ctypes.c_char_p, _P(CoffeeParams)]),
    "coffee_env_create": (_i, [_P(CoffeeParams), _i, _pp]),
    "coffee_env_destroy": (_i, [_vp]),
    "coffee_env_grid": (_i, [_vp, _P(CoffeeGrid)]),
    "coffee_env_params": (_i, [_vp, _P(CoffeeParams)]),
    "coffee_fields_create": (_i, [_vp, _i, _pp]),
    "coffee_fields_destroy": (_i, [_vp]),
    "coffee_fields_ptr": (_i, [_vp, _i, _pp]),
    "coffee_fields_upload": (_i, [_vp, _i, _vp]),
    "coffee_fields_download": (_i, [_vp, _i, _vp]),
    "coffee_fields_fill_guards": (_i, [_vp]),
    "coffee_solver_create": (_i, [_vp, _vp, _i, _i, _vp, _pp]),
    "coffee_solver_destroy": (_i, [_vp]),
    "coffee_solver_step": (_i, [_vp, _d, _i]),
    "coffee_solver_set_aux": (_i, [_vp, _i]),
    "coffee_solver_set_arithmetic": (_i, [_vp, _i]),
    "coffee_solver_set_taper_lanes": (_i, [_vp, _i]),
    "coffee_solver_set_energy_diag": (_i, [_vp, _i]),
    "coffee_solver_set_timing": (_i, [_vp, _i]),
    "coffee_solver_last_timing": (_i, [_vp, _P(_d), _P(_i), _P(_d)]),
    "coffee_fields_init_fourier": (_i, [_vp, _P(_d), _i, _P(_d), _P(_d), _P(_d), _i, _P(_d),
                                        _P(_d), _P(_d)]),
    "coffee_solver_launches_per_step": (_i, [_vp]),
    "coffee_diag_reduce": (_i, [_vp, _i, _P(_d)]),
    "coffee_diag_luminosity": (_i, [_vp, _d, _P(_d)]),
    "coffee_solver_check_finite": (_i, [_vp]),
    "coffee_solver_save_snapshot": (_i, [_vp, ctypes.c_char_p, _d, ctypes.c_int64]),
    "coffee_solver_load_snapshot": (_i, [_vp, ctypes.c_char_p, _P(_d), _P(ctypes.c_int64)]),
    "coffee_batch_create": (_i, [_P(_vp), _i, _vp, _P(_vp)]),
    "coffee_batch_step": (_i, [_vp, _P(_d), _i]),
    "coffee_batch_info": (_i, [_vp, _P(_i), _P(_i), _P(_i), _P(_d)]),
    "coffee_batch_destroy": (_i, [_vp]),
    "coffee_batch_set_persistent": (_i, [_vp, _i]),
    "coffee_batch_set_wait_limit": (_i, [_vp, ctypes.c_longlong, _i]),
    "coffee_evolve_noalloc": (_i, [_P(CoffeeParams), _i, _P(_vp), _d, _i, _vp]),
    # learned warm start (include/coffee_surrogate.h); all pointers are device pointers
    "coffee_conv3d_forward": (_i, [_vp, _i, _i, _i, _i, _i, _vp, _i, _vp, _vp, _vp, _i,
                                   ctypes.c_float, _vp]),
    "coffee_conv3d_forward_tc": (_i, [_vp, _i, _i, _i, _i, _i, _vp, _i, _vp, _vp, _vp, _i,
                                      ctypes.c_float, _vp]),
    "coffee_conv3d_tc_fault": (_i, [_P(_i), _i]),
    "coffee_conv3d_tc_set_test_wait": (_i, [ctypes.c_longlong, _i]),
    "coffee_conv3d_flip_weights": (_i, [_vp, _i, _i, _vp, _vp]),
    "coffee_conv3d_backward_data": (_i, [_vp, _i, _i, _i, _i, _i, _vp, _i, _vp, _vp]),
    "coffee_conv3d_backward_weight_workspace": (ctypes.c_size_t, [_i, _i]),
    "coffee_conv3d_backward_weight": (_i, [_vp, _vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp]),
    "coffee_conv3d_backward_weight_tc": (_i, [_vp, _vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp]),
    "coffee_bias_grad": (_i, [_vp, ctypes.c_longlong, _i, _vp, _vp]),
    "coffee_leaky_backward": (_i, [_vp, _vp, ctypes.c_longlong, ctypes.c_float, _vp, _vp, _vp]),
    "coffee_pool2_forward": (_i, [_vp, _i, _i, _i, _i, _i, _vp, _vp]),
    "coffee_pool2_backward_add": (_i, [_vp, _i, _i, _i, _i, _i, _vp, _vp]),
    "coffee_up2_forward": (_i, [_vp, _i, _i, _i, _i, _i, _vp, _i, _i, _vp]),
    "coffee_up2_backward": (_i, [_vp, _i, _i, _i, _i, _i, _i, _i, _vp, _vp]),
    "coffee_channels_copy": (_i, [_vp, ctypes.c_longlong, _i, _vp, _i, _i, _vp]),
    "coffee_channels_add": (_i, [_vp, ctypes.c_longlong, _i, _i, _i, _vp, _vp]),
    "coffee_mse": (_i, [_vp, _vp, _vp, ctypes.c_longlong, _i, _d, _vp, _vp, _vp]),
    "coffee_adam": (_i, [_vp, _vp, _vp, _vp, ctypes.c_longlong, ctypes.c_float, ctypes.c_float,
                         ctypes.c_float, ctypes.c_float, _i, _vp, _vp]),
    "coffee_to_bf16": (_i, [_vp, ctypes.c_longlong, _vp, _vp]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load the shared library once (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise CoffeeError(-1, f"{path} is missing: build it with `python -m coffee_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int):
    if rc != COFFEE_OK:
        msg = load().coffee_last_error_string().decode(errors="replace")
        raise CoffeeError(rc, msg)
    return rc

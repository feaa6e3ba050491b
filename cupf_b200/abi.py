"""ctypes mirror of include/cupf.h, cupf_ek2d.h and the loader of the CUDA library.

The library (cupf_b200/libcupf.so) is built in-tree by cupf_b200/build.py.
Loading fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcupf.so")

CUPF_MAX_PF = 16


class cupf_apt_params(C.Structure):
    _fields_ = [
        ("fnx", C.c_int32), ("fny", C.c_int32), ("fnz", C.c_int32),
        ("num_pf", C.c_int32), ("num_theta", C.c_int32),
        ("bcX", C.c_int32), ("bcY", C.c_int32), ("bcZ", C.c_int32),
        ("thermalType", C.c_int32),
        ("Nx", C.c_int32), ("Ny", C.c_int32), ("Nz", C.c_int32), ("Nt", C.c_int32),
        ("kin_delta", C.c_float), ("eps", C.c_float), ("G", C.c_float), ("z0", C.c_float),
        ("underCoolingRate", C.c_float), ("underCoolingRate0", C.c_float), ("L_cp", C.c_float),
        ("hi", C.c_float), ("lamd", C.c_float), ("dt", C.c_float), ("tau0", C.c_float),
        ("lyd", C.c_float), ("lzd", C.c_float),
        ("r0", C.c_float), ("x0", C.c_float), ("angle", C.c_float), ("V", C.c_float),
        ("mp_len", C.c_float), ("order", C.c_float),
        ("dx", C.c_float), ("W0", C.c_float),
        ("undcool_mean", C.c_float), ("undcool_std", C.c_float), ("nuc_Nmax", C.c_float),
        ("nuc_Nmax0", C.c_float), ("nuc_rad", C.c_float), ("sqrt2", C.c_float),
        ("pts_cell", C.c_int32), ("seed", C.c_int32), ("haloWidth", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


FP = C.POINTER(C.c_float)


class cupf_apt_inputs(C.Structure):
    _fields_ = [(n, FP) for n in ("x", "y", "z", "sint", "cost", "X_mac", "Y_mac", "Z_mac",
                                  "t_mac", "psi_mac", "T_3D")]


class cupf_server_config(C.Structure):
    _fields_ = [("device", C.c_int32), ("precision", C.c_int32), ("num_pf", C.c_int32),
                ("max_active", C.c_int32), ("steps_per_round", C.c_int32),
                ("autotune", C.c_int32), ("hbm_budget_bytes", C.c_int64), ("tile_y", C.c_int32)]


class cupf_ek2d_params(C.Structure):
    """Parameters of the 2D Echebarria–Karma line model (include/cupf_ek2d.h)."""
    _fields_ = ([(n, C.c_int32) for n in ("nx", "ny", "Mt", "seed_val", "tipp", "noi_period")] +
                [("reserved_i", C.c_int32 * 2)] +
                [(n, C.c_float) for n in (
                    "G", "R", "delta", "k", "c_infm", "Dl", "d0", "W0", "c_infty", "eps", "alpha0",
                    "dx", "asp_ratio", "lxd", "eta", "U0", "cfl",
                    "lT", "lamd", "tau0", "R_tilde", "Dl_tilde", "lT_tilde", "dt", "lyd", "hi",
                    "cosa", "sina", "sqrt2", "a_s", "epsilon", "a_12", "dt_sqrt", "blank", "ls")] +
                [("y0", C.c_double), ("reserved_d", C.c_double * 3)])


class cupf_ek2d_info(C.Structure):
    _fields_ = [("steps", C.c_int64), ("shifts", C.c_int64), ("cur_tip", C.c_int32),
                ("tip_thres", C.c_int32), ("t", C.c_double), ("intR", C.c_double),
                ("lT_tilde", C.c_double)]


STATUS = {0: "CUPF_OK", 1: "CUPF_ERR_INVALID", 2: "CUPF_ERR_CUDA", 3: "CUPF_ERR_OOM",
          4: "CUPF_ERR_UNSUPPORTED", 5: "CUPF_ERR_TIMEOUT", 6: "CUPF_ERR_IO", 7: "CUPF_ERR_STATE"}

PREC = {"fp32": 0, "bf16": 1, "fp16": 2}
PREC_EK2D = {"fp32": 0, "bf16": 1, "fp16": 2, "fp64": 3}


class CupfError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS.get(status, status), msg))
        self.status = status


_lib = None


def lib():
    """Load libcupf.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libcupf.so not built (run cupf_b200/build.py): %s" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.cupf_last_error.restype = C.c_char_p
        L.cupf_abi_version.restype = C.c_int
        L.cupf_struct_size.argtypes = [C.c_int]
        L.cupf_struct_size.restype = C.c_size_t
        for name, args in {
            "cupf_apt_create": [C.POINTER(cupf_apt_params), C.POINTER(cupf_apt_inputs), C.c_int,
                                C.c_int, C.POINTER(vp)],
            "cupf_apt_destroy": [vp],
            "cupf_apt_init_from_argmax": [vp, FP, C.POINTER(C.c_int32)],
            "cupf_apt_set_slots": [vp, FP, C.POINTER(C.c_int32), C.c_int64],
            "cupf_apt_get_slots": [vp, FP, C.POINTER(C.c_int32)],
            "cupf_apt_step": [vp, C.c_int32, C.c_int32],
            "cupf_apt_steps_done": [vp, C.POINTER(C.c_int64)],
            "cupf_apt_collect": [vp, C.c_int32, FP, C.POINTER(C.c_int32)],
            "cupf_apt_grain_volumes": [vp, C.c_int32, C.POINTER(C.c_int64)],
            "cupf_apt_qoi_sums": [vp, C.POINTER(C.c_double)],
            "cupf_apt_move_domain": [vp, C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32)],
            "cupf_apt_get_archive": [vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)],
            "cupf_apt_get_z": [vp, FP],
            "cupf_apt_sync": [vp, C.c_int32],
            "cupf_apt_time_steps": [vp, C.c_int32, FP],
            "cupf_apt_set_tuning": [vp, C.c_int32],
            "cupf_apt_set_skip_quiet": [vp, C.c_int32],
            "cupf_apt_set_wait_limit": [vp, C.c_int64],
            "cupf_apt_set_tile": [vp, C.c_int32],
            "cupf_apt_active_cells": [vp, C.POINTER(C.c_uint64)],
            "cupf_apt_merge_overflows": [vp, C.POINTER(C.c_uint64)],
            "cupf_apt_nucl_init": [vp],
            "cupf_apt_nucleate": [vp, C.c_int32, C.POINTER(C.c_int32)],
            "cupf_apt_nucl_reset": [vp],
            "cupf_apt_junction_candidates": [vp, C.POINTER(C.c_int64), C.c_int64,
                                             C.POINTER(C.c_int64), C.POINTER(C.c_uint8)],
            "cupf_host_junctions_3d_cells": [C.c_int] * 3 + [C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int64), C.c_int64,
                                             C.POINTER(C.c_uint8), C.POINTER(C.c_int32), C.c_int],
            "cupf_line_junction_candidates": [C.c_int32, C.c_int32, C.c_int32,
                                              C.POINTER(C.c_int32), C.c_int32,
                                              C.POINTER(C.c_int64), C.c_int64,
                                              C.POINTER(C.c_int64)],
            "cupf_host_line_junctions": [C.c_int] * 4 + [C.POINTER(C.c_int32)] * 3 + [
                C.c_int, C.POINTER(C.c_int32), C.c_int64],
            "cupf_host_line_junctions_cells": [C.c_int] * 4 + [C.POINTER(C.c_int32)] * 2 + [
                C.POINTER(C.c_int64), C.c_int64, C.POINTER(C.c_int32), C.c_int,
                C.POINTER(C.c_int32), C.c_int64],
            "cupf_host_voronoi_substrate": [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int,
                                            C.POINTER(C.c_int32), FP],
            "cupf_host_write_substrate": [C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_int32),
                                          C.c_int, FP],
            "cupf_host_quaternions_to_angles": [C.c_int, C.POINTER(C.c_double), FP],
            "cupf_grain_volumes_noalloc": [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                           C.POINTER(C.c_int64), vp],
            "cupf_dense_create": [C.POINTER(cupf_apt_params), C.POINTER(cupf_apt_inputs), C.c_float,
                                  C.c_int, C.POINTER(vp)],
            "cupf_dense_destroy": [vp],
            "cupf_dense_init_from_argmax": [vp, FP, C.POINTER(C.c_int32)],
            "cupf_dense_prestep": [vp],
            "cupf_dense_step": [vp, C.c_int32],
            "cupf_dense_steps_done": [vp, C.POINTER(C.c_int64)],
            "cupf_dense_collect": [vp, C.c_int32, FP, C.POINTER(C.c_int32)],
            "cupf_dense_get_slots": [vp, FP],
            "cupf_dense_set_slots": [vp, FP, C.c_int64],
            "cupf_dense_move_domain": [vp, C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32),
                                       C.POINTER(C.c_int32)],
            "cupf_dense_get_archive": [vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)],
            "cupf_dense_get_z": [vp, FP],
            "cupf_dense_sync": [vp, C.c_int32],
            "cupf_dense_time_steps": [vp, C.c_int32, FP],
            "cupf_dense_set_tuning": [vp, C.c_int32],
            "cupf_dense_overflow_cells": [vp, C.POINTER(C.c_int64)],
            "cupf_server_create": [C.POINTER(cupf_server_config), C.POINTER(vp)],
            "cupf_server_destroy": [vp],
            "cupf_server_submit": [vp, C.POINTER(cupf_apt_params), C.POINTER(cupf_apt_inputs), FP,
                                   C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_int64)],
            "cupf_server_pump": [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                 C.POINTER(C.c_int32)],
            "cupf_server_result": [vp, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_int64), C.c_int32, C.POINTER(C.c_double),
                                   C.POINTER(C.c_double)],
            "cupf_server_release": [vp, C.c_int64],
            "cupf_server_request_tile": [vp, C.c_int64, C.POINTER(C.c_int32),
                                         C.POINTER(C.c_int32)],
            "cupf_server_set_tile": [vp, C.c_int32],
            "cupf_server_stats": [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64)],
            "cupf_ek2d_derive": [C.POINTER(cupf_ek2d_params), C.c_float],
            "cupf_ek2d_parse_input": [C.c_char_p, C.POINTER(cupf_ek2d_params),
                                      C.POINTER(C.c_int32), C.POINTER(C.c_int32), FP],
            "cupf_ek2d_create": [C.POINTER(cupf_ek2d_params), C.c_int32, C.c_int32, C.POINTER(vp)],
            "cupf_ek2d_destroy": [vp],
            "cupf_ek2d_set_thermal": [vp, C.c_int32, FP, FP, FP],
            "cupf_ek2d_set_state": [vp, FP, FP, FP],
            "cupf_ek2d_prestep": [vp],
            "cupf_ek2d_step": [vp, C.c_int32],
            "cupf_ek2d_get_state": [vp, FP, FP, FP, FP],
            "cupf_ek2d_get_state_f64": [vp] + [C.POINTER(C.c_double)] * 4,
            "cupf_ek2d_get_y": [vp, C.POINTER(C.c_double)],
            "cupf_ek2d_info_get": [vp, C.POINTER(cupf_ek2d_info)],
            "cupf_ek2d_row_means": [vp, C.POINTER(C.c_double)],
            "cupf_ek2d_time_steps": [vp, C.c_int32, FP],
            "cupf_ek2d_stream": [vp, C.POINTER(vp)],
            "cupf_host_ek2d_initial_fields": [C.POINTER(cupf_ek2d_params), C.c_int, FP, FP, FP, FP,
                                              FP, FP, FP, FP],
            "cupf_host_ek2d_perturb": [C.POINTER(cupf_ek2d_params), C.c_int, C.c_float, FP, FP],
            "cupf_host_ek2d_qois": [FP, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_double,
                                    C.POINTER(C.c_double)],
        }.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.cupf_apt_stream.argtypes = [vp]
        L.cupf_apt_stream.restype = vp
        _lib = L
    return _lib


def check(status):
    if status != 0:
        raise CupfError(status, lib().cupf_last_error().decode())
    return status

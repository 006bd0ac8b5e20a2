"""ctypes binding of librrtmg_b200.so (the C-ABI in include/rrtmg_b200.h)."""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "librrtmg_b200.so"

_F = ctypes.c_void_p  # device pointers


class Config(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nk", ctypes.c_int),
                ("p_top", ctypes.c_double),
                ("co2vmr", ctypes.c_float), ("n2ovmr", ctypes.c_float), ("ch4vmr", ctypes.c_float),
                ("cfc11vmr", ctypes.c_float), ("cfc12vmr", ctypes.c_float), ("solcon", ctypes.c_float),
                ("has_reqc", ctypes.c_int), ("has_reqi", ctypes.c_int), ("has_reqs", ctypes.c_int),
                ("icloud", ctypes.c_int), ("cldovrlp", ctypes.c_int), ("fp64_steps", ctypes.c_int)]


LW_IN_FIELDS = ("p3d", "p8w", "pi3d", "t3d", "t8w", "tsk", "dz8w", "qv3d", "qc3d", "qi3d", "qs3d",
                "cldfra3d", "o33d", "emiss", "xland", "xice", "snow", "re_cloud", "re_ice", "re_snow")
LW_OUT_FIELDS = ("rthratenlw", "rthratenlwc", "lwupt", "lwuptc", "lwuptcln", "lwdnt", "lwdntc",
                 "lwdntcln", "lwupb", "lwupbc", "lwupbcln", "lwdnb", "lwdnbc", "lwdnbcln", "glw",
                 "olr", "lwcf")
SW_IN_FIELDS = ("p3d", "p8w", "pi3d", "t3d", "t8w", "tsk", "dz8w", "qv3d", "qc3d", "qi3d", "qs3d",
                "cldfra3d", "o33d", "albedo", "coszr", "xland", "xice", "snow", "re_cloud", "re_ice",
                "re_snow")
SW_OUT_FIELDS = ("rthratensw", "rthratenswc", "swupt", "swuptc", "swuptcln", "swdnt", "swdntc",
                 "swdntcln", "swupb", "swupbc", "swupbcln", "swdnb", "swdnbc", "swdnbcln", "swcf",
                 "gsw", "swddir", "swddni", "swddif", "swdownc", "swddnic", "swddirc", "coszr")


class LwIn(ctypes.Structure):
    _fields_ = [(n, _F) for n in LW_IN_FIELDS]


class LwOut(ctypes.Structure):
    _fields_ = [(n, _F) for n in LW_OUT_FIELDS]


# optional Noah-MP albedos (sf_surface_physics == 8); NULL when not given
SW_ALBEDO_FIELDS = ("alswvisdir", "alswvisdif", "alswnirdir", "alswnirdif")


class SwIn(ctypes.Structure):
    _fields_ = [(n, _F) for n in SW_IN_FIELDS + SW_ALBEDO_FIELDS]


class SwOut(ctypes.Structure):
    _fields_ = [(n, _F) for n in SW_OUT_FIELDS]


class Schedule(ctypes.Structure):
    """rrtmg_schedule (include/rrtmg_b200.h)."""
    _fields_ = [("lw_chunk_columns", ctypes.c_int), ("sw_chunk_columns", ctypes.c_int),
                ("sw_split_max_columns", ctypes.c_int), ("lw_split_max_columns", ctypes.c_int)]


class GemmArgs(ctypes.Structure):
    """rrtmg_gemm_args (include/rrtmg_surrogate.h)."""
    _fields_ = [("A", _F), ("lda", ctypes.c_int), ("B", _F), ("ldb", ctypes.c_int),
                ("M", ctypes.c_int), ("N", ctypes.c_int), ("K", ctypes.c_int), ("ksplit", ctypes.c_int),
                ("epilogue", ctypes.c_int), ("bias", _F), ("C", _F), ("ldc", ctypes.c_int),
                ("split_stride", ctypes.c_size_t), ("H", _F), ("ldh", ctypes.c_int), ("Ht", _F),
                ("ldht", ctypes.c_int), ("aux", _F), ("ldaux", ctypes.c_int), ("Z", _F), ("ldz", ctypes.c_int)]


EPI_F32, EPI_GELU, EPI_DGELU = 0, 1, 2

_I, _FL = ctypes.c_int, ctypes.c_float


class SurFeaturesArgs(ctypes.Structure):
    _fields_ = [("ncol", _I), ("nk", _I), ("ny", _I)] + \
        [(n, _F) for n in ("p3d", "p8w", "t3d", "qv", "qc", "qi", "qs", "cldfra", "o3", "tsk", "albedo", "coszr",
                           "emiss")] + \
        [("row_offset", _I), ("raw", _F), ("ldf", _I), ("mean", _F), ("rstd", _F), ("X", _F), ("ldx", _I),
         ("Xt", _F), ("ldxt", _I), ("lo", _F), ("hi", _F), ("flags", _F), ("x_layout", _I)]


class SurTargetsArgs(ctypes.Structure):
    _fields_ = [("ncol", _I), ("nk", _I), ("ny", _I)] + \
        [(n, _F) for n in ("rthratenlw", "rthratensw", "pi3d", "p8w", "glw", "lwupb", "swdnb", "swupb")] + \
        [("row_offset", _I), ("T", _F), ("ldt", _I)]


class SurAdamArgs(ctypes.Structure):
    _fields_ = [("rows", _I), ("cols", _I), ("w", _F), ("m", _F), ("v", _F), ("grad", _F), ("lr", _FL),
                ("beta1", _FL), ("beta2", _FL), ("eps", _FL), ("bc1", _FL), ("bc2", _FL), ("weight_decay", _FL),
                ("wb", _F), ("ldwb", _I), ("wbt", _F), ("ldwbt", _I)]


class SurDecodeArgs(ctypes.Structure):
    _fields_ = [("ncol", _I), ("nk", _I), ("ny", _I), ("Y", _F), ("ldy", _I), ("out_mean", _F), ("out_std", _F),
                ("coszr", _F), ("pi3d", _F), ("p8w", _F), ("energy_tol", _FL)] + \
        [(n, _F) for n in ("rthratenlw", "rthratensw", "glw", "lwupb", "swdnb", "swupb", "flags")]


class SurMlpArgs(ctypes.Structure):
    """rrtmg_sur_mlp_args (include/rrtmg_surrogate.h)."""
    _fields_ = [("ncol", _I), ("nk", _I), ("ny", _I), ("X", _F), ("W", _F), ("bias", _F * 4),
                ("out_mean", _F), ("out_std", _F), ("coszr", _F), ("pi3d", _F), ("p8w", _F),
                ("energy_tol", _FL)] + \
        [(n, _F) for n in ("rthratenlw", "rthratensw", "glw", "lwupb", "swdnb", "swupb", "flags")]


WEIGHT_IMAGE_BYTES = 1703936  # RRTMG_SUR_WEIGHT_IMAGE_BYTES
MAX_FIELDS = 32  # RRTMG_SUR_MAX_FIELDS


class SurFields(ctypes.Structure):
    """rrtmg_sur_fields (include/rrtmg_surrogate.h)."""
    _fields_ = [("nfields", _I), ("src", _F * MAX_FIELDS), ("dst", _F * MAX_FIELDS), ("nz", _I * MAX_FIELDS)]

class PrologueScalars(ctypes.Structure):
    """rrtmg_prologue_scalars (include/rrtmg_prologue.h)."""
    _fields_ = [("tloctm0", _FL), ("sin_declin", _FL), ("cos_declin", _FL), ("month_lo", _I), ("month_hi", _I),
                ("fact_lo", _FL), ("fact_hi", _FL)]


PROLOGUE_IN_FIELDS = ("qv3d", "qc3d", "qi3d", "qs3d", "t3d", "p3d", "xlat", "xlong")
PROLOGUE_OUT_FIELDS = ("cldfra3d", "o33d", "coszr", "condensate_present")


class PrologueIn(ctypes.Structure):
    _fields_ = [(n, _F) for n in PROLOGUE_IN_FIELDS]


class PrologueOut(ctypes.Structure):
    _fields_ = [(n, _F) for n in PROLOGUE_OUT_FIELDS]


class TendencyBounds(ctypes.Structure):
    """rrtmg_tendency_bounds (include/rrtmg_tendency.h)."""
    _fields_ = [(n, _I) for n in ("ids", "ide", "jds", "jde", "kds", "kde", "ims", "ime", "jms", "jme", "kms",
                                  "kme", "its", "ite", "jts", "jte", "kts", "kte", "specified", "nested",
                                  "periodic_x")]


STATUS = {0: "RRTMG_OK", 1: "RRTMG_BAD_ARG", 2: "RRTMG_UNSUPPORTED_OPTION", 3: "RRTMG_CUDA",
          4: "RRTMG_TIMEOUT"}

EXPORTS = ("rrtmg_create", "rrtmg_create_from_memory", "rrtmg_destroy", "rrtmg_lwrad", "rrtmg_swrad",
           "rrtmg_lwrad_static_scratch", "rrtmg_lwrad_live", "rrtmg_swrad_live", "rrtmg_timing_enable",
           "rrtmg_timing_read", "rrtmg_set_schedule", "rrtmg_get_schedule", "rrtmg_lw_nlayers",
           "rrtmg_last_error", "rrtmg_status_string", "rrtmg_column_status_enable", "rrtmg_last_column_errors",
           "rrtmg_lw_workspace_bytes", "rrtmg_sw_workspace_bytes", "rrtmg_lwrad_ws", "rrtmg_swrad_ws")
FFI_EXPORTS = ("rrtmg_ffi_lwrad", "rrtmg_ffi_swrad", "rrtmg_ffi_set_table_blob", "rrtmg_ffi_lw_workspace_bytes",
               "rrtmg_ffi_sw_workspace_bytes")
SURROGATE_EXPORTS = ("rrtmg_gemm_bf16", "rrtmg_gemm_error", "rrtmg_gemm_set_tile", "rrtmg_gemm_set_wait_ns",
                     "rrtmg_gemm_test_withhold_commit", "rrtmg_sur_features", "rrtmg_sur_targets",
                     "rrtmg_sur_column_stats", "rrtmg_sur_normalize", "rrtmg_sur_gather", "rrtmg_sur_loss_grad",
                     "rrtmg_sur_row_sum", "rrtmg_sur_reduce_splits", "rrtmg_sur_adam", "rrtmg_sur_decode",
                     "rrtmg_sur_compact", "rrtmg_sur_move_columns", "rrtmg_sur_timestamp",
                     "rrtmg_sur_pack_weights", "rrtmg_sur_mlp", "rrtmg_sur_move_fields")
PROLOGUE_EXPORTS = ("rrtmg_radconst", "rrtmg_prologue_scalars_from_calendar", "rrtmg_set_ozone_climatology",
                    "rrtmg_radiation_prologue", "rrtmg_cal_cldfra1", "rrtmg_calc_coszen", "rrtmg_cam_o3rad")
TENDENCY_EXPORTS = ("rrtmg_radiation_tendency", "rrtmg_phy_ra_ten")
TABLES_EXPORTS = ("rrtmg_blob_with_wrf_data", "rrtmg_create_with_wrf_data")

_lib = None


def load(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Load librrtmg_b200.so and declare its signatures (raises if it is missing)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(
            f"{p} is missing: build the CUDA library first (__graft_entry__.build() or "
            "python -m wrf_jax_b200 build); there is no CPU fallback")
    lib = ctypes.CDLL(str(p))
    lib.rrtmg_create.restype = ctypes.c_int
    lib.rrtmg_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    lib.rrtmg_create_from_memory.restype = ctypes.c_int
    lib.rrtmg_create_from_memory.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_void_p)]
    lib.rrtmg_destroy.restype = None
    lib.rrtmg_destroy.argtypes = [ctypes.c_void_p]
    lib.rrtmg_lwrad.restype = ctypes.c_int
    lib.rrtmg_lwrad.argtypes = [ctypes.c_void_p, ctypes.POINTER(Config), ctypes.POINTER(LwIn),
                                ctypes.POINTER(LwOut), ctypes.c_void_p]
    lib.rrtmg_swrad.restype = ctypes.c_int
    lib.rrtmg_swrad.argtypes = [ctypes.c_void_p, ctypes.POINTER(Config), ctypes.POINTER(SwIn),
                                ctypes.POINTER(SwOut), ctypes.c_void_p]
    lib.rrtmg_lwrad_live.restype = ctypes.c_int
    lib.rrtmg_lwrad_live.argtypes = [ctypes.c_void_p, ctypes.POINTER(Config), ctypes.POINTER(LwIn),
                                     ctypes.POINTER(LwOut), ctypes.c_void_p, ctypes.c_void_p]
    lib.rrtmg_swrad_live.restype = ctypes.c_int
    lib.rrtmg_swrad_live.argtypes = [ctypes.c_void_p, ctypes.POINTER(Config), ctypes.POINTER(SwIn),
                                     ctypes.POINTER(SwOut), ctypes.c_void_p, ctypes.c_void_p]
    lib.rrtmg_lwrad_static_scratch.restype = ctypes.c_int
    lib.rrtmg_lwrad_static_scratch.argtypes = [ctypes.c_void_p, ctypes.POINTER(Config), ctypes.POINTER(LwIn),
                                               ctypes.POINTER(LwOut), ctypes.c_void_p]
    lib.rrtmg_timing_enable.restype = ctypes.c_int
    lib.rrtmg_timing_enable.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.rrtmg_timing_read.restype = ctypes.c_int
    lib.rrtmg_timing_read.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.c_int]
    lib.rrtmg_gemm_bf16.restype = ctypes.c_int
    lib.rrtmg_gemm_bf16.argtypes = [ctypes.POINTER(GemmArgs), ctypes.c_void_p]
    lib.rrtmg_gemm_error.restype = ctypes.c_int
    lib.rrtmg_gemm_error.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_uint)]
    lib.rrtmg_gemm_set_wait_ns.restype = ctypes.c_int
    lib.rrtmg_gemm_set_wait_ns.argtypes = [ctypes.c_ulonglong]
    lib.rrtmg_gemm_test_withhold_commit.restype = ctypes.c_int
    lib.rrtmg_gemm_test_withhold_commit.argtypes = [ctypes.c_int]
    V, I, P, FL, SZ = ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_float, ctypes.c_size_t
    sigs = {
        "rrtmg_sur_features": [ctypes.POINTER(SurFeaturesArgs), V],
        "rrtmg_sur_targets": [ctypes.POINTER(SurTargetsArgs), V],
        "rrtmg_sur_column_stats": [P, I, I, I, P, P, P, P, V],
        "rrtmg_sur_normalize": [P, I, I, I, P, P, P, I, I, V],
        "rrtmg_sur_gather": [P, I, P, I, P, I, P, P, I, P, V],
        "rrtmg_sur_loss_grad": [P, P, P, I, I, FL, P, P, I, P, V],
        "rrtmg_sur_row_sum": [P, I, I, I, P, V],
        "rrtmg_sur_reduce_splits": [P, I, SZ, P, V],
        "rrtmg_sur_adam": [ctypes.POINTER(SurAdamArgs), V],
        "rrtmg_sur_decode": [ctypes.POINTER(SurDecodeArgs), V],
        "rrtmg_sur_compact": [P, I, P, P, V],
        "rrtmg_sur_move_columns": [P, P, I, I, I, P, P, I, I, I, V],
        "rrtmg_gemm_set_tile": [I],
        "rrtmg_sur_timestamp": [P, V],
        "rrtmg_sur_pack_weights": [ctypes.POINTER(ctypes.c_void_p * 4), V, V],
        "rrtmg_sur_mlp": [ctypes.POINTER(SurMlpArgs), V],
        "rrtmg_sur_move_fields": [P, P, I, I, ctypes.POINTER(SurFields), I, I, I, V],
        "rrtmg_set_schedule": [V, ctypes.POINTER(Schedule)],
        "rrtmg_radconst": [ctypes.c_double, ctypes.POINTER(FL), ctypes.POINTER(FL)],
        "rrtmg_prologue_scalars_from_calendar": [ctypes.c_double] * 4 + [ctypes.POINTER(PrologueScalars)],
        "rrtmg_set_ozone_climatology": [V, P, I, P, I, P],
        "rrtmg_radiation_prologue": [V, I, I, I, ctypes.POINTER(PrologueScalars), ctypes.POINTER(PrologueIn),
                                     ctypes.POINTER(PrologueOut), V],
        "rrtmg_cal_cldfra1": [V, I, I, I, P, P, P, P, P, P, P, V],
        "rrtmg_calc_coszen": [V, I, I, P, P, ctypes.POINTER(PrologueScalars), P, V],
        "rrtmg_cam_o3rad": [V, I, I, I, P, P, ctypes.POINTER(PrologueScalars), P, V],
        "rrtmg_radiation_tendency": [ctypes.POINTER(TendencyBounds), P, P, P, P, P, I, P, P, V],
        "rrtmg_phy_ra_ten": [ctypes.POINTER(TendencyBounds), P, P, V],
        "rrtmg_blob_with_wrf_data": [ctypes.c_char_p] * 4,
        "rrtmg_create_with_wrf_data": [ctypes.c_char_p] * 3 + [I, ctypes.POINTER(ctypes.c_void_p)],
        "rrtmg_get_schedule": [V, ctypes.POINTER(Schedule)],
        "rrtmg_column_status_enable": [V, I],
        "rrtmg_last_column_errors": [V, I, P, I, V],
    }
    for name, argtypes in sigs.items():
        fn = getattr(lib, name)
        fn.restype = ctypes.c_int
        fn.argtypes = argtypes
    lib.rrtmg_lw_nlayers.restype = ctypes.c_int
    lib.rrtmg_lw_nlayers.argtypes = [ctypes.c_double, ctypes.c_int]
    lib.rrtmg_last_error.restype = ctypes.c_char_p
    lib.rrtmg_last_error.argtypes = [ctypes.c_void_p]
    lib.rrtmg_status_string.restype = ctypes.c_char_p
    lib.rrtmg_status_string.argtypes = [ctypes.c_int]
    if path is None:
        _lib = lib
    return lib

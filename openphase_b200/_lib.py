"""ctypes binding of the opgpu C ABI (include/opgpu.h).

The library is the in-tree build openphase_b200/lib/libopgpu.so.  Loading it needs no GPU; every
compute entry point reports OPGPU_E_NODEVICE when none is present.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libopgpu.so"

OPGPU_OK = 0
E_OVERFLOW_K = 1 << 0
E_OVERFLOW_LIST = 1 << 1
E_EMPTY_VOXEL = 1 << 2
E_NORMALIZE_WARN = 1 << 3
E_LIMITER_CAP = 1 << 4
E_NONFINITE = 1 << 5
E_ADJOINT_MISMATCH = 1 << 6
E_AVERAGE_SKIPPED = 1 << 7
E_INVALID = 1 << 8
E_CUDA = 1 << 9
E_IO = 1 << 10
E_STATE = 1 << 11
E_NODEVICE = 1 << 12
SOFT_MASK = 0xFF

FP64, FP32 = 0, 1
STENCIL = {"SIMPLE": 0, "ISOTROPIC": 1, "LB": 2}
STAGE_STABLE, STAGE_SEED, STAGE_NUCLEUS = 0, 1, 2

_CODE_NAMES = {
    E_OVERFLOW_K: "OVERFLOW_K", E_OVERFLOW_LIST: "OVERFLOW_LIST", E_EMPTY_VOXEL: "EMPTY_VOXEL",
    E_NORMALIZE_WARN: "NORMALIZE_WARN", E_LIMITER_CAP: "LIMITER_CAP", E_NONFINITE: "NONFINITE",
    E_ADJOINT_MISMATCH: "ADJOINT_MISMATCH",
    E_AVERAGE_SKIPPED: "AVERAGE_SKIPPED",
    E_INVALID: "INVALID", E_CUDA: "CUDA", E_IO: "IO", E_STATE: "STATE", E_NODEVICE: "NODEVICE",
}


def code_names(code: int):
    return [n for b, n in _CODE_NAMES.items() if code & b]


class OpgpuError(RuntimeError):
    def __init__(self, code, msg=""):
        self.code = code
        super().__init__(f"opgpu error {code:#x} {code_names(code)} {msg}".strip())


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("dx", C.c_double),
                ("iwidth", C.c_double), ("laplacian_stencil", C.c_int32), ("gradient_stencil", C.c_int32),
                ("precision", C.c_int32), ("k_slots", C.c_int32), ("device", C.c_int32)]


class Model(C.Structure):
    _fields_ = [("nphases", C.c_int32), ("sigma", C.POINTER(C.c_double)), ("mu", C.POINTER(C.c_double)),
                ("limit", C.POINTER(C.c_double)), ("limiting", C.c_int32), ("regularization", C.c_double),
                ("tj_factor", C.c_double), ("consider_nucleus_volume", C.c_int32),
                ("nucleus_volume_factor", C.c_double), ("energy_model", C.POINTER(C.c_int32)),
                ("cubic_eps", C.POINTER(C.c_double)), ("phase_solid", C.POINTER(C.c_int32)),
                ("model_eps", C.POINTER(C.c_double)), ("facet_start", C.POINTER(C.c_int32)),
                ("facet_data", C.POINTER(C.c_double)), ("facet_family", C.POINTER(C.c_int32)),
                ("mobility_model", C.POINTER(C.c_int32)), ("mobility_eps", C.POINTER(C.c_double)),
                ("mobility_facet_start", C.POINTER(C.c_int32)), ("mobility_facet_data", C.POINTER(C.c_double)),
                ("mobility_facet_family", C.POINTER(C.c_int32))]


class Stats(C.Structure):
    _fields_ = [("steps", C.c_int64), ("wide_last", C.c_int64), ("wide_total", C.c_int64),
                ("entries_in_total", C.c_int64), ("entries_out_total", C.c_int64),
                ("status", C.c_uint32), ("overflow_voxels", C.c_uint32), ("timed_launches", C.c_int64),
                ("timed_kernel_ms", C.c_double), ("general_path_total", C.c_int64),
                ("crowded_window_total", C.c_int64), ("timed_classify_ms", C.c_double),
                ("kernel_launches", C.c_int64)]


_lib = None

# name -> (restype, argtypes); every symbol include/opgpu.h declares
_P = C.c_void_p
_SIGS = {
    "opgpu_create": (C.c_uint32, [C.POINTER(Grid), C.POINTER(_P)]),
    "opgpu_destroy": (C.c_uint32, [_P]),
    "opgpu_last_error": (C.c_char_p, [_P]),
    "opgpu_abi_version": (C.c_int32, []),
    "opgpu_build_info": (C.c_char_p, []),
    "opgpu_step_save_input": (C.c_uint32, [_P, C.c_double, C.c_int32]),
    "opgpu_device_count": (C.c_int32, []),
    "opgpu_set_model": (C.c_uint32, [_P, C.POINTER(Model)]),
    "opgpu_set_grains": (C.c_uint32, [_P, C.c_int32, _P, _P]),
    "opgpu_set_pair_table": (C.c_uint32, [_P, _P, _P]),
    "opgpu_set_pair_hash": (C.c_uint32, [_P, C.c_uint64, C.c_double, C.c_double]),
    "opgpu_set_driving_force": (C.c_uint32, [_P, _P]),
    "opgpu_set_orientations": (C.c_uint32, [_P, _P]),
    "opgpu_set_averaging": (C.c_uint32, [_P, C.c_int32, C.c_int32, C.c_double]),
    "opgpu_upload_lists": (C.c_uint32, [_P, _P, _P, _P]),
    "opgpu_read_raw": (C.c_uint32, [_P, C.c_char_p]),
    "opgpu_write_raw": (C.c_uint32, [_P, C.c_char_p]),
    "opgpu_finalize_initialization": (C.c_uint32, [_P]),
    "opgpu_write_grains": (C.c_uint32, [_P, C.c_char_p]),
    "opgpu_read_grains": (C.c_uint32, [_P, C.c_char_p]),
    "opgpu_write_vtk": (C.c_uint32, [_P, C.c_char_p]),
    "opgpu_write_vtk_host": (C.c_uint32, [C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, C.c_int32, _P, C.c_int32,
                                          C.c_int32, C.c_int32, C.c_char_p]),
    "opgpu_total_entries": (C.c_uint32, [_P, C.POINTER(C.c_int64)]),
    "opgpu_download_lists": (C.c_uint32, [_P, _P, _P, _P]),
    "opgpu_download_flags": (C.c_uint32, [_P, _P]),
    "opgpu_download_flags_noalloc": (C.c_uint32, [_P, _P]),
    "opgpu_step": (C.c_uint32, [_P, C.c_double, C.c_int32]),
    "opgpu_step_async": (C.c_uint32, [_P, C.c_double, C.c_int32]),
    "opgpu_sync": (C.c_uint32, [_P]),
    "opgpu_grains": (C.c_uint32, [_P, _P, _P, _P, _P, _P]),
    "opgpu_get_stats": (C.c_uint32, [_P, C.POINTER(Stats)]),
    "opgpu_clear_status": (C.c_uint32, [_P]),
    "opgpu_set_timing": (C.c_uint32, [_P, C.c_int32]),
    "opgpu_set_kernel_variant": (C.c_uint32, [_P, C.c_int32]),
    "opgpu_stream": (_P, [_P]),
    "opgpu_checkpoint_reserve": (C.c_uint32, [_P, C.c_int32]),
    "opgpu_checkpoint_save": (C.c_uint32, [_P, C.c_int32]),
    "opgpu_checkpoint_load": (C.c_uint32, [_P, C.c_int32]),
    "opgpu_adjoint_begin": (C.c_uint32, [_P, _P]),
    "opgpu_adjoint_step": (C.c_uint32, [_P, C.c_int32, C.c_double]),
    "opgpu_adjoint_gradients": (C.c_uint32, [_P, _P, _P, _P]),
    "opgpu_tlm_begin": (C.c_uint32, [_P, _P, _P, _P]),
    "opgpu_tlm_step": (C.c_uint32, [_P, C.c_double, C.c_int32]),
    "opgpu_tlm_volumes": (C.c_uint32, [_P, _P]),
    "opgpu_set_volume_window": (C.c_uint32, [_P, C.c_int32, C.c_int32]),
    "opgpu_plane_bytes": (C.c_int64, [_P]),
    "opgpu_pack_plane": (C.c_uint32, [_P, C.c_int32, _P]),
    "opgpu_unpack_plane": (C.c_uint32, [_P, C.c_int32, _P]),
    "opgpu_volume_recount": (C.c_uint32, [_P]),
    "opgpu_step_partial": (C.c_uint32, [_P, C.c_double]),
    "opgpu_set_stream_ordered": (C.c_uint32, [_P, C.c_int32]),
    "opgpu_volume_accumulator": (C.c_uint32, [_P, _P]),
    "opgpu_step_complete": (C.c_uint32, [_P, _P, C.c_int32]),
    "opgpu_uniform": (C.c_double, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64]),
    "opgpu_voronoi_owner_host": (C.c_uint32, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64,
                                              C.c_int32, _P]),
    "opgpu_spread_boundaries_host": (C.c_uint32, [C.c_int32, C.c_int32, C.c_int32, _P, C.c_int32, _P, _P,
                                                  C.POINTER(C.c_int64)]),
    "opgpu_pair_table_host": (C.c_uint32, [C.c_int32, C.c_uint64, C.c_uint64, C.c_double, C.c_double, _P]),
    "opgpu_grain_values_host": (C.c_uint32, [C.c_int32, C.c_uint64, C.c_uint64, C.c_double, _P]),
}


def lib():
    """Load libopgpu.so (fails loudly if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise OpgpuError(E_NODEVICE, f"{LIB_PATH} is not built; run python -m openphase_b200.build_ext")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def device_count() -> int:
    return int(lib().opgpu_device_count())

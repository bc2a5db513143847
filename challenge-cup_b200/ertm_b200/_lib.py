"""ctypes binding of the C ABI in ``include/ertm_b200.h``.

The library is the in-tree ``libertm_b200.so`` built for sm_100a by
``challenge-cup_b200/build.py``.  There is no CPU fallback: when the library
or a B200 is missing, every call raises ``SolverError``.
"""

from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

import numpy as np

from .exceptions import NonFiniteWavefieldError, SolverError

# ERTM_B200_LIBRARY selects another build of the library (e.g. one compiled
# with different tile options); the default is the in-tree build.
LIB_PATH = Path(os.environ.get("ERTM_B200_LIBRARY") or Path(__file__).resolve().parent / "libertm_b200.so")

ENGINE = {"acoustic": 0, "elastic": 1, "viscoacoustic": 2}
COMP = {"p": 0, "vx": 1, "vz": 2, "sxx": 3, "szz": 4, "sxz": 5}
MECH = {"explosive": 0, "shear": 1, "force_z": 2}
COND = {"zero_lag": 0, "normalized": 1, "excitation": 2}
WAVE = {"P": 0, "S": 1}
SEP = {"stress": 0, "divcurl": 1}
ACCUM = {"fp64": 0, "kahan": 1}


class PropConfig(C.Structure):
    _fields_ = [
        ("engine", C.c_int32), ("order", C.c_int32), ("nx", C.c_int32), ("nz", C.c_int32),
        ("dx", C.c_double), ("dz", C.c_double), ("x0", C.c_double), ("z0", C.c_double), ("dt", C.c_double),
        ("free_surface", C.c_int32), ("npml_x_left", C.c_int32), ("npml_x_right", C.c_int32),
        ("npml_z_top", C.c_int32), ("npml_z_bottom", C.c_int32), ("n_mech", C.c_int32), ("n_q", C.c_int32),
        ("compensation", C.c_int32), ("amplitude_cap", C.c_double), ("lowpass_interval", C.c_int32),
        ("reserved", C.c_int32),
    ]


class PropInfo(C.Structure):
    _fields_ = [
        ("nzp", C.c_int32), ("nxp", C.c_int32), ("ld", C.c_int32), ("pad", C.c_int32),
        ("state_bytes", C.c_int64), ("field_bytes", C.c_int64), ("step_index", C.c_int64),
        ("n_fields", C.c_int32), ("clipped", C.c_int32), ("lowpass_steps", C.c_int32),
        ("n_receivers", C.c_int32), ("fast_div_x", C.c_int32), ("fast_div_z", C.c_int32),
        ("tile_rows", C.c_int32), ("reserved", C.c_int32),
    ]


class MigrateConfig(C.Structure):
    _fields_ = [
        ("nt", C.c_int32), ("nt_spec", C.c_int32), ("interval", C.c_int32), ("condition", C.c_int32),
        ("illumination", C.c_int32), ("start_step", C.c_int32), ("separation", C.c_int32),
        ("n_images", C.c_int32), ("src_wave", C.c_int32 * 4), ("rcv_wave", C.c_int32 * 4),
        ("accum", C.c_int32), ("n_comp", C.c_int32), ("comp", C.c_int32 * 8),
    ]


class BatchShot(C.Structure):
    _fields_ = [
        ("fwd", C.c_void_p), ("back", C.c_void_p), ("cfg", MigrateConfig), ("wavelet", C.c_void_p),
        ("record", C.c_void_p), ("num", C.c_void_p), ("illum", C.c_void_p), ("rillum", C.c_void_p),
    ]


_P = C.c_void_p
_I32 = C.c_int32
_SIGNATURES = {
    "ertm_last_error": (C.c_char_p, []),
    "ertm_version": (_I32, []),
    "ertm_init": (_I32, [_I32]),
    "ertm_launch_count": (C.c_int64, []),
    "ertm_set_tile_rows": (_I32, [_I32]),
    "ertm_set_tile_split": (_I32, [_I32]),
    "ertm_set_tick_lanes": (_I32, [_I32]),
    "ertm_set_lane_assign": (_I32, [_I32]),
    "ertm_set_frame_rows": (_I32, [_I32]),
    "ertm_set_line_threads": (_I32, [_I32]),
    "ertm_set_march": (_I32, [_I32]),
    "ertm_set_march_stress": (_I32, [_I32]),
    "ertm_set_autotune": (_I32, [_I32]),
    "ertm_set_tma": (_I32, [_I32]),
    "ertm_stage_timeouts": (C.c_int64, []),
    "ertm_autotune_report": (C.c_char_p, []),
    "ertm_division_check": (_I32, [C.c_float, _I32, C.POINTER(C.c_uint64)]),
    "ertm_profile_stencil": (_I32, [_I32, _I32]),
    "ertm_profile_read": (_I32, [C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_double)]),
    "ertm_prop_create": (_P, [C.POINTER(PropConfig)] + [_P] * 12 + [_P]),
    "ertm_prop_destroy": (None, [_P]),
    "ertm_prop_info_get": (_I32, [_P, C.POINTER(PropInfo)]),
    "ertm_prop_reset": (_I32, [_P]),
    "ertm_prop_status": (_I32, [_P, _P]),
    "ertm_prop_set_source": (_I32, [_P, _I32, _I32, _I32]),
    "ertm_prop_set_receivers": (_I32, [_P, _I32, _P, _P]),
    "ertm_prop_step": (_I32, [_P, _I32, _P]),
    "ertm_prop_sample": (_I32, [_P, _I32, _P, _P]),
    "ertm_prop_inject": (_I32, [_P, _I32, _P]),
    "ertm_prop_image_field": (_I32, [_P, _I32, _I32, _P]),
    "ertm_prop_read_field": (_I32, [_P, _I32, _P]),
    "ertm_prop_write_field": (_I32, [_P, _I32, _P]),
    "ertm_prop_read_psi": (_I32, [_P, _I32, _I32, _P]),
    "ertm_prop_write_psi": (_I32, [_P, _I32, _I32, _P]),
    "ertm_prop_set_step_index": (_I32, [_P, C.c_int64]),
    "ertm_prop_save_state": (_I32, [_P, _P]),
    "ertm_prop_load_state": (_I32, [_P, _P]),
    "ertm_forward": (_I32, [_P, _I32, _P, _I32, _P, _P]),
    "ertm_migrate": (_I32, [_P, _P, C.POINTER(MigrateConfig), _P, _P, _P, _P, _P]),
    "ertm_migrate_batch": (_I32, [_I32, C.POINTER(BatchShot)]),
    "ertm_postprocess": (_I32, [_I32, _I32, C.c_double, C.c_double, _P, _P, _P, _I32, _I32, C.c_double,
                                _I32, C.c_double, _I32, _I32, _P, _P]),
    "ertm_stack": (_I32, [_I32, C.c_int64, _P, _I32, _P, _P]),
    "ertm_stack_noalloc": (_I32, [_I32, C.c_int64, _P, _I32, _P, _P]),
    "ertm_stack_partial": (_I32, [_I32, C.c_int64, _P, _I32, _P, _P]),
    "ertm_lowpass_wavenumber": (_I32, [_I32, _I32, C.c_double, C.c_double, C.c_double, _P, _P, _P]),
    "ertm_resample": (_I32, [_P, C.c_int64, C.c_int64, _P, _P, _I32, C.c_int64, _P, _P]),
    "ertm_mute": (_I32, [_P, C.c_int64, C.c_int64, _P, _P, _P, _P, _P]),
    "ertm_taper": (_I32, [_P, C.c_int64, C.c_int64, _P, C.c_int64, _P, _P]),
    "ertm_rotate": (_I32, [_P, _P, C.c_int64, C.c_double, C.c_double, _P, _P, _P]),
    "ertm_stft_filter": (_I32, [_P, C.c_int64, C.c_int64, _I32, _I32, _I32, _P, _P, _P, _P]),
    "ertm_segy_decode": (_I32, [_P, C.c_int64, C.c_int64, _I32, C.c_int64, _P, _P, _P, _P, C.c_int64, _P]),
    "ertm_segy_encode": (_I32, [_P, C.c_int64, C.c_int64, _I32, _P, _P, _P]),
    "ertm_session_create": (_I32, [C.POINTER(C.c_void_p)]),
    "ertm_session_add": (_I32, [_P, C.POINTER(BatchShot), C.c_int64]),
    "ertm_session_advance": (_I32, [_P, _I32, C.POINTER(C.c_int64), _I32, C.POINTER(C.c_int32)]),
    "ertm_session_active": (_I32, [_P]),
    "ertm_session_take_failed": (_I32, [_P, _P, _I32, _P]),
    "ertm_session_ticks": (C.c_int64, [_P]),
    "ertm_session_destroy": (_I32, [_P]),
    "ertm_stack_finish": (_I32, [C.c_int64, _P, C.c_int64, _P, _P]),
}

_lock = threading.Lock()
_lib: C.CDLL | None = None
_device_ready: int | None = None


def exported_symbols() -> list[str]:
    """Names every binding expects; the CPU tests check the .so exports them."""
    return list(_SIGNATURES)


def load() -> C.CDLL:
    """Load the shared library (no device needed)."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise SolverError(f"CUDA library {LIB_PATH.name} is not built; run challenge-cup_b200/build.py")
            lib = C.CDLL(str(LIB_PATH))
            for name, (res, args) in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def lib(device: int = 0) -> C.CDLL:
    """The library with the CUDA device initialised (sm_100 checked)."""
    global _device_ready
    L = load()
    if _device_ready != device:
        rc = L.ertm_init(device)
        if rc != 0:
            raise SolverError(f"CUDA device unavailable: {last_error()}")
        _device_ready = device
    return L


def last_error() -> str:
    msg = load().ertm_last_error()
    return msg.decode() if msg else ""


ERR_NONFINITE = -4
STATUS_NONFINITE = 1


def check(rc: int, what: str) -> None:
    if rc == ERR_NONFINITE:
        raise NonFiniteWavefieldError(f"{what} failed: {last_error()}")
    if rc != 0:
        raise SolverError(f"{what} failed: {last_error()}")


def ptr(a) -> int | None:
    """Address of a contiguous numpy array or torch tensor (None → NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError(f"cannot take the address of {type(a).__name__}")

"""ctypes binding of the C ABI in ``include/jaxphys_fdtd.h``.

The shared library is built in-tree (``jaxphys_b200/_lib/libjaxphys_fdtd.so``,
see ``jaxphys_b200/build.py``).  There is no fallback: if the library is
missing or a call fails, an exception is raised.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from .exceptions import NumericalInstabilityError, SimulationError

LIB_DIR = Path(__file__).resolve().parent / "_lib"
LIB_PATH = LIB_DIR / "libjaxphys_fdtd.so"

OK = 0
ERR_INVALID = 1
ERR_CUDA = 2
ERR_OOM = 3
ERR_TIMEOUT = 4
ERR_NONFINITE = 5

BND_ABSORBING = 0
BND_PERIODIC = 1
BND_PEC = 2
BND_CPML = 3
BND_REFLECTING = 4

PATH_AUTO = 0
PATH_GENERIC = 1
PATH_TMA = 2


class Grid3DDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("dx", C.c_double), ("dt", C.c_double),
        ("boundary", C.c_int32), ("pml_layers", C.c_int32),
        ("cpml_order", C.c_double), ("cpml_r0", C.c_double),
        ("cpml_kappa_max", C.c_double), ("cpml_alpha_max", C.c_double),
        ("path", C.c_int32), ("device", C.c_int32),
    ]


class Grid3DInfo(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("coef_h", C.c_double), ("coef_e", C.c_double),
        ("step", C.c_int64), ("path", C.c_int32),
        ("tile_z", C.c_int32), ("tile_y", C.c_int32), ("rows_per_thread", C.c_int32),
        ("stages", C.c_int32), ("x_chunk", C.c_int32),
        ("device_bytes", C.c_int64),
        ("kernels_per_step", C.c_int32),
        ("shell_blocks", C.c_int32), ("interior_blocks", C.c_int32),
        ("tma_config", C.c_int32), ("axis_split", C.c_int32),
        ("blocked_config", C.c_int32), ("blocked_x_chunk", C.c_int32),
        ("blocked_kernels_per_pass", C.c_int32),
    ]


class NoAllocDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("dx", C.c_double), ("dt", C.c_double),
        ("boundary", C.c_int32), ("pml_layers", C.c_int32),
        ("device", C.c_int32),
    ]


class Grid2DDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("dx", C.c_double), ("dt", C.c_double),
        ("boundary", C.c_int32), ("pml_layers", C.c_int32),
        ("device", C.c_int32),
    ]


# learned band layout (include/jaxphys_fdtd.h)
BAND_PARAMS = 9360
BAND_FACES = 6
BAND_FEATURES = 54

_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_pf = C.POINTER(C.c_float)
_pd = C.POINTER(C.c_double)
_pi32 = C.POINTER(C.c_int32)
_pi64 = C.POINTER(C.c_int64)

# name -> (restype, argtypes); every symbol declared in include/jaxphys_fdtd.h
SIGNATURES = {
    "jxf_last_error": (C.c_char_p, []),
    "jxf_version": (C.c_int, []),
    "jxf_num_tma_configs": (C.c_int, []),
    "jxf_grid3d_create": (C.c_int, [C.POINTER(Grid3DDesc), C.POINTER(_vp)]),
    "jxf_grid3d_destroy": (C.c_int, [_vp]),
    "jxf_grid3d_get_info": (C.c_int, [_vp, C.POINTER(Grid3DInfo)]),
    "jxf_grid3d_set_launch": (C.c_int, [_vp, _i32, _i32]),
    "jxf_grid3d_set_axis_split": (C.c_int, [_vp, _i32]),
    "jxf_num_blocked_configs": (C.c_int, []),
    "jxf_batch3d_kernels_per_step": (C.c_int, [_vp]),
    "jxf_batch3d_launch": (C.c_int, [_vp, C.POINTER(C.c_int32)]),
    "jxf_grid3d_set_blocked": (C.c_int, [_vp, _i32, _i32]),
    "jxf_grid3d_set_eps_host": (C.c_int, [_vp, _vp]),
    "jxf_grid3d_set_eps_device": (C.c_int, [_vp, _vp, _vp]),
    "jxf_grid3d_set_sources": (C.c_int, [_vp, _i32, _vp, _vp, _vp, _vp]),
    "jxf_grid3d_set_waveforms": (C.c_int, [_vp, _i32, _i64, _vp]),
    "jxf_grid3d_set_probes": (C.c_int, [_vp, _i32, _vp, _vp]),
    "jxf_grid3d_step": (C.c_int, [_vp, _i32, _vp, _vp]),
    "jxf_grid3d_reset": (C.c_int, [_vp, _vp]),
    "jxf_grid3d_field_ptr": (C.c_int, [_vp, _i32, C.POINTER(_vp)]),
    "jxf_grid3d_get_field": (C.c_int, [_vp, _i32, _vp, _i32, _vp]),
    "jxf_grid3d_set_field": (C.c_int, [_vp, _i32, _vp, _i32, _vp]),
    "jxf_grid3d_snapshot": (C.c_int, [_vp, _vp, _vp]),
    "jxf_grid3d_check_error": (C.c_int, [_vp, _vp]),
    "jxf_grid3d_check_finite": (C.c_int, [_vp, _vp]),
    "jxf_grid3d_adjoint_forward": (C.c_int, [_vp, _i32, _i32, _vp, _vp]),
    "jxf_grid3d_adjoint_backward": (C.c_int, [_vp, _vp, _vp, _vp]),
    "jxf_grid3d_create_slab": (C.c_int, [C.POINTER(Grid3DDesc), _i32, _i32, C.POINTER(_vp)]),
    "jxf_grid3d_half_step": (C.c_int, [_vp, _i32, _vp, _vp]),
    "jxf_grid3d_half_step_part": (C.c_int, [_vp, _i32, _i32, _vp, _vp]),
    "jxf_grid3d_plane": (C.c_int, [_vp, _i32, _i32, _vp, _i32, _vp]),
    "jxf_batch3d_create": (C.c_int, [_i32, C.POINTER(_vp), C.POINTER(_vp)]),
    "jxf_batch3d_destroy": (C.c_int, [_vp]),
    "jxf_batch3d_reset": (C.c_int, [_vp, _vp]),
    "jxf_batch3d_step": (C.c_int, [_vp, _i32, _i32, _vp]),
    "jxf_batch3d_probes": (C.c_int, [_vp, _i32, _i32, _vp, _vp]),
    "jxf_band_create": (C.c_int, [_i32, C.POINTER(_vp)]),
    "jxf_band_destroy": (C.c_int, [_vp]),
    "jxf_band_set_params": (C.c_int, [_vp, _vp]),
    "jxf_band_get_params": (C.c_int, [_vp, _vp]),
    "jxf_band_eval": (C.c_int, [_vp, _i32, _vp, _vp, _vp]),
    "jxf_band_collect": (C.c_int, [_vp, C.POINTER(_vp), _i32, _i32, _i32, C.POINTER(_vp), _i32,
                                   _i32, _i32, _i32, _i32, _i32, _vp]),
    "jxf_band_dataset_size": (C.c_int, [_vp, _vp]),
    "jxf_band_dataset_clear": (C.c_int, [_vp]),
    "jxf_band_dataset_get": (C.c_int, [_vp, _i32, _i64, _i64, _vp, _vp, _vp]),
    "jxf_band_grad": (C.c_int, [_vp, _vp, _vp, _vp]),
    "jxf_band_train": (C.c_int, [_vp, _i32, _i32, C.c_float, C.c_uint64, _vp, _vp]),
    "jxf_band_check_error": (C.c_int, [_vp, _vp]),
    "jxf_batch3d_set_band": (C.c_int, [_vp, _vp]),
    "jxf_grid3d_set_band": (C.c_int, [_vp, _vp]),
    "jxf_grid3d_run_noalloc": (C.c_int, [C.POINTER(NoAllocDesc), C.POINTER(_vp), _vp, _i32, _vp]),
    "jxf_slice_absmax": (C.c_int, [_vp, _i64, _i64, _i64, _i64, _i32, _i64, _vp, _vp]),
    "jxf_slice_rgb": (C.c_int, [_vp, _i64, _i64, _i64, _i64, _i32, _i64, _vp, C.c_float, _vp,
                                _vp, _vp]),
    "jxf_grid2d_create": (C.c_int, [C.POINTER(Grid2DDesc), C.POINTER(_vp)]),
    "jxf_grid2d_destroy": (C.c_int, [_vp]),
    "jxf_grid2d_set_sources": (C.c_int, [_vp, _i32, _vp, _vp, _vp]),
    "jxf_grid2d_set_waveforms": (C.c_int, [_vp, _i32, _i64, _vp]),
    "jxf_grid2d_set_walls": (C.c_int, [_vp, _i32, _vp, _vp, _vp]),
    "jxf_grid2d_step": (C.c_int, [_vp, _i32, _vp]),
    "jxf_grid2d_reset": (C.c_int, [_vp, _vp]),
    "jxf_grid2d_field_ptr": (C.c_int, [_vp, _i32, C.POINTER(_vp)]),
    "jxf_grid2d_get_field": (C.c_int, [_vp, _i32, _vp, _i32, _vp]),
    "jxf_grid2d_set_field": (C.c_int, [_vp, _i32, _vp, _i32, _vp]),
    "jxf_grid2d_snapshot": (C.c_int, [_vp, _vp, _vp]),
    "jxf_grid2d_check_error": (C.c_int, [_vp, _vp]),
}

_lib = None


def load():
    """Load (once) and return the FDTD shared library; raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("JXF_LIB", str(LIB_PATH)))
    if not path.exists():
        raise SimulationError(
            f"native FDTD library not found at {path}; build it with "
            "`python -m jaxphys_b200.build` (needs nvcc with sm_100a support)")
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    msg = load().jxf_last_error()
    return msg.decode(errors="replace") if msg else ""


def check(rc: int, what: str) -> None:
    """Raise the matching exception for a non-zero status."""
    if rc == OK:
        return
    msg = f"{what}: {last_error()} (status {rc})"
    if rc == ERR_NONFINITE:
        raise NumericalInstabilityError(msg)
    if rc == ERR_INVALID:
        from .exceptions import ConfigurationError
        raise ConfigurationError(msg)
    raise SimulationError(msg)


def ptr(t) -> C.c_void_p:
    """Device / host data pointer of a torch tensor or NumPy array."""
    if hasattr(t, "data_ptr"):
        return C.c_void_p(t.data_ptr())
    return C.c_void_p(t.ctypes.data)


def stream_handle(stream=None) -> C.c_void_p:
    """cudaStream_t of a torch stream (current stream by default)."""
    import torch

    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)

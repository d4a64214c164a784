"""ctypes binding of the C ABI in ``include/kennett_b200.h`` (``libkennett_b200.so``).

The library is the only compute path: if it is missing, or no CUDA device is visible,
every entry point raises.  There is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

__all__ = ["lib", "check", "KennettError", "LIB_PATH", "exported_symbols"]

LIB_PATH = Path(__file__).resolve().with_name("libkennett_b200.so")

KR_OK = 0
KR_ERR_INVALID_ARGUMENT = 1
KR_ERR_INVALID_MODEL = 2
KR_ERR_CUDA = 3
KR_ERR_CUFFT = 4
KR_ERR_WORKSPACE = 5
KR_ERR_TOO_LARGE = 6

KR_FREE_SURFACE = 0x1
KR_BATCH_GRADIENT = 0x2
KR_BATCH_STORE_R = 0x4


class BatchConfig(ctypes.Structure):
    """kr_batch_config."""

    _fields_ = [("threads", ctypes.c_int32), ("tile_w", ctypes.c_int32),
                ("reserved0", ctypes.c_int32), ("reserved1", ctypes.c_int32)]


# numpy dtype with the layout of kr_model_desc (64 bytes)
MODEL_DESC_FIELDS = [("n_layers", "<i4"), ("n_p", "<i4"), ("n_w", "<i4"), ("flags", "<u4"),
                     ("layers_off", "<i8"), ("p_off", "<i8"), ("omega_off", "<i8"),
                     ("R_off", "<i8"), ("obs_off", "<i8"), ("grad_off", "<i8")]

_c_double_p = ctypes.c_void_p  # device pointers travel as integers
_size_t = ctypes.c_size_t
_i32 = ctypes.c_int32
_u32 = ctypes.c_uint32
_vp = ctypes.c_void_p

# name -> (restype, argtypes); kept in step with include/*.h
_SIGNATURES = {
    "kr_status_string": (ctypes.c_char_p, [_i32]),
    "kr_last_error": (ctypes.c_char_p, []),
    "kr_version": (_i32, []),
    "kr_validate_layers": (_i32, [_vp, _i32]),
    "kr_reflectivity": (_i32, [_vp, _i32, _vp, _i32, _vp, _i32, _u32, _vp, _vp]),
    "kr_gmm_reflectivity": (_i32, [_vp, _i32, _vp, _i32, _vp, _i32, _u32, _vp, _vp]),
    "kr_jacobian_workspace_bytes": (_size_t, [_i32, _i32, _i32]),
    "kr_jacobian": (_i32, [_vp, _i32, _vp, _i32, _vp, _i32, _u32, _vp, _vp, _vp, _size_t, _vp]),
    "kr_misfit_gradient_workspace_bytes": (_size_t, [_i32, _i32, _i32]),
    "kr_misfit_gradient": (_i32, [_vp, _i32, _vp, _i32, _vp, _i32, _u32, _vp, _vp, _vp, _vp,
                                  _size_t, _vp]),
    "kr_vjp_workspace_bytes": (_size_t, [_i32, _i32, _i32]),
    "kr_vjp": (_i32, [_vp, _i32, _vp, _i32, _vp, _i32, _u32, _vp, _vp, _vp, _vp, _size_t, _vp]),
    "kr_misfit_hvp_workspace_bytes": (_size_t, [_i32, _i32, _i32, _i32]),
    "kr_misfit_hvp": (_i32, [_vp, _i32, _vp, _i32, _vp, _i32, _u32, _vp, _vp, _i32, _vp, _vp,
                             _size_t, _vp]),
    "kr_jacobian_dot_workspace_bytes": (_size_t, [_i32, _i32, _i32, _i32]),
    "kr_jacobian_dot": (_i32, [_vp, _i32, _vp, _i32, _vp, _i32, _u32, _vp, _i32, _vp, _vp,
                               _size_t, _vp]),
    "kr_bessel_sum_workspace_bytes": (_size_t, [_i32, _i32, _i32]),
    "kr_bessel_sum": (_i32, [_vp, _vp, _vp, _i32, ctypes.c_double, _vp, _i32, _vp, _i32, _vp,
                             _vp, _size_t, _vp]),
    "kr_bessel_sum_noalloc": (_i32, [_vp, _vp, _vp, _i32, ctypes.c_double, _vp, _i32, _vp,
                                     _i32, _vp, _vp]),
    "kr_bessel_sum_noalloc_scratch_bytes": (_size_t, []),
    "kr_traces_workspace_bytes": (_size_t, [_i32, _i32]),
    "kr_traces": (_i32, [_vp, _vp, _i32, _i32, _vp, _vp, _vp, _size_t, _vp]),
    "kr_set_forward_variant": (None, [_i32]),
    "kr_set_deriv_variant": (None, [_i32]),
    "kr_batch_plan_bytes": (_size_t, [_vp, _i32, _vp]),
    "kr_batch_plan": (_i32, [_vp, _i32, _vp, _vp, _size_t, _vp]),
    "kr_batch_plan_meta_bytes": (_size_t, [_vp, _i32, _vp]),
    "kr_batch_plan_host": (_i32, [_vp, _i32, _vp, _vp, _size_t]),
    "kr_batch_launch": (_i32, [_vp, _vp, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    # include/kennett_b200_bench.h
    "kr_bench_fp64_fma": (_i32, [_i32, _i32, _vp, _vp]),
    "kr_bench_fp64_fma_flops": (ctypes.c_double, [_i32, _i32]),
}

_lock = threading.Lock()
_lib = None


class KennettError(RuntimeError):
    """A device-side failure reported by the library (CUDA or cuFFT)."""


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def lib() -> ctypes.CDLL:
    """Load ``libkennett_b200.so`` once; raise ImportError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise ImportError(
                    f"{LIB_PATH.name} is not built; run `python -m seismicinversion_b200.build` "
                    "(the CUDA library is the only compute path)"
                )
            h = ctypes.CDLL(str(LIB_PATH))
            for name, (res, args) in _SIGNATURES.items():
                fn = getattr(h, name)
                fn.restype = res
                fn.argtypes = args
            _lib = h
    return _lib


def check(status: int, what: str) -> None:
    """Map a kr_status to the reference's exception style (ValueError for bad input)."""
    if status == KR_OK:
        return
    h = lib()
    name = h.kr_status_string(status).decode()
    detail = h.kr_last_error().decode()
    msg = f"{what}: {name}" + (f" ({detail})" if detail else "")
    if status in (KR_ERR_INVALID_ARGUMENT, KR_ERR_INVALID_MODEL, KR_ERR_TOO_LARGE,
                  KR_ERR_WORKSPACE):
        raise ValueError(msg)
    raise KennettError(msg)

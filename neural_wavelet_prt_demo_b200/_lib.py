"""ctypes binding of libnwprt.so (include/nwprt.h).

Loading never falls back to anything: if the library is missing or fails to load,
``lib()`` raises.  Every status other than NWPRT_OK becomes an ``NwprtError``
carrying the library's last-error message.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libnwprt.so")

OK, INVALID_ARG, OOM, CUDA_ERROR, TIMEOUT, NOT_READY, IO_ERROR, UNSUPPORTED = range(8)
PREC_FP32, PREC_BF16, PREC_FP8 = 0, 1, 2
MAX_FRAMES = 16

# Every symbol include/nwprt.h declares (checked by the CPU test suite).
EXPORTS = (
    "nwprt_abi_version", "nwprt_status_string", "nwprt_last_error", "nwprt_create", "nwprt_destroy",
    "nwprt_get_network_info", "nwprt_load_weights", "nwprt_load_weights_dir", "nwprt_ready",
    "nwprt_env_from_faces", "nwprt_env_from_wavelets", "nwprt_env_get_wavelets", "nwprt_env_release",
    "nwprt_prepare", "nwprt_relight", "nwprt_relight_batch", "nwprt_relight_ranges",
    "nwprt_calibrate_fp8", "nwprt_get_fp8_calibration", "nwprt_selftest_device_wait", "nwprt_sync",
    "nwprt_haar_topk", "nwprt_env_rotate", "nwprt_tonemap_srgb", "nwprt_sh_vertex_radiance",
    "nwprt_sh_interpolate",
    "nwprt_sh_project_workspace_size", "nwprt_sh_project", "nwprt_sh_project_static", "nwprt_sh_dot",
)


class NwprtError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class GBuffer(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int),
                ("first_hit_pos", C.c_void_p), ("world_normal", C.c_void_p),
                ("reflect_dir", C.c_void_p), ("roughness", C.c_void_p), ("kd", C.c_void_p),
                ("ks", C.c_void_p), ("direct", C.c_void_p), ("env_map_flag", C.c_void_p)]


class RelightOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("clamp_terms", C.c_int), ("kahan", C.c_int)]


class Weights(C.Structure):
    _fields_ = [("hash_params", C.c_void_p), ("n_hash_params", C.c_size_t),
                ("out_prd", C.c_void_p), ("n_out_prd", C.c_size_t),
                ("cmp_net", C.c_void_p), ("n_cmp_net", C.c_size_t),
                ("wve_enc", C.c_void_p), ("n_wve_enc", C.c_size_t)]


class NetworkInfo(C.Structure):
    _fields_ = [("enc_dims", C.c_int), ("n_coeffs", C.c_int), ("face_size", C.c_int),
                ("aux_width", C.c_int), ("n_hash_params", C.c_size_t), ("n_out_prd", C.c_size_t),
                ("n_cmp_net", C.c_size_t), ("n_wve_enc", C.c_size_t), ("flops_per_eval", C.c_double)]


class Request(C.Structure):
    _fields_ = [("env_id", C.c_int), ("frame_id", C.c_int), ("indirect", C.c_void_p),
                ("with_direct", C.c_void_p)]


class RangeRequest(C.Structure):
    _fields_ = [("env_id", C.c_int), ("frame_id", C.c_int), ("indirect", C.c_void_p),
                ("with_direct", C.c_void_p), ("px_begin", C.c_int64), ("px_end", C.c_int64)]


_LIB = None
_vp, _i, _st = C.c_void_p, C.c_int, C.c_int


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with "
                          "`python -m neural_wavelet_prt_demo_b200.build`")
    L = C.CDLL(LIB_PATH)
    sig = {
        "nwprt_abi_version": (_i, []),
        "nwprt_status_string": (C.c_char_p, [_i]),
        "nwprt_last_error": (C.c_char_p, [_vp]),
        "nwprt_create": (_st, [C.c_char_p, _i, C.POINTER(_vp)]),
        "nwprt_destroy": (None, [_vp]),
        "nwprt_get_network_info": (_st, [_vp, C.POINTER(NetworkInfo)]),
        "nwprt_load_weights": (_st, [_vp, C.POINTER(Weights)]),
        "nwprt_load_weights_dir": (_st, [_vp, C.c_char_p]),
        "nwprt_ready": (_i, [_vp]),
        "nwprt_env_from_faces": (_st, [_vp, _vp, _i, _i, _i, _vp, C.POINTER(_i)]),
        "nwprt_env_from_wavelets": (_st, [_vp, _vp, _vp, _i, _i, _vp, C.POINTER(_i)]),
        "nwprt_env_get_wavelets": (_st, [_vp, _i, _vp, _vp, _i, C.POINTER(_i)]),
        "nwprt_env_release": (_st, [_vp, _i]),
        "nwprt_prepare": (_st, [_vp, _i, C.POINTER(GBuffer), _vp]),
        "nwprt_relight": (_st, [_vp, _i, _i, C.POINTER(RelightOpts), _vp, _vp, _vp]),
        "nwprt_relight_batch": (_st, [_vp, C.POINTER(Request), _i, C.POINTER(RelightOpts), _vp]),
        "nwprt_relight_ranges": (_st, [_vp, C.POINTER(RangeRequest), _i, C.POINTER(RelightOpts), _vp]),
        "nwprt_calibrate_fp8": (_st, [_vp, _i, _i, C.c_int64, C.c_int64, _vp]),
        "nwprt_get_fp8_calibration": (_st, [_vp, C.POINTER(C.c_float), _i, C.POINTER(_i)]),
        "nwprt_selftest_device_wait": (_st, [_vp, _i, _vp]),
        "nwprt_sync": (_st, [_vp]),
        "nwprt_env_rotate": (_st, [_vp, _i, _vp, _vp, _vp]),
        "nwprt_tonemap_srgb": (_st, [_vp, C.c_int64, _vp, _vp]),
        "nwprt_sh_vertex_radiance": (_st, [_vp, _vp, _vp, C.c_int64, _i, _vp, _vp]),
        "nwprt_sh_interpolate": (_st, [_vp, _vp, C.c_int64, _vp, _vp, C.c_int64, _vp, _vp]),
        "nwprt_haar_topk": (_st, [_vp, _i, _i, _i, _vp, _vp, _vp]),
        "nwprt_sh_project_workspace_size": (C.c_size_t, [_i]),
        "nwprt_sh_project": (_st, [_vp, _i, _vp, _vp, C.c_size_t, _vp]),
        "nwprt_sh_project_static": (_st, [_vp, _i, _vp, _vp]),
        "nwprt_sh_dot": (_st, [_vp, C.c_int64, _i, _vp, _i, _vp, _vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def check(status: int, ctx=None):
    if status != OK:
        msg = lib().nwprt_last_error(ctx)
        raise NwprtError(status, (msg or b"").decode(errors="replace"))

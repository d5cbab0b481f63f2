"""ctypes driver for the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg,
never by the product package.  ``liboracle.so`` is built by oracle/Makefile;
``_ref/libref_utils.so`` (the reference's own utils_kernels.h compiled for the
host) is optional and only present where the reference tree was available.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

MAX_LEVELS = 32
MAX_LAYERS = 16


class OrcNet(C.Structure):
    _fields_ = [
        ("n_levels", C.c_int), ("n_features", C.c_int),
        ("level_res", C.c_int * MAX_LEVELS), ("level_size", C.c_int * MAX_LEVELS),
        ("level_offset", C.c_int * MAX_LEVELS),
        ("aux_width", C.c_int),
        ("op_nl", C.c_int), ("op_in", C.c_int * MAX_LAYERS), ("op_out", C.c_int * MAX_LAYERS),
        ("cn_nl", C.c_int), ("cn_in", C.c_int * MAX_LAYERS), ("cn_out", C.c_int * MAX_LAYERS),
        ("n_coeffs", C.c_int),
    ]


class OrcWeights(C.Structure):
    _fields_ = [("hash", C.c_void_p), ("op", C.c_void_p), ("cn", C.c_void_p), ("emb", C.c_void_p)]


class OrcGbuf(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int),
                ("pos", C.c_void_p), ("normal", C.c_void_p), ("reflect", C.c_void_p),
                ("roughness", C.c_void_p), ("kd", C.c_void_p), ("ks", C.c_void_p),
                ("direct", C.c_void_p), ("flag", C.c_void_p)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        _LIB.orc_wavelet_key.restype = C.c_float
        _LIB.orc_wavelet_key.argtypes = [C.c_float] * 3
    return _LIB


def ref_lib():
    """The reference's utils_kernels.h built for the host, or None if not built."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libref_utils.so")
        if not os.path.exists(path):
            return None
        _REF = C.CDLL(path)
    return _REF


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else C.c_void_p(0)


def net_struct(desc) -> OrcNet:
    n = OrcNet()
    n.n_levels = desc.n_levels
    n.n_features = desc.n_features
    for l in range(desc.n_levels):
        n.level_res[l] = desc.level_res[l]
        n.level_size[l] = desc.level_size[l]
        n.level_offset[l] = desc.level_offset[l]
    n.aux_width = desc.aux_width
    ops, cns = desc.op_layers(), desc.cn_layers()
    n.op_nl = len(ops)
    for i, (a, b) in enumerate(ops):
        n.op_in[i], n.op_out[i] = a, b
    n.cn_nl = len(cns)
    for i, (a, b) in enumerate(cns):
        n.cn_in[i], n.cn_out[i] = a, b
    n.n_coeffs = desc.n_coeffs
    return n


class Bound:
    """Keeps numpy arrays alive while the C structs point at them."""

    def __init__(self, desc, weights, gbuf=None):
        self.desc = desc
        self.keep = []
        self.net = net_struct(desc)
        w = [np.ascontiguousarray(a, np.float32) for a in
             (weights.hash_params, weights.out_prd, weights.cmp_net, weights.wve_enc)]
        self.keep += w
        self.w = OrcWeights(*[_p(a) for a in w])
        self.g = None
        if gbuf is not None:
            self.set_gbuf(gbuf)

    def set_gbuf(self, gb):
        arrs = [np.ascontiguousarray(a) for a in gb.arrays()]
        self.keep += arrs
        self.g = OrcGbuf(gb.width, gb.height, *[_p(a) for a in arrs])
        self.n_px = gb.width * gb.height


def wavelet_key(r, g, b) -> float:
    return lib().orc_wavelet_key(r, g, b)


def haar_face(face: np.ndarray) -> np.ndarray:
    f = np.ascontiguousarray(face, np.float32).copy()
    lib().orc_haar_face(_p(f), C.c_int(f.shape[0]))
    return f


def haar_inverse_f64(coeffs: np.ndarray) -> np.ndarray:
    f = np.ascontiguousarray(coeffs, np.float64).copy()
    lib().orc_haar_inverse_face_f64(_p(f), C.c_int(f.shape[0]))
    return f


def haar_topk(faces: np.ndarray, K: int, n_threads: int = 0):
    """faces [6,S,S,3] or [E,6,S,S,3] -> (idx int32 [..,K], strength f32 [..,K,3])."""
    f = np.ascontiguousarray(faces, np.float32)
    batched = f.ndim == 5
    if not batched:
        f = f[None]
    E, S = f.shape[0], f.shape[2]
    idx = np.empty((E, K), np.int32)
    st = np.empty((E, K, 3), np.float32)
    rc = lib().orc_haar_topk_batch(_p(f), C.c_int(E), C.c_int(S), C.c_int(K), _p(idx), _p(st),
                                   C.c_int(n_threads))
    if rc != 0:
        raise ValueError("orc_haar_topk rejected the arguments")
    return (idx, st) if batched else (idx[0], st[0])


def env_rotate(faces: np.ndarray, R: np.ndarray) -> np.ndarray:
    f = np.ascontiguousarray(faces, np.float32)
    r = np.ascontiguousarray(np.asarray(R, np.float32).reshape(9))
    out = np.empty_like(f)
    lib().orc_env_rotate(_p(f), C.c_int(f.shape[1]), _p(r), _p(out))
    return out


def powf_series(x, y) -> np.ndarray:
    """Elementwise float x^y by the oracle's series (the arithmetic of the final-colour pass)."""
    xs = np.ascontiguousarray(x, np.float32).ravel()
    f = lib().orc_powf_series
    f.restype = C.c_float
    f.argtypes = [C.c_float, C.c_float]
    return np.array([f(float(v), float(y)) for v in xs], np.float32).reshape(np.shape(x))


def tonemap_srgb(src: np.ndarray) -> np.ndarray:
    """float4 [n, 4] linear radiance -> uint32 [n] RGBA8 (Renderer/toneMap.cu:47-71)."""
    s = np.ascontiguousarray(src, np.float32).reshape(-1, 4)
    out = np.empty(s.shape[0], np.uint32)
    lib().orc_tonemap_srgb(_p(s), C.c_int64(s.shape[0]), _p(out))
    return out


def srgb_thresholds() -> np.ndarray:
    t = np.empty(256, np.float32)
    lib().orc_srgb_thresholds(_p(t))
    return t


def srgb_threshold_mismatches(t: np.ndarray, radius: int) -> int:
    f = lib().orc_srgb_threshold_mismatches
    f.restype = C.c_int64
    return int(f(_p(np.ascontiguousarray(t, np.float32)), C.c_int(radius)))


def sh_vertex_radiance(T: np.ndarray, brdf: np.ndarray, L: np.ndarray) -> np.ndarray:
    """T [V, n, n], brdf [V, n, 3], L [n, 3] -> |sum_k (T L)[k] * brdf[k]| [V, 3]."""
    T = np.ascontiguousarray(T, np.float32)
    brdf = np.ascontiguousarray(brdf, np.float32)
    L = np.ascontiguousarray(L, np.float32)
    V, n = T.shape[0], T.shape[1]
    out = np.empty((V, 3), np.float32)
    lib().orc_sh_vertex_radiance(_p(T), _p(brdf), _p(L), C.c_int64(V), C.c_int(n), _p(out))
    return out


def sh_interpolate(vc: np.ndarray, tri: np.ndarray, uv: np.ndarray):
    """Vertex colours [V, 3], triangles [P, 3] int32, barycentrics [P, 2] -> ([P, 4], n_bad)."""
    vc = np.ascontiguousarray(vc, np.float32)
    tri = np.ascontiguousarray(tri, np.int32)
    uv = np.ascontiguousarray(uv, np.float32)
    out = np.empty((tri.shape[0], 4), np.float32)
    f = lib().orc_sh_interpolate
    f.restype = C.c_int64
    bad = f(_p(vc), C.c_int64(vc.shape[0]), _p(tri), _p(uv), C.c_int64(tri.shape[0]), _p(out))
    return out, int(bad)


def sh_eval_f64(d, lmax=8) -> np.ndarray:
    out = np.zeros((lmax + 1) ** 2, np.float64)
    lib().orc_sh_eval_f64(C.c_double(d[0]), C.c_double(d[1]), C.c_double(d[2]), C.c_int(lmax),
                          _p(out))
    return out


def sh_project_f64(faces: np.ndarray, lmax=8):
    f = np.ascontiguousarray(faces, np.float32)
    nc = (lmax + 1) ** 2
    L = np.zeros((nc, 3), np.float64)
    La = np.zeros((nc, 3), np.float64)
    lib().orc_sh_project_f64(_p(f), C.c_int(f.shape[1]), C.c_int(lmax), _p(L), _p(La))
    return L, La


def sh_dot_f32(T: np.ndarray, L: np.ndarray, abs_out=True, n_threads=0) -> np.ndarray:
    T = np.ascontiguousarray(T, np.float32)
    L = np.ascontiguousarray(L, np.float32)
    out = np.empty((T.shape[0], 4), np.float32)
    lib().orc_sh_dot_f32(_p(T), C.c_int64(T.shape[0]), C.c_int(T.shape[1]), _p(L),
                         C.c_int(int(abs_out)), _p(out), C.c_int(n_threads))
    return out


def sh_dot_f64(T: np.ndarray, L: np.ndarray, abs_out=True) -> np.ndarray:
    T = np.ascontiguousarray(T, np.float32)
    L = np.ascontiguousarray(L, np.float64)
    out = np.empty((T.shape[0], 3), np.float64)
    lib().orc_sh_dot_f64(_p(T), C.c_int64(T.shape[0]), C.c_int(T.shape[1]), _p(L),
                         C.c_int(int(abs_out)), _p(out))
    return out


def remap_f32(b: Bound, px: int) -> np.ndarray:
    row = np.empty(16, np.float32)
    lib().orc_remap_f32(C.byref(b.g), C.c_int64(px), _p(row))
    return row


def hash_encode_f32(b: Bound, pos) -> np.ndarray:
    p = np.ascontiguousarray(pos, np.float32)
    out = np.empty(b.desc.enc_dims, np.float32)
    lib().orc_hash_encode_f32(C.byref(b.net), C.c_void_p(b.w.hash), _p(p), _p(out))
    return out


def hash_encode_f64(b: Bound, pos) -> np.ndarray:
    p = np.ascontiguousarray(pos, np.float32)
    out = np.empty(b.desc.enc_dims, np.float64)
    lib().orc_hash_encode_f64(C.byref(b.net), C.c_void_p(b.w.hash), _p(p), _p(out))
    return out


def transport(b: Bound, px: int, idx: np.ndarray, f64=False) -> np.ndarray:
    idx = np.ascontiguousarray(idx, np.int32)
    K = idx.shape[0]
    out = np.empty((K, 3), np.float64 if f64 else np.float32)
    fn = lib().orc_transport_f64 if f64 else lib().orc_transport_f32
    rc = fn(C.byref(b.net), C.byref(b.w), C.byref(b.g), C.c_int64(px), _p(idx), C.c_int(K), _p(out))
    if rc != 0:
        raise ValueError("unsupported network for the oracle")
    return out


def relight_f32(b: Bound, idx, strength, clamp=True, kahan=True, px_begin=0, px_end=None,
                n_threads=0):
    idx = np.ascontiguousarray(idx, np.int32)
    st = np.ascontiguousarray(strength, np.float32)
    K = idx.shape[0]
    px_end = b.n_px if px_end is None else px_end
    ind = np.zeros((b.n_px, 4), np.float32)
    wd = np.zeros((b.n_px, 4), np.float32)
    rc = lib().orc_relight_f32(C.byref(b.net), C.byref(b.w), C.byref(b.g), _p(idx), _p(st),
                               C.c_int(K), C.c_int(int(clamp)), C.c_int(int(kahan)),
                               C.c_int64(px_begin), C.c_int64(px_end), C.c_int(n_threads),
                               _p(ind), _p(wd))
    if rc != 0:
        raise ValueError("orc_relight_f32 failed")
    return ind, wd


def relight_rows_f32(b: Bound, rows, idx, strength, px_begin, clamp=True, kahan=True, n_threads=0):
    """relight_f32 over pixels [px_begin, px_begin + len(rows)) with the 16-float input rows
    given (e.g. the reference's own waveletDataCopy rows) instead of remapped here."""
    rows = np.ascontiguousarray(rows, np.float32).reshape(-1, 16)
    idx = np.ascontiguousarray(idx, np.int32)
    st = np.ascontiguousarray(strength, np.float32)
    K = idx.shape[0]
    px_end = px_begin + rows.shape[0]
    ind = np.zeros((b.n_px, 4), np.float32)
    wd = np.zeros((b.n_px, 4), np.float32)
    rc = lib().orc_relight_rows_f32(C.byref(b.net), C.byref(b.w), C.byref(b.g), _p(rows), _p(idx),
                                    _p(st), C.c_int(K), C.c_int(int(clamp)), C.c_int(int(kahan)),
                                    C.c_int64(px_begin), C.c_int64(px_end), C.c_int(n_threads),
                                    _p(ind), _p(wd))
    if rc != 0:
        raise ValueError("orc_relight_rows_f32 failed")
    return ind, wd


def relight_f64(b: Bound, idx, strength, clamp=True, px_begin=0, px_end=None, n_threads=0):
    idx = np.ascontiguousarray(idx, np.int32)
    st = np.ascontiguousarray(strength, np.float32)
    K = idx.shape[0]
    px_end = b.n_px if px_end is None else px_end
    rgb = np.zeros((px_end - px_begin, 3), np.float64)
    rc = lib().orc_relight_f64(C.byref(b.net), C.byref(b.w), C.byref(b.g), _p(idx), _p(st),
                               C.c_int(K), C.c_int(int(clamp)), C.c_int64(px_begin),
                               C.c_int64(px_end), C.c_int(n_threads), _p(rgb))
    if rc != 0:
        raise ValueError("orc_relight_f64 failed")
    return rgb


def max_threads() -> int:
    return lib().orc_max_threads()


# ---------------------------------------------------------------- reference kernels (host)

def ref_wavelet_data_copy(gb):
    """prt::waveletDataCopy of the reference (host build): [N, WAVELETNUM, 16] rows."""
    r = ref_lib()
    n = gb.width * gb.height
    K = r.ref_wavelet_num()
    out = np.empty((n * K, 16), np.float32)
    arrs = [np.ascontiguousarray(a) for a in (gb.pos, gb.normal, gb.reflect, gb.roughness,
                                              gb.kd, gb.ks)]
    r.ref_wavelet_data_copy(C.c_int(gb.width), C.c_int(gb.height), *[_p(a) for a in arrs], _p(out))
    return out.reshape(n, K, 16)


def ref_compute_response(gb, response, light):
    """response [N, 64, 3], light [64, 3] -> (indirect [N,4], with_direct [N,4])."""
    r = ref_lib()
    n = gb.width * gb.height
    resp = np.ascontiguousarray(response, np.float32)
    li = np.ascontiguousarray(light, np.float32)
    ind = np.empty((n, 4), np.float32)
    wd = np.empty((n, 4), np.float32)
    r.ref_compute_response(C.c_int(gb.width), C.c_int(gb.height), _p(resp),
                           _p(np.ascontiguousarray(gb.direct)), _p(li),
                           _p(np.ascontiguousarray(gb.flag)), _p(ind), _p(wd))
    return ind, wd


def ref_ptwise_mlt(enc_fm, emb, coefs):
    """enc_fm [D, batch] feature-major; emb [D * 24576]; coefs [64] -> out [D, batch]."""
    r = ref_lib()
    enc = np.ascontiguousarray(enc_fm, np.float32)
    out = np.empty_like(enc)
    D, batch = enc.shape
    r.ref_ptwise_mlt(C.c_uint32(D * batch), C.c_uint32(batch), _p(enc),
                     _p(np.ascontiguousarray(emb, np.float32)),
                     _p(np.ascontiguousarray(coefs, np.int32)), _p(out))
    return out

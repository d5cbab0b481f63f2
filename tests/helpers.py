"""Shared case builders and error metrics for the test suite."""
from dataclasses import dataclass

import numpy as np

from neural_wavelet_prt_demo_b200 import netconfig, synth
from oracle import oracle as O


@dataclass
class Case:
    desc: object
    cfg: dict
    weights: object
    gbuf: object
    faces: np.ndarray
    idx: np.ndarray
    strength: np.ndarray
    bound: object


def make_case(cfg, width, height, K, seed=0, hash_scale=1e-4, flag_prob=1.0, param_round="fp32"):
    desc = netconfig.parse(cfg)
    w = synth.make_weights(desc, seed=seed, hash_scale=hash_scale, param_round=param_round)
    gb = synth.make_gbuffer(width, height, seed=seed + 1, flag_prob=flag_prob)
    faces = synth.make_env_faces(desc.face_size, seed=seed + 2)
    idx, st = O.haar_topk(faces, K)
    return Case(desc, cfg, w, gb, faces, idx, st, O.Bound(desc, w, gb))


def rel_err(x, ref, floor_frac=1e-6):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    floor = max(floor_frac * float(np.abs(ref).max()), 1e-30)
    e = np.abs(x - ref) / np.maximum(np.abs(ref), floor)
    return float(e.max()), float(e.mean())


def psnr(x, ref):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    mse = float(np.mean((x - ref) ** 2))
    peak = float(np.abs(ref).max())
    if mse == 0:
        return float("inf")
    return 10.0 * np.log10(peak * peak / mse)


def bits_equal(a, b) -> bool:
    """Bitwise float32 equality, except that any NaN equals any NaN (x86 and the GPU
    produce different NaN payloads for the same invalid operation)."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return False
    return bool(np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32)))


def err_stats(x, ref, floor_frac=1e-6) -> dict:
    """Error of an image against its reference, as every accuracy report states it:
    max / mean relative error with denominators floored at ``floor_frac`` of the image
    maximum, PSNR over the image maximum, and the largest absolute error as a fraction of
    that maximum (the per-pixel bound that near-zero channels do not inflate)."""
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    mx, mean = rel_err(x, ref, floor_frac)
    peak = float(np.abs(ref).max())
    return {"max_rel_err": mx, "mean_rel_err": mean, "psnr_db": psnr(x, ref),
            "max_abs_err_over_peak": float(np.abs(x - ref).max()) / peak if peak > 0 else 0.0}


def load_golden(name):
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name + ".npz")
    return dict(np.load(path))


def rgbe_encode(img):
    """float [h, w, 3] -> RGBE bytes [h, w, 4]: exponent from the largest channel, mantissas
    truncated (integers below 256 are stored exactly)."""
    img = np.asarray(img, np.float64)
    m = img.max(axis=-1)
    frac, e = np.frexp(m)
    live = m > 1e-38
    scale = np.ldexp(1.0, np.where(live, 8 - e, 0))
    mant = np.where(live[..., None], np.clip(np.floor(img * scale[..., None]), 0, 255), 0)
    expo = np.where(live, e + 128, 0)
    return np.concatenate([mant, expo[..., None]], axis=-1).astype(np.uint8)


def write_hdr(path, img, rle=True):
    """Radiance .hdr writer: run-length encoded scanlines (runs of >= 3 equal bytes, else
    literal dumps) or flat RGBE quadruples."""
    h, w, _ = np.asarray(img).shape
    px = rgbe_encode(img)
    out = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {h} +X {w}\n".encode())
    for y in range(h):
        if not rle:
            out += px[y].tobytes()
            continue
        out += bytes([2, 2, w >> 8, w & 255])
        for c in range(4):
            comp = px[y, :, c]
            x = 0
            while x < w:
                n = 1
                while x + n < w and comp[x + n] == comp[x] and n < 127:
                    n += 1
                if n >= 3:
                    out += bytes([128 + n, comp[x]])
                    x += n
                else:
                    m = 1
                    while (x + m < w and m < 128
                           and not (x + m + 2 < w and comp[x + m] == comp[x + m + 1] == comp[x + m + 2])):
                        m += 1
                    out += bytes([m]) + comp[x:x + m].tobytes()
                    x += m
    with open(path, "wb") as f:
        f.write(bytes(out))

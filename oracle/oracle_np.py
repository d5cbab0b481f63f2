"""numpy twin of the C oracle -- TEST INFRASTRUCTURE ONLY.

An independent, vectorised restatement of the same definitions as
oracle/nwprt_oracle.c, used to cross-check the C oracle on small cases
(FP32 Haar / keys bit for bit, FP64 relight to ~1e-12).  Sources followed:
Renderer/tinycudann/utils_kernels.h:7-127 (remap, embedding gather, clamped sum),
Renderer/tinycudann/prt_network.h:73-154 (network composition),
Renderer/EnvironmentMap.cpp:149-151 (luminance weights).
"""
from __future__ import annotations

import numpy as np

LUM = (np.float32(0.212671), np.float32(0.715160), np.float32(0.072169))


def haar_face(face: np.ndarray) -> np.ndarray:
    """FP32 non-standard 2-D Haar, Mallat layout (same arithmetic as the C oracle)."""
    f = np.array(face, np.float32, copy=True)
    S = f.shape[0]
    n = S
    half = np.float32(0.5)
    while n >= 2:
        h = n // 2
        blk = f[:n, :n]
        a, b = blk[0::2, 0::2], blk[0::2, 1::2]
        c, d = blk[1::2, 0::2], blk[1::2, 1::2]
        s0, d0, s1, d1 = a + b, a - b, c + d, c - d
        out = np.empty_like(blk)
        out[:h, :h] = (s0 + s1) * half
        out[:h, h:] = (d0 + d1) * half
        out[h:, :h] = (s0 - s1) * half
        out[h:, h:] = (d0 - d1) * half
        f[:n, :n] = out
        n = h
    return f


def keys(coeffs: np.ndarray) -> np.ndarray:
    r, g, b = coeffs[..., 0], coeffs[..., 1], coeffs[..., 2]
    t = LUM[0] * r
    t = t + LUM[1] * g
    t = t + LUM[2] * b
    t = np.abs(t).astype(np.float32)
    t[np.isnan(t)] = 0
    return t


def haar_topk(faces: np.ndarray, K: int):
    S = faces.shape[1]
    c = np.stack([haar_face(faces[f]) for f in range(6)]).reshape(6 * S * S, 3)
    k = keys(c)
    order = np.lexsort((np.arange(k.size), -k.astype(np.float64)))
    sel = order[:K]
    return sel.astype(np.int32), c[sel]


def hash_encode_f64(desc, hash_params, pos):
    """pos [N,3] float32 -> [N, L*F] float64 (Instant-NGP encoding as pinned in netconfig)."""
    pos = np.clip(np.asarray(pos, np.float32), np.float32(0), np.float32(1))
    N = pos.shape[0]
    F = desc.n_features
    hp = np.asarray(hash_params, np.float32).reshape(-1, F).astype(np.float64)
    out = np.zeros((N, desc.n_levels * F), np.float64)
    for l in range(desc.n_levels):
        R = desc.level_res[l]
        xl = pos * np.float32(R)
        i0 = np.minimum(np.floor(xl).astype(np.int64), R - 1)
        w = (xl - i0.astype(np.float32)).astype(np.float64)
        N1 = R + 1
        T = desc.level_size[l]
        dense = N1 ** 3 <= T
        acc = np.zeros((N, F), np.float64)
        for c in range(8):
            bits = np.array([(c >> 0) & 1, (c >> 1) & 1, (c >> 2) & 1])
            ijk = (i0 + bits).astype(np.uint64)
            wc = np.prod(np.where(bits == 1, w, 1.0 - w), axis=1)
            if dense:
                e = ijk[:, 0] + ijk[:, 1] * N1 + ijk[:, 2] * N1 * N1
            else:
                m = np.uint64(0xFFFFFFFF)
                h = (ijk[:, 0] ^ ((ijk[:, 1] * np.uint64(2654435761)) & m)
                     ^ ((ijk[:, 2] * np.uint64(805459861)) & m)) & m
                e = h & np.uint64(T - 1)
            acc += wc[:, None] * hp[desc.level_offset[l] + e.astype(np.int64)]
        out[:, l * F:(l + 1) * F] = acc
    return out


def _layers(flat, shapes):
    mats, o = [], 0
    for n_in, n_out in shapes:
        mats.append(np.asarray(flat[o:o + n_in * n_out], np.float64).reshape(n_out, n_in))
        o += n_in * n_out
    return mats


def remap_f64(gb):
    n = gb.width * gb.height
    row = np.zeros((n, 16), np.float64)
    row[:, 0:3] = gb.pos[:, :3]
    row[:, 3:6] = gb.normal[:, :3]
    row[:, 6:9] = gb.reflect[:, :3]
    row[:, 9] = np.log(25.0 * gb.roughness.astype(np.float64) + 1.0) / np.log(26.0)
    row[:, 10:13] = 2.0 * gb.kd[:, :3].astype(np.float64) - 1.0
    row[:, 13:16] = 2.0 * gb.ks[:, :3].astype(np.float64) - 1.0
    return row


def relight_f64(desc, w, gb, idx, strength, clamp=True):
    """Full relight in FP64 -> rgb [N,3] (indirect only; flagged pixels)."""
    row = remap_f64(gb)
    enc = hash_encode_f64(desc, w.hash_params, gb.pos[:, :3])
    n = row.shape[0]
    K = len(idx)
    E = np.asarray(w.wve_enc, np.float64)[:, np.asarray(idx)]          # [D, K]
    x = enc[:, None, :] * E.T[None, :, :]                              # [N, K, D]
    ops = _layers(w.out_prd, desc.op_layers())
    for li, M in enumerate(ops):
        x = x @ M.T
        if li < len(ops) - 1:
            x = np.maximum(x, 0.0)
    aux = np.ones((n, desc.aux_width), np.float64)
    aux[:, :13] = row[:, 3:16]
    x = np.concatenate([x, np.broadcast_to(aux[:, None, :], (n, K, desc.aux_width))], axis=2)
    cns = _layers(w.cmp_net, desc.cn_layers())
    for li, M in enumerate(cns):
        x = x @ M.T
        if li < len(cns) - 1:
            x = np.maximum(x, 0.0)
    terms = np.asarray(strength, np.float64)[None] * x                 # [N, K, 3]
    if clamp:
        terms = np.maximum(terms, 0.0)
    rgb = terms.sum(axis=1)
    rgb[gb.flag == 0] = 0.0
    return rgb

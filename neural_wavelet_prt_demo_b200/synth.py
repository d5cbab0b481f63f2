"""Seeded synthetic inputs: weights, environment maps and G-buffers.

The reference's trained weights, env maps and scenes are external downloads
(README.MD:37-38), so every workload here is synthetic.  Each tensor draws from
its own numpy PCG64 stream keyed by (seed, stream id), so any tensor can be
regenerated alone and all consumers (GPU path, oracle, fixtures) see the same
bytes.

G-buffer encodings follow the reference's OptiX camera program
(Renderer/device_functions/camera.cu:248-270): position bbox-normalised to
[0,1]^3, world normal and reflection direction stored as v/2+0.5, kd/ks raw,
roughness raw; reflection = reflect(-view, n) (devicePrograms.cu:303).
All float4 buffers carry w = 1 as the reference writes them.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .netconfig import NetDesc

# stream ids (stable: changing them changes every fixture)
_S_HASH, _S_OP, _S_CN, _S_EMB = 1, 2, 3, 4
_S_POS, _S_NRM, _S_VIEW, _S_KD, _S_KS, _S_RGH, _S_DIR, _S_FLAG = 10, 11, 12, 13, 14, 15, 16, 17
_S_ENV = 30
_S_SHT = 40
_S_TMAT, _S_BRDF, _S_TRI, _S_UV = 41, 42, 43, 44


def rng(seed: int, stream: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64([int(seed), int(stream)]))


@dataclass
class Weights:
    hash_params: np.ndarray   # f32 [sum T_l * F]
    out_prd: np.ndarray       # f32, concatenated row-major [out][in] layers
    cmp_net: np.ndarray       # f32
    wve_enc: np.ndarray       # f32 [D][n_coeffs] dimension-major


def _xavier(g, shapes, dtype_round):
    parts = []
    for n_in, n_out in shapes:
        a = np.sqrt(6.0 / (n_in + n_out))
        parts.append(g.uniform(-a, a, size=(n_out, n_in)).astype(np.float32).ravel())
    w = np.concatenate(parts)
    return _round(w, dtype_round)


def _round(x, dtype_round):
    if dtype_round == "fp16":
        return x.astype(np.float16).astype(np.float32)
    return x.astype(np.float32)


def make_weights(desc: NetDesc, seed: int = 0, hash_scale: float = 1e-4,
                 emb_std: float = 0.1, param_round: str = "fp32") -> Weights:
    """Random-init weights of the given architecture.

    hash params U(-hash_scale, hash_scale) (1e-4 is Instant-NGP's init), embedding
    N(0, emb_std), MLP layers Xavier-uniform.  ``param_round="fp16"`` rounds every
    parameter to the nearest fp16 value (the 1080p config's "FP16 params").
    """
    hp = rng(seed, _S_HASH).uniform(-hash_scale, hash_scale, size=desc.n_hash_params)
    hp = _round(hp.astype(np.float32), param_round)
    op = _xavier(rng(seed, _S_OP), desc.op_layers(), param_round)
    cn = _xavier(rng(seed, _S_CN), desc.cn_layers(), param_round)
    emb = rng(seed, _S_EMB).normal(0.0, emb_std, size=(desc.enc_dims, desc.n_coeffs))
    emb = _round(emb.astype(np.float32), param_round)
    return Weights(hp, op, cn, np.ascontiguousarray(emb))


def make_env_faces(face_size: int, seed: int = 0, sigma: float = 1.5, index: int = 0) -> np.ndarray:
    """6 x S x S x 3 float32 cubemap with log-normal(0, sigma) radiance.

    Face order +X, -X, +Y, -Y, -Z, +Z and row-major texels as produced by
    Environment_Map::initCubeFaces (EnvironmentMap.cpp:112-126).
    """
    g = rng(seed, _S_ENV + 1000 * index)
    return np.exp(g.normal(0.0, sigma, size=(6, face_size, face_size, 3))).astype(np.float32)


def _unit_sphere(g, n):
    v = g.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v


@dataclass
class GBuffer:
    width: int
    height: int
    pos: np.ndarray       # f32 [N,4]
    normal: np.ndarray    # f32 [N,4]
    reflect: np.ndarray   # f32 [N,4]
    roughness: np.ndarray  # f32 [N]
    kd: np.ndarray        # f32 [N,4]
    ks: np.ndarray        # f32 [N,4]
    direct: np.ndarray    # f32 [N,4]
    flag: np.ndarray      # u8 [N]

    @property
    def n(self):
        return self.width * self.height

    def arrays(self):
        return (self.pos, self.normal, self.reflect, self.roughness, self.kd, self.ks,
                self.direct, self.flag)


def make_gbuffer(width: int, height: int, seed: int = 0, flag_prob: float = 1.0) -> GBuffer:
    n = width * height
    f4 = lambda xyz: np.concatenate([xyz, np.ones((n, 1))], axis=1).astype(np.float32)
    raw = rng(seed, _S_POS).uniform(-1.0, 1.0, size=(n, 3))
    pos = (raw - (-1.0)) / 2.0                      # (p - bbox.lower) / bbox.size, camera.cu:260
    nrm = _unit_sphere(rng(seed, _S_NRM), n)
    view = _unit_sphere(rng(seed, _S_VIEW), n)
    d = -view
    r = d - 2.0 * np.sum(d * nrm, axis=1, keepdims=True) * nrm
    r /= np.linalg.norm(r, axis=1, keepdims=True)
    kd = rng(seed, _S_KD).uniform(0.0, 1.0, size=(n, 3))
    ks = rng(seed, _S_KS).uniform(0.0, 1.0, size=(n, 3))
    rough = rng(seed, _S_RGH).uniform(0.05, 1.0, size=n).astype(np.float32)
    direct = rng(seed, _S_DIR).uniform(0.0, 0.5, size=(n, 3))
    if flag_prob >= 1.0:
        flag = np.ones(n, np.uint8)
    else:
        flag = (rng(seed, _S_FLAG).uniform(size=n) < flag_prob).astype(np.uint8)
    return GBuffer(width, height, f4(pos), f4(nrm / 2 + 0.5), f4(r / 2 + 0.5), rough,
                   f4(kd), f4(ks), f4(direct), flag)


def make_sh_transport(n_px: int, n_coeffs: int = 81, seed: int = 0) -> np.ndarray:
    """Per-pixel SH transport vectors T[N][n_coeffs] ~ N(0,1)/l^2, l = floor(sqrt(j)); l=0 uses 1."""
    g = rng(seed, _S_SHT)
    l = np.floor(np.sqrt(np.arange(n_coeffs))).astype(np.float64)
    l[l == 0] = 1.0
    scale = (1.0 / (l * l)).astype(np.float32)
    out = np.empty((n_px, n_coeffs), np.float32)
    step = 1 << 20
    for s in range(0, n_px, step):
        e = min(n_px, s + step)
        out[s:e] = g.standard_normal(size=(e - s, n_coeffs), dtype=np.float32) * scale
    return out


def make_sh_mesh(n_vertices: int, n_px: int, n_coeffs: int = 81, seed: int = 0):
    """Synthetic inputs of the per-vertex SH path: T [V][n][n] ~ N(0,1)/(l_k l_j) (the SH
    transfer matrix of a diffuse-ish vertex decays with both bands), BRDF SH [V][n][3] ~
    N(0,1)/l_k^2 scaled by a U(0,1) albedo, and for every pixel a random triangle of
    vertices plus barycentrics (u, v) uniform on the triangle."""
    l = np.floor(np.sqrt(np.arange(n_coeffs))).astype(np.float64)
    l[l == 0] = 1.0
    inv = (1.0 / l).astype(np.float32)
    g = rng(seed, _S_TMAT)
    T = np.empty((n_vertices, n_coeffs, n_coeffs), np.float32)
    step = max(1, (1 << 22) // (n_coeffs * n_coeffs))
    for s0 in range(0, n_vertices, step):
        e = min(n_vertices, s0 + step)
        T[s0:e] = g.standard_normal(size=(e - s0, n_coeffs, n_coeffs), dtype=np.float32) * inv[None, :, None] * inv[None, None, :]
    g = rng(seed, _S_BRDF)
    alb = g.uniform(0, 1, size=(n_vertices, 1, 3)).astype(np.float32)
    brdf = g.standard_normal(size=(n_vertices, n_coeffs, 3), dtype=np.float32) * (inv * inv)[None, :, None] * alb
    g = rng(seed, _S_TRI)
    tri = g.integers(0, n_vertices, size=(n_px, 3), dtype=np.int32)
    g = rng(seed, _S_UV)
    a, b = g.uniform(0, 1, size=n_px), g.uniform(0, 1, size=n_px)
    flip = a + b > 1
    a[flip], b[flip] = 1 - a[flip], 1 - b[flip]
    uv = np.stack([a, b], 1).astype(np.float32)
    return T, brdf, tri, uv

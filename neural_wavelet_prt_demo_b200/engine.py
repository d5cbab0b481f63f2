"""Python host mirror of the reference's neural-relight interface over libnwprt.

Names and argument meaning follow the reference so callers and tests read alike:

* ``RenderEngine``   -- ``initTCNN`` / ``TCNNAvaliable`` / ``TCNNPass_p1`` /
  ``TCNNPass_p2`` / ``TCNNSync`` / ``buildLights`` (Renderer/RenderEngine.h:58-83,
  Renderer/tinycudann/tcnn.cu:49-162).
* ``EnvironmentMap`` -- ``faces``, ``topWaveletCoefficients``, ``topWaveletStrength``,
  ``shCoefficients`` (Renderer/EnvironmentMap.h:11-40).
* ``FullFrame``      -- the fullFrameCUDA fields the relight reads and writes
  (Renderer/frames.h:96-214).
* ``RenderConfig``   -- renderConfig (Renderer/RenderEngine.h:29-42) plus the relight
  arithmetic options.

Errors raise (``NwprtError``), as the reference's CUDA_CHECK throws
std::runtime_error (Renderer/optix7.h:27-38).  torch only provides device memory and
streams; every computation runs in libnwprt.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import re
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from ._lib import NwprtError, check, lib
from . import netconfig

__all__ = ["RenderEngine", "EnvironmentMap", "FullFrame", "RenderConfig", "NwprtError",
           "haar_topk", "env_rotate", "sh_project", "sh_dot"]


def _ptr(t: Optional[torch.Tensor]):
    return C.c_void_p(0 if t is None else t.data_ptr())


def _stream_ptr(stream) -> C.c_void_p:
    if stream is None:
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, torch.cuda.Stream):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(int(stream))


@dataclass
class RenderConfig:
    """renderConfig (RenderEngine.h:29-42) fields that matter to the relight, plus
    the arithmetic of the transport MLP."""
    waveletMode: bool = True
    precision: str = "fp32"        # "fp32" (drop-in) | "bf16" | "fp8" (tcgen05; fp8 after calibrateFP8)
    clamp_terms: bool = True       # utils_kernels.h:87-89 max(L*T, 0)
    kahan: bool = True

    def opts(self) -> _lib.RelightOpts:
        prec = {"fp32": _lib.PREC_FP32, "bf16": _lib.PREC_BF16, "fp8": _lib.PREC_FP8}.get(self.precision)
        if prec is None:
            raise ValueError(f"unknown precision {self.precision!r}")
        return _lib.RelightOpts(prec, int(self.clamp_terms), int(self.kahan))


@dataclass
class FullFrame:
    """Device G-buffer + relight outputs of one frame (frames.h:143-183 field names)."""
    width: int
    height: int
    fbFirstHitPos: torch.Tensor
    fbworldNormal: torch.Tensor
    fbFirstHitReflecDir: torch.Tensor
    fbRoughness: torch.Tensor
    fbFirstHitKd: torch.Tensor
    fbFirstHitKs: torch.Tensor
    fbDirectDenoised: torch.Tensor
    fbEnvironmentMapFlag: torch.Tensor
    fbPredictedIndirect: torch.Tensor
    fbPredictedIndirectWithDirect: torch.Tensor
    fbFinalColor: Optional[torch.Tensor] = None   # int32 [n] packed RGBA8, by computeFinalPixelColors

    @staticmethod
    def from_gbuffer(gb, device="cuda:0") -> "FullFrame":
        """From a synth.GBuffer (numpy) -> device tensors, outputs zero-initialised."""
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        n = gb.width * gb.height
        return FullFrame(gb.width, gb.height, t(gb.pos), t(gb.normal), t(gb.reflect), t(gb.roughness),
                         t(gb.kd), t(gb.ks), t(gb.direct), t(gb.flag),
                         torch.zeros((n, 4), dtype=torch.float32, device=device),
                         torch.zeros((n, 4), dtype=torch.float32, device=device))

    def gbuffer_struct(self) -> _lib.GBuffer:
        for name in ("fbFirstHitPos", "fbworldNormal", "fbFirstHitReflecDir", "fbFirstHitKd",
                     "fbFirstHitKs", "fbDirectDenoised"):
            t = getattr(self, name)
            if t.dtype != torch.float32 or not t.is_contiguous() or t.numel() != 4 * self.width * self.height:
                raise ValueError(f"{name} must be a contiguous float32 [N,4] tensor")
        if self.fbRoughness.dtype != torch.float32 or self.fbRoughness.numel() != self.width * self.height:
            raise ValueError("fbRoughness must be float32 [N]")
        if self.fbEnvironmentMapFlag.dtype not in (torch.uint8, torch.bool):
            raise ValueError("fbEnvironmentMapFlag must be uint8 or bool")
        return _lib.GBuffer(self.width, self.height, *[
            _ptr(getattr(self, n)) for n in ("fbFirstHitPos", "fbworldNormal", "fbFirstHitReflecDir",
                                             "fbRoughness", "fbFirstHitKd", "fbFirstHitKs",
                                             "fbDirectDenoised", "fbEnvironmentMapFlag")])


def read_hdr(path: str) -> np.ndarray:
    """Radiance RGBE image -> float32 [h, w, 3], rows in file order (top first).

    "#?RADIANCE" signature, header lines up to an empty line, a "-Y <h> +X <w>" resolution
    line, then h scanlines: run-length encoded per component (marker 2, 2, w // 256, w % 256;
    count > 128 = a run of count - 128 copies, else count literal bytes) or flat RGBE
    quadruples where (1, 1, 1, n) repeats the previous pixel n << shift times.  A channel
    is mantissa / 256 * 2^(E - 128), as the reference converts it (HDRloader.cpp:108-125)."""
    with open(path, "rb") as f:
        data = f.read()
    if not data.startswith(b"#?RADIANCE"):
        raise RuntimeError(f"not a Radiance .hdr file: {path}")
    pos = data.index(b"\n") + 1
    while True:
        end = data.find(b"\n", pos)
        if end < 0:
            raise RuntimeError(f"truncated .hdr header: {path}")
        line, pos = data[pos:end], end + 1
        if not line:
            break
    end = data.find(b"\n", pos)
    m = re.match(rb"-Y (\d+) \+X (\d+)$", data[pos:end] if end >= 0 else b"")
    if not m or int(m.group(1)) < 1 or int(m.group(2)) < 1:
        raise RuntimeError(f"unsupported .hdr resolution line: {path}")
    h, w = int(m.group(1)), int(m.group(2))
    pos = end + 1
    buf = np.frombuffer(data, np.uint8)
    n_buf = buf.shape[0]
    px = np.zeros((h, w, 4), np.uint8)

    def take(n):
        nonlocal pos
        if pos + n > n_buf:
            raise RuntimeError(f"truncated .hdr data: {path}")
        pos += n
        return buf[pos - n:pos]

    for y in range(h):
        q = take(4)
        if 8 <= w <= 0x7FFF and q[0] == 2 and q[1] == 2 and not (q[2] & 0x80):
            if (int(q[2]) << 8 | int(q[3])) != w:
                raise RuntimeError(f".hdr scanline width mismatch: {path}")
            for c in range(4):
                x = 0
                while x < w:
                    n = int(take(1)[0])
                    if n > 128:
                        n -= 128
                        if x + n > w:
                            raise RuntimeError(f".hdr run overflows its scanline: {path}")
                        px[y, x:x + n, c] = take(1)[0]
                    else:
                        if n == 0 or x + n > w:
                            raise RuntimeError(f"bad .hdr dump: {path}")
                        px[y, x:x + n, c] = take(n)
                    x += n
        else:
            x, shift, first = 0, 0, True
            while x < w:
                if not first:
                    q = take(4)
                first = False
                if q[0] == 1 and q[1] == 1 and q[2] == 1:
                    n = int(q[3]) << shift
                    if x == 0 or x + n > w:
                        raise RuntimeError(f"bad .hdr repeat code: {path}")
                    px[y, x:x + n] = px[y, x - 1]
                    x += n
                    shift += 8
                else:
                    px[y, x] = q
                    x += 1
                    shift = 0
    scale = np.ldexp(np.float32(1.0), px[..., 3].astype(np.int32) - 128).astype(np.float32)
    return (px[..., :3].astype(np.float32) / np.float32(256.0)) * scale[..., None]


def _load_sh(path: str) -> np.ndarray:
    """SH coefficients [(l+1)^2, 3] (Environment_Map::load_sh, EnvironmentMap.cpp:70-77)."""
    a = np.load(path)
    if a.ndim != 2 or a.shape[1] != 3:
        raise RuntimeError(f"SH .npy must be [n, 3]: {path}")
    l = int(round(np.sqrt(a.shape[0]))) - 1
    if (l + 1) ** 2 != a.shape[0]:
        raise RuntimeError(f"SH .npy must hold (l+1)^2 rows: {path}")
    return a.astype(np.float32)


class EnvironmentMap:
    """Environment_Map (EnvironmentMap.h:11-40): cubemap faces and their wavelet table.

    ``faces`` is float32 [6, S, S, 3] in the reference face order (+X,-X,+Y,-Y,-Z,+Z).
    The wavelet table either comes from precomputed arrays (the reference's
    waveletcoeffs/ + waveletstrength/ npy pair) or is computed on the GPU by
    ``computeWavelets`` (Haar + top-K).
    """

    def __init__(self, faces: Optional[np.ndarray] = None, top_coefficients=None, top_strength=None,
                 sh_coefficients=None):
        self.faces = None if faces is None else np.ascontiguousarray(faces, np.float32)
        self.topWaveletCoefficients = (None if top_coefficients is None
                                       else np.ascontiguousarray(top_coefficients, np.int32).ravel())
        self.topWaveletStrength = (None if top_strength is None
                                   else np.ascontiguousarray(top_strength, np.float32).reshape(-1, 3))
        self.shCoefficients = None if sh_coefficients is None else np.asarray(sh_coefficients, np.float32)

    @staticmethod
    def cross_to_faces(cross: np.ndarray, from_npy: bool = True) -> np.ndarray:
        """4x3 cross image [3S, 4S, 3], rows as stored in the file (top first) -> faces
        [6, S, S, 3] (EnvironmentMap.cpp:80-126).  The rows are flipped first: the reference
        keeps both .npy crosses (:96-101) and .hdr crosses (HDRLoaderResult::get,
        Renderer/HDRloader.h:21-25) bottom row first.  ``from_npy=False`` takes an image
        that is already bottom row first."""
        img = np.asarray(cross, np.float32)
        if img.ndim != 3 or img.shape[2] != 3:
            raise ValueError("cross image must be [3S, 4S, 3]")
        if from_npy:
            img = img[::-1]
        S = img.shape[0] // 3
        if S < 1 or img.shape[0] != 3 * S or img.shape[1] != 4 * S:
            raise ValueError("cross image must be 3S x 4S")
        # get_submatrix(from_c, from_r, ...) offsets in face units, initCubeFaces order
        cells = [(2, 1), (0, 1), (1, 2), (1, 0), (1, 1), (3, 1)]
        return np.stack([img[r * S:(r + 1) * S, c * S:(c + 1) * S] for c, r in cells]).copy()

    @staticmethod
    def from_file(inFileName: str, sh_coeff: bool = False) -> "EnvironmentMap":
        """Environment_Map(inFileName, sh_coeff) (EnvironmentMap.cpp:10-18): a 4x3 cross
        cubemap in a .hdr or .npy file, or, with ``sh_coeff``, SH coefficients (.npy [n, 3])."""
        if sh_coeff:
            return EnvironmentMap(sh_coefficients=_load_sh(inFileName))
        if not os.path.exists(inFileName):
            raise RuntimeError("Invalid Env map File Name")
        ext = os.path.splitext(inFileName)[1]
        if ext == ".hdr":
            img = read_hdr(inFileName)
        elif ext == ".npy":
            img = np.load(inFileName)
            if img.dtype != np.float32:
                raise RuntimeError(f"{inFileName} must hold float32 data")
        else:
            raise RuntimeError("Unknown type " + ext)
        return EnvironmentMap(EnvironmentMap.cross_to_faces(img))

    @staticmethod
    def from_folder(folder: str, name: str) -> "EnvironmentMap":
        """Environment_Map(envMapFolder, envMapName) (EnvironmentMap.cpp:20-68): cube/<name>.hdr
        (required), then sh/<name>.npy and the waveletcoeffs/<name>.npy +
        waveletstrength/<name>.npy pair when present.  The latlong map feeds the reference's
        direct-light shader only and is not read."""
        if not os.path.isdir(folder):
            raise RuntimeError("Invalid Env map Folder Name, it should not be a file")
        cube = os.path.join(folder, "cube", name + ".hdr")
        if not os.path.exists(cube):
            raise RuntimeError("Invalid Env map File Name")
        em = EnvironmentMap(EnvironmentMap.cross_to_faces(read_hdr(cube)))
        wc = os.path.join(folder, "waveletcoeffs", name + ".npy")
        ws = os.path.join(folder, "waveletstrength", name + ".npy")
        if os.path.exists(wc) and os.path.exists(ws):
            st = np.load(ws)
            if st.ndim != 2 or st.shape[1] != 3:
                raise RuntimeError("waveletstrength must be [K, 3]")
            em.topWaveletCoefficients = np.ascontiguousarray(np.load(wc), np.int32).ravel()
            em.topWaveletStrength = np.ascontiguousarray(st, np.float32)
        sh = os.path.join(folder, "sh", name + ".npy")
        if os.path.exists(sh):
            em.shCoefficients = _load_sh(sh)
        return em

    def computeWavelets(self, K: int, device="cuda:0") -> None:
        """Haar transform + top-K selection on the GPU; fills the two wavelet arrays."""
        f = torch.from_numpy(self.faces).to(device)
        idx, st = haar_topk(f, K)
        self.topWaveletCoefficients = idx.cpu().numpy()
        self.topWaveletStrength = st.cpu().numpy()

    def computeSH(self, device="cuda:0") -> None:
        f = torch.from_numpy(self.faces).to(device)
        self.shCoefficients = sh_project(f).cpu().numpy()


class RenderEngine:
    """The reference RenderEngine's neural-relight surface over one libnwprt context."""

    def __init__(self, config, device: int = 0, debug: bool = False):
        if isinstance(config, dict):
            config = json.dumps(config)
        self.desc = netconfig.parse(config)
        self.device = device
        self.debug = debug
        self._ctx = C.c_void_p()
        check(lib().nwprt_create(config.encode(), device, C.byref(self._ctx)))
        self.fullframeCUDABuffer: List[Optional[FullFrame]] = [None, None]
        self.envIds: List[int] = []
        self.TCNNSetup = False
        self.EnvmapSetup = False

    # ---------------------------------------------------------------- lifetime
    def close(self):
        if self._ctx:
            lib().nwprt_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status):
        check(status, self._ctx)

    # ---------------------------------------------------------------- weights
    def initTCNN(self, modelPath: str) -> None:
        """RenderEngine::initTCNN(modelPath): loads vtx_enc/out_prd/cmp_net/wve_enc .npy."""
        self._check(lib().nwprt_load_weights_dir(self._ctx, modelPath.encode()))
        self.TCNNSetup = True

    def loadWeights(self, w) -> None:
        """Same from in-memory arrays (a synth.Weights)."""
        arrs = [np.ascontiguousarray(a, np.float32).ravel()
                for a in (w.hash_params, w.out_prd, w.cmp_net, w.wve_enc)]
        ws = _lib.Weights(arrs[0].ctypes.data, arrs[0].size, arrs[1].ctypes.data, arrs[1].size,
                          arrs[2].ctypes.data, arrs[2].size, arrs[3].ctypes.data, arrs[3].size)
        self._check(lib().nwprt_load_weights(self._ctx, C.byref(ws)))
        self.TCNNSetup = True

    def TCNNAvaliable(self) -> bool:
        return bool(lib().nwprt_ready(self._ctx))

    def networkInfo(self) -> _lib.NetworkInfo:
        info = _lib.NetworkInfo()
        self._check(lib().nwprt_get_network_info(self._ctx, C.byref(info)))
        return info

    # ---------------------------------------------------------------- env maps
    def addEnvironmentMap(self, env: EnvironmentMap, K: Optional[int] = None, stream=None) -> int:
        """Registers one env map; returns its envMapID.  With K given (or no precomputed
        table) the wavelet table is computed on the GPU from the faces."""
        env_id = C.c_int(-1)
        if K is not None or env.topWaveletCoefficients is None:
            if env.faces is None:
                raise ValueError("env map has neither faces nor a wavelet table")
            K = 64 if K is None else K
            self._check(lib().nwprt_env_from_faces(
                self._ctx, env.faces.ctypes.data_as(C.c_void_p), 0, env.faces.shape[1], int(K),
                _stream_ptr(stream), C.byref(env_id)))
        else:
            idx = np.ascontiguousarray(env.topWaveletCoefficients, np.int32)
            st = np.ascontiguousarray(env.topWaveletStrength, np.float32)
            if st.shape != (idx.size, 3):
                raise ValueError("topWaveletStrength must be [K, 3] matching the coefficients")
            self._check(lib().nwprt_env_from_wavelets(
                self._ctx, idx.ctypes.data_as(C.c_void_p), st.ctypes.data_as(C.c_void_p), idx.size, 0,
                _stream_ptr(stream), C.byref(env_id)))
        self.envIds.append(env_id.value)
        self.EnvmapSetup = True
        return len(self.envIds) - 1

    def buildLights(self, envMaps: List[EnvironmentMap], K: Optional[int] = None) -> None:
        """RenderEngine::buildLights (RenderEngine.cpp:113-175): registers every env map."""
        for e in envMaps:
            self.addEnvironmentMap(e, K)

    def envWavelets(self, envMapID: int):
        env_id = self.envIds[envMapID]
        K = C.c_int(0)
        self._check(lib().nwprt_env_get_wavelets(self._ctx, env_id, None, None, 0, C.byref(K)))
        idx = np.empty(K.value, np.int32)
        st = np.empty((K.value, 3), np.float32)
        self._check(lib().nwprt_env_get_wavelets(self._ctx, env_id, idx.ctypes.data_as(C.c_void_p),
                                                 st.ctypes.data_as(C.c_void_p), K.value, C.byref(K)))
        return idx, st

    # ---------------------------------------------------------------- frames
    def setFrame(self, frameID: int, frame: FullFrame) -> None:
        while len(self.fullframeCUDABuffer) <= frameID:
            self.fullframeCUDABuffer.append(None)
        self.fullframeCUDABuffer[frameID] = frame

    def TCNNPass_p1(self, frameID: int, stream=None) -> None:
        """tcnn.cu:83-108: the frame's G-buffer -> packed per-pixel input rows."""
        f = self.fullframeCUDABuffer[frameID]
        if f is None:
            raise RuntimeError(f"frame {frameID} has no buffers (setFrame first)")
        gb = f.gbuffer_struct()
        self._check(lib().nwprt_prepare(self._ctx, frameID, C.byref(gb), _stream_ptr(stream)))

    def TCNNPass_p2(self, envMapID: int, frameID: int, config: Optional[RenderConfig] = None,
                    stream=None) -> None:
        """tcnn.cu:111-152: relight the prepared frame with env `envMapID` into the frame's
        fbPredictedIndirect / fbPredictedIndirectWithDirect.  Asynchronous."""
        config = config or RenderConfig()
        f = self.fullframeCUDABuffer[frameID]
        opts = config.opts()
        self._check(lib().nwprt_relight(self._ctx, self.envIds[envMapID], frameID, C.byref(opts),
                                        _ptr(f.fbPredictedIndirect), _ptr(f.fbPredictedIndirectWithDirect),
                                        _stream_ptr(stream)))

    def relightBatch(self, requests, config: Optional[RenderConfig] = None, stream=None) -> None:
        """Several (envMapID, frameID, indirect, with_direct) relights in one device pass."""
        config = config or RenderConfig()
        arr = (_lib.Request * len(requests))()
        for i, (e, fr, ind, wd) in enumerate(requests):
            arr[i] = _lib.Request(self.envIds[e], fr, ind.data_ptr(), wd.data_ptr())
        opts = config.opts()
        self._check(lib().nwprt_relight_batch(self._ctx, arr, len(requests), C.byref(opts),
                                              _stream_ptr(stream)))

    def calibrateFP8(self, envMapID: int, frameID: int, px_begin: int = 0, px_end: int = 0,
                     stream=None) -> np.ndarray:
        """Per-layer E4M3 scales from a BF16 pass over pixels [px_begin, px_end) of a prepared
        frame; they stay fixed for every precision="fp8" relight until the next calibration
        or weight load.  Blocking.  Returns the calibrated activation maxima."""
        self._check(lib().nwprt_calibrate_fp8(self._ctx, int(envMapID), int(frameID), int(px_begin), int(px_end),
                                              _stream_ptr(stream)))
        return self.fp8Calibration()

    def fp8Calibration(self) -> np.ndarray:
        n = C.c_int(0)
        buf = (C.c_float * 32)()
        self._check(lib().nwprt_get_fp8_calibration(self._ctx, buf, 32, C.byref(n)))
        return np.array(buf[:n.value], np.float32)

    def relightRanges(self, ranges, config: Optional[RenderConfig] = None, stream=None) -> None:
        """Pixel-range relights (envMapID, frameID, indirect, with_direct, px_begin, px_end) in
        one device pass (BF16) -- the primitive the serving loop packs requests into."""
        config = config or RenderConfig()
        arr = (_lib.RangeRequest * len(ranges))()
        for i, (e, fr, ind, wd, b, en) in enumerate(ranges):
            arr[i] = _lib.RangeRequest(self.envIds[e], fr, ind.data_ptr(), wd.data_ptr(), int(b), int(en))
        opts = config.opts()
        self._check(lib().nwprt_relight_ranges(self._ctx, arr, len(ranges), C.byref(opts),
                                               _stream_ptr(stream)))

    def addEnvironmentFaces(self, faces: torch.Tensor, K: int, stream=None) -> int:
        """Registers an env map from device-resident faces [6,S,S,3] (Haar + top-K on the GPU)."""
        if faces.dtype != torch.float32 or not faces.is_cuda or not faces.is_contiguous():
            raise ValueError("faces must be a contiguous float32 CUDA tensor")
        env_id = C.c_int(-1)
        self._check(lib().nwprt_env_from_faces(self._ctx, _ptr(faces), 1, faces.shape[1], int(K),
                                               _stream_ptr(stream), C.byref(env_id)))
        self.envIds.append(env_id.value)
        self.EnvmapSetup = True
        return len(self.envIds) - 1

    def releaseEnvironmentMap(self, envMapID: int) -> None:
        self._check(lib().nwprt_env_release(self._ctx, self.envIds[envMapID]))
        self.envIds[envMapID] = -1

    def captureRelight(self, envMapID: int, frameID: int, config: Optional[RenderConfig] = None):
        """TCNNPass_p1 + TCNNPass_p2 of one frame and env map captured into a CUDA graph
        (torch.cuda.CUDAGraph).  Each replay() relights whatever the frame's G-buffer tensors
        hold at that moment into its output tensors, with no host work per frame.  One eager
        pass runs first, so one-time set-up (buffer growth, the env's embedding rows) stays out
        of the graph.  The frame's tensors, the env map and the weights must stay in place
        while the graph is used: a weight load, a frame of another size or releasing the env
        map invalidates it."""
        config = config or RenderConfig()
        self.TCNNPass_p1(frameID)
        self.TCNNPass_p2(envMapID, frameID, config)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, capture_error_mode="relaxed"):
            self.TCNNPass_p1(frameID)
            self.TCNNPass_p2(envMapID, frameID, config)
        return g

    def selftestDeviceWait(self, timeout_ms: int = 50, stream=None) -> None:
        """Diagnostics: a device wait that can never finish gives up after timeout_ms and is
        reported by the next TCNNSync as a TIMEOUT error; the context stays usable."""
        self._check(lib().nwprt_selftest_device_wait(self._ctx, int(timeout_ms), _stream_ptr(stream)))

    def TCNNSync(self) -> None:
        """tcnn.cu:154-158; also surfaces device-side error reports."""
        self._check(lib().nwprt_sync(self._ctx))

    def shInterpolate(self, vertex_rgb: torch.Tensor, tri: torch.Tensor, uv: torch.Tensor,
                      out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        """Pixel colours of the SH path from per-vertex colours (devicePrograms.cu:488-490):
        vertex_rgb [V, 3] float32, tri [P, 3] int32, uv [P, 2] float32 -> [P, 4] (rgb, 1).
        A triangle index outside the vertex range reads as (0, 0, 0, 1) and is reported by
        TCNNSync."""
        if vertex_rgb.dtype != torch.float32 or tri.dtype != torch.int32 or uv.dtype != torch.float32:
            raise ValueError("vertex_rgb float32 [V, 3], tri int32 [P, 3], uv float32 [P, 2]")
        P = tri.shape[0]
        if out is None:
            out = torch.empty((P, 4), dtype=torch.float32, device=vertex_rgb.device)
        self._check(lib().nwprt_sh_interpolate(self._ctx, _ptr(vertex_rgb.contiguous()), vertex_rgb.shape[0],
                                               _ptr(tri.contiguous()), _ptr(uv.contiguous()), P, _ptr(out),
                                               _stream_ptr(stream)))
        return out

    def computeFinalPixelColors(self, frameID: int, renderingMode: str = "full", stream=None) -> torch.Tensor:
        """RenderEngine::computeFinalPixelColors (toneMap.cu:73-98) for the wavelet path: the
        relit frame (indirect + direct for "full", indirect alone for "indirect") -> packed
        RGBA8 in frame.fbFinalColor (int32 tensor holding the uint32 pixels).  Asynchronous."""
        fr = self.fullframeCUDABuffer[frameID]
        src = {"full": fr.fbPredictedIndirectWithDirect, "indirect": fr.fbPredictedIndirect}.get(renderingMode)
        if src is None:
            raise ValueError(f"unknown renderingMode {renderingMode!r}")
        n = fr.width * fr.height
        if fr.fbFinalColor is None or fr.fbFinalColor.numel() != n:
            fr.fbFinalColor = torch.empty(n, dtype=torch.int32, device=src.device)
        return tonemap_srgb(src, out=fr.fbFinalColor, stream=stream)


# -------------------------------------------------------------------- context-free kernels

def haar_topk(faces: torch.Tensor, K: int, stream=None):
    """faces float32 cuda [6,S,S,3] or [E,6,S,S,3] -> (idx int32 [..,K], strength [..,K,3])."""
    if faces.dtype != torch.float32 or not faces.is_cuda or not faces.is_contiguous():
        raise ValueError("faces must be a contiguous float32 CUDA tensor")
    batched = faces.dim() == 5
    f = faces if batched else faces.unsqueeze(0)
    E, S = f.shape[0], f.shape[2]
    idx = torch.empty((E, K), dtype=torch.int32, device=faces.device)
    st = torch.empty((E, K, 3), dtype=torch.float32, device=faces.device)
    check(lib().nwprt_haar_topk(_ptr(f), E, S, int(K), _ptr(idx), _ptr(st), _stream_ptr(stream)))
    return (idx, st) if batched else (idx[0], st[0])


def tonemap_srgb(src: torch.Tensor, out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
    """float32 cuda [n, 4] linear radiance -> int32 [n] packed RGBA8 (the reference's
    final-colour pass, toneMap.cu:47-71)."""
    if src.dtype != torch.float32 or not src.is_cuda or not src.is_contiguous() or src.shape[-1] != 4:
        raise ValueError("src must be a contiguous float32 CUDA tensor [n, 4]")
    n = src.numel() // 4
    if out is None:
        out = torch.empty(n, dtype=torch.int32, device=src.device)
    if out.dtype != torch.int32 or out.numel() != n or not out.is_contiguous():
        raise ValueError("out must be a contiguous int32 tensor of n pixels")
    check(lib().nwprt_tonemap_srgb(_ptr(src), n, _ptr(out), _stream_ptr(stream)))
    return out


def env_rotate(faces: torch.Tensor, R, out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
    """Rotated cubemap dst(d) = src(R^T d), point-sampled like the reference's env lookup."""
    if faces.dtype != torch.float32 or not faces.is_cuda or not faces.is_contiguous():
        raise ValueError("faces must be a contiguous float32 CUDA tensor")
    r = np.ascontiguousarray(np.asarray(R, np.float32).reshape(9))
    if out is None:
        out = torch.empty_like(faces)
    check(lib().nwprt_env_rotate(_ptr(faces), faces.shape[1], r.ctypes.data_as(C.c_void_p), _ptr(out),
                                 _stream_ptr(stream)))
    return out


def sh_project(faces: torch.Tensor, stream=None) -> torch.Tensor:
    """faces float32 cuda [6,S,S,3] -> L [81,3] (order-8 SH of the cubemap)."""
    if faces.dtype != torch.float32 or not faces.is_cuda or not faces.is_contiguous():
        raise ValueError("faces must be a contiguous float32 CUDA tensor")
    S = faces.shape[1]
    nbytes = lib().nwprt_sh_project_workspace_size(S)
    ws = torch.empty(max(1, nbytes // 4), dtype=torch.float32, device=faces.device)
    L = torch.empty((81, 3), dtype=torch.float32, device=faces.device)
    check(lib().nwprt_sh_project(_ptr(faces), S, _ptr(L), _ptr(ws), nbytes, _stream_ptr(stream)))
    return L


def sh_vertex_radiance(T: torch.Tensor, brdf: torch.Tensor, L: torch.Tensor, out: Optional[torch.Tensor] = None,
                       stream=None) -> torch.Tensor:
    """Per-vertex SH shading (devicePrograms.cu:476-486): T [V, n, n], brdf [V, n, 3], L [n, 3]
    (float32 CUDA) -> [V, 3] = |sum_k (T L)[k] * brdf[k]|."""
    for a in (T, brdf, L):
        if a.dtype != torch.float32 or not a.is_cuda or not a.is_contiguous():
            raise ValueError("T, brdf and L must be contiguous float32 CUDA tensors")
    V, n = T.shape[0], T.shape[1]
    if T.shape != (V, n, n) or brdf.shape != (V, n, 3) or L.shape != (n, 3):
        raise ValueError("shapes must be T [V, n, n], brdf [V, n, 3], L [n, 3]")
    if out is None:
        out = torch.empty((V, 3), dtype=torch.float32, device=T.device)
    check(lib().nwprt_sh_vertex_radiance(_ptr(T), _ptr(brdf), _ptr(L), V, n, _ptr(out), _stream_ptr(stream)))
    return out


def sh_dot(T: torch.Tensor, L: torch.Tensor, abs_out: bool = True, out: Optional[torch.Tensor] = None,
           stream=None) -> torch.Tensor:
    """T float32 cuda [N, nc], L [nc, 3] -> out [N, 4] = (|T L|, 1)."""
    if T.dtype != torch.float32 or not T.is_contiguous() or L.dtype != torch.float32:
        raise ValueError("T and L must be contiguous float32")
    N, nc = T.shape
    if out is None:
        out = torch.empty((N, 4), dtype=torch.float32, device=T.device)
    check(lib().nwprt_sh_dot(_ptr(T), N, nc, _ptr(L.contiguous()), int(abs_out), _ptr(out),
                             _stream_ptr(stream)))
    return out

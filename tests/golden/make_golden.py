"""Writes the golden fixtures under tests/golden/ (run from the repository root):

    python tests/golden/make_golden.py

The reference ships no tests, fixtures or trained data, so these known answers are made
here from seeded synthetic inputs by the CPU oracle, plus the reference's own
utils_kernels.h built for the host (oracle/_ref, needed for the ``fp32_refrows`` arrays):

* every synthetic input is pinned by the SHA-256 of its bytes, so a changed generator
  shows up as a fixture failure instead of as a silent new baseline;
* ``cfg0.npz``  config 0: 128x128, K=64 from a 6x32x32 env map, hash 8x2 2^16, 42->64->64->3;
* ``cfg2.npz``  config 2: 1920x1080, K=300 from a 6x64x64 env map, hash 16x2 2^19, 64-wide
  MLPs with 3 hidden layers and FP16-rounded parameters (eight 128-pixel ranges);
* ``cfg1.npz``  config 1: the SH projection of a 6x128x128 env map and the SH dot of 1,024
  transport vectors.

Each relight fixture holds the Haar + top-K table (indices and strength bits), the FP32
oracle's output, the FP64 oracle's output, and the FP32 output computed from the
reference's own G-buffer remap rows (prt::waveletDataCopy, whose roughness column uses
logf where this library uses a correctly rounded log) on a pixel sample.
"""
from __future__ import annotations

import dataclasses
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from neural_wavelet_prt_demo_b200 import netconfig, synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

# the cases (shared with the tests that read the fixtures)
CFG0 = dict(cfg=netconfig.CONFIG_SMALL, width=128, height=128, K=64, seed=0, hash_scale=1e-4,
            param_round="fp32", px_stride=7)
CFG2 = dict(cfg=netconfig.CONFIG_LARGE, width=1920, height=1080, K=300, seed=0, hash_scale=1e-4,
            param_round="fp16", runs=8, run_px=128)
CFG1 = dict(face_size=128, env_seed=0, n_px=1024, t_seed=3)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def relight_inputs(c):
    """The seeded weights, G-buffer and env map of a relight case (seed, seed+1, seed+2)."""
    desc = netconfig.parse(c["cfg"])
    w = synth.make_weights(desc, seed=c["seed"], hash_scale=c["hash_scale"], param_round=c["param_round"])
    gb = synth.make_gbuffer(c["width"], c["height"], seed=c["seed"] + 1)
    faces = synth.make_env_faces(desc.face_size, seed=c["seed"] + 2)
    return desc, w, gb, faces


def input_digests(w, gb, faces) -> dict:
    d = {"faces": sha(faces), "hash_params": sha(w.hash_params), "out_prd": sha(w.out_prd),
         "cmp_net": sha(w.cmp_net), "wve_enc": sha(w.wve_enc)}
    for name, a in zip(("pos", "normal", "reflect", "roughness", "kd", "ks", "direct", "flag"), gb.arrays()):
        d["gb_" + name] = sha(a)
    return d


def sample_pixels(c, n_px: int) -> np.ndarray:
    """The pixel indices a fixture covers."""
    if "px_stride" in c:
        return np.arange(0, n_px, c["px_stride"], dtype=np.int64)
    runs, per = c["runs"], c["run_px"]
    starts = [int(i * (n_px - per) / (runs - 1)) for i in range(runs)]
    return np.concatenate([np.arange(s, s + per, dtype=np.int64) for s in starts])


def contiguous_runs(px: np.ndarray):
    """Splits sorted pixel indices into [begin, end) runs."""
    cut = np.nonzero(np.diff(px) != 1)[0] + 1
    return [(int(r[0]), int(r[-1]) + 1) for r in np.split(px, cut)]


def _sub_gbuffer(gb, b, e):
    """Pixels [b, e) of a G-buffer as a 1-row G-buffer (waveletDataCopy is per pixel)."""
    sl = slice(b, e)
    return dataclasses.replace(gb, width=e - b, height=1, pos=gb.pos[sl], normal=gb.normal[sl],
                               reflect=gb.reflect[sl], roughness=gb.roughness[sl], kd=gb.kd[sl],
                               ks=gb.ks[sl], direct=gb.direct[sl], flag=gb.flag[sl])


def relight_fixture(c) -> dict:
    desc, w, gb, faces = relight_inputs(c)
    idx, st = O.haar_topk(faces, c["K"])
    b = O.Bound(desc, w, gb)
    px = sample_pixels(c, gb.n)
    f32, f64, refrows = [], [], []
    for (s, e) in contiguous_runs(px) if "runs" in c else [(0, gb.n)]:
        ind, _ = O.relight_f32(b, idx, st, px_begin=s, px_end=e)
        f32.append(ind[s:e])
        f64.append(O.relight_f64(b, idx, st, px_begin=s, px_end=e))
        rows = O.ref_wavelet_data_copy(_sub_gbuffer(gb, s, e))[:, 0, :]
        rr, _ = O.relight_rows_f32(b, rows, idx, st, s)
        refrows.append(rr[s:e])
    f32, f64, refrows = (np.concatenate(a) for a in (f32, f64, refrows))
    if "px_stride" in c:
        f32, f64, refrows = f32[px], f64[px], refrows[px]
    dig = input_digests(w, gb, faces)
    return {"px": px, "topk_idx": idx, "topk_strength": st, "fp32_indirect": f32, "fp64_rgb": f64,
            "fp32_refrows_indirect": refrows, "digest_keys": np.array(list(dig.keys())),
            "digest_values": np.array(list(dig.values()))}


def sh_fixture(c) -> dict:
    faces = synth.make_env_faces(c["face_size"], seed=c["env_seed"])
    L64 = O.sh_project_f64(faces)[0]
    T = synth.make_sh_transport(c["n_px"], seed=c["t_seed"])
    L32 = L64.astype(np.float32)
    return {"L_f64": L64, "sh_dot_f32": O.sh_dot_f32(T, L32), "sh_dot_f64": O.sh_dot_f64(T, L32),
            "digest_keys": np.array(["faces", "T"]), "digest_values": np.array([sha(faces), sha(T)])}


def main():
    if O.ref_lib() is None:
        raise SystemExit("oracle/_ref/libref_utils.so is missing: build it with make -C oracle REF=<reference tree>")
    for name, fn, c in (("cfg0", relight_fixture, CFG0), ("cfg2", relight_fixture, CFG2),
                        ("cfg1", sh_fixture, CFG1)):
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **fn(c))
        print(f"{path}: {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()

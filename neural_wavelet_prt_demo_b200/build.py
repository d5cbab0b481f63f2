"""Builds libnwprt.so (the C-ABI library) in-tree for sm_100a.

    python -m neural_wavelet_prt_demo_b200.build [--force] [--verbose]

Each translation unit under csrc/ is compiled by nvcc (in parallel, incremental by
mtime) into _build/, then linked into neural_wavelet_prt_demo_b200/libnwprt.so.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libnwprt.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
SOURCES = ["api.cu", "config.cpp", "haar_topk.cu", "sh.cu", "relight_common.cu", "relight_fp32.cu",
           "relight_tc.cu", "sh_noalloc.cu", "env_rotate.cu", "tonemap.cu", "sh_vertex.cu"]
HEADERS = ["nwprt_internal.cuh"]


def _newer(src_paths, out):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(p) > t for p in src_paths)


def _compile(src, verbose, extra):
    s = os.path.join(CSRC, src)
    o = os.path.join(BUILD, src + ".o")
    deps = [s] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "nwprt.h")]
    if not _newer(deps, o):
        return o, None
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", s, "-o", o]
    if src.endswith(".cpp"):
        cmd = [NVCC, *FLAGS, *extra, "-x", "c++", "-c", s, "-o", o]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return o, f"{src}:\n{r.stdout}\n{r.stderr}"
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)
    return o, None


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            if f.endswith(".o"):
                os.remove(os.path.join(BUILD, f))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose, list(extra)), SOURCES))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if force or _newer(objs, LIB):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/smem usage")
    a = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.ptxas_v else []
    print(build(force=a.force or a.ptxas_v, verbose=a.verbose or a.ptxas_v, extra=extra))


if __name__ == "__main__":
    sys.exit(main())

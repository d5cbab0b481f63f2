"""Benchmark of the neural wavelet PRT relight pass (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision auto|bf16|fp32]
                    [--workload relight1080|sh1080|shvertex|haar|tonemap|serve|sweep]

Default workload: relight of a 1920x1080 synthetic G-buffer with K=300 wavelets of a
6x64x64 env map through the 16-level hash grid + 64-wide MLP network (FP16-rounded
random-init params).  One step = TCNNPass_p1 + TCNNPass_p2 of one frame.  Metric:
pixel*wavelet evaluations per second, whole job.  The line also carries the end-to-end
figure through the public API with host buffers (``e2e``), the plain FP32 drop-in and the
FP8 form of the same step, the relight kernel's roofline, and the CPU baseline.

Other workloads: ``sh1080`` (SH dot, HBM roofline), ``shvertex`` (per-vertex SH shading +
interpolation), ``haar`` (Haar + top-K of 1024 env maps), ``tonemap`` (final-colour pass),
``serve`` (the config-4 serving stream: p50/p99 latency and throughput) and ``sweep`` (the
config-3 precision sweep against the FP64 oracle).

Multi-GPU (torchrun): every rank relights its own frame (request-level data
parallelism, no collective on the data path); timing is the max over ranks.

``--impl reference`` times the reference's relighting math on the host cores (the CPU
oracle, all threads) on a bounded pixel sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "px*wavelet evals/s at 1080p K=300"
WIDTH, HEIGHT, K_WAVELETS = 1920, 1080, 300


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["auto", "bf16", "fp32"], default="auto")
    ap.add_argument("--workload", choices=["relight1080", "sh1080", "shvertex", "haar", "tonemap", "serve", "sweep"], default="relight1080")
    ap.add_argument("--sweep-px", type=int, default=4096, help="pixels checked against the FP64 oracle per K")
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-rate", type=float, default=120.0)
    ap.add_argument("--serve-quantum-ms", type=float, default=12.0,
                    help="serve: kernel time per scheduling quantum")
    ap.add_argument("--serve-nets", choices=["both", "large", "small"], default="both",
                    help="serve: which network(s) to run (config 2, config 0, or both)")
    ap.add_argument("--serve-order", choices=["fifo", "srpt", "edf"], default="edf",
                    help="serve: quantum packing order (earliest deadline with deadlines proportional to "
                         "request size, arrival, or least remaining work)")
    ap.add_argument("--serve-max-active", type=int, default=0,
                    help="serve: admit at most this many requests at once (0: the byte budget alone)")
    ap.add_argument("--serve-in-flight", type=int, default=2,
                    help="serve: relight launches kept queued on the GPU (1: a new request waits behind at "
                         "most one quantum, at the cost of a gap between launches)")
    ap.add_argument("--serve-serial-prefix", type=int, default=40,
                    help="requests of the stream also served by the plain FP32 serial baseline")
    ap.add_argument("--fp8-steps", type=int, default=5, help="timed steps of the FP8 form (0: skip)")
    ap.add_argument("--graph-steps", type=int, default=5, help="timed replays of the captured step (0: skip)")
    ap.add_argument("--fp32-steps", type=int, default=2, help="timed steps of the plain FP32 path")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--width", type=int, default=1920, help="frame width (profiling runs use smaller cases)")
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--K", type=int, default=300, help="wavelets per pixel")
    a = ap.parse_args()
    global WIDTH, HEIGHT, K_WAVELETS
    WIDTH, HEIGHT, K_WAVELETS = a.width, a.height, a.K
    return a


# ---------------------------------------------------------------------------- helpers

def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        load = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def load_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# ---------------------------------------------------------------------------- workload

def relight_config(world: int, h2d_bytes: int) -> dict:
    """The `config` of the relight workload, identical on both arms."""
    return {"workload": f"relight {WIDTH}x{HEIGHT}, K={K_WAVELETS} of a 6x64x64 env map, "
                        "hash 16x2 2^19, MLPs 32->64x3->64 | 80->64x3->3",
            "pixels_per_gpu": WIDTH * HEIGHT, "K": K_WAVELETS,
            "l2": f"inputs {h2d_bytes / 1e6:.0f} MB/frame vs 126 MB L2 (no flush)",
            "parallelism": f"request-dp{world}", "step": "TCNNPass_p1 + TCNNPass_p2"}


# accuracy sample: ACC_RUNS contiguous runs of ACC_RUN pixels spread over the frame
ACC_RUNS, ACC_RUN = 8, 256


def accuracy_sample_starts(n_px: int):
    return [int(i * (n_px - ACC_RUN) / (ACC_RUNS - 1)) for i in range(ACC_RUNS)]


def error_stats(x, ref) -> dict:
    """max / mean relative error (denominators floored at 1e-6 of the image maximum), PSNR
    over the image maximum, and the largest absolute error over that maximum."""
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    peak = float(np.abs(ref).max())
    rel = np.abs(x - ref) / np.maximum(np.abs(ref), max(1e-6 * peak, 1e-30))
    mse = float(np.mean((x - ref) ** 2))
    return {"max_rel_err": float(rel.max()), "mean_rel_err": float(rel.mean()),
            "psnr_db": 10 * np.log10(peak * peak / mse) if mse > 0 else float("inf"),
            "max_abs_err_over_peak": float(np.abs(x - ref).max()) / peak if peak > 0 else 0.0}


def accuracy_report(desc, w, gb, idx, st, outputs: dict) -> dict:
    """Each precision's sampled output against the FP64 oracle of the same network, weights,
    G-buffer and wavelet table (computed after the timed regions)."""
    from oracle import oracle as O
    b = O.Bound(desc, w, gb)
    starts = accuracy_sample_starts(gb.n)
    ref = np.concatenate([O.relight_f64(b, idx, st, px_begin=s, px_end=s + ACC_RUN) for s in starts])
    rep = {name: error_stats(out, ref) for name, out in outputs.items()}
    rep["sample"] = f"{ACC_RUNS} runs of {ACC_RUN} pixels spread over the frame, RGB of fbPredictedIndirect"
    rep["reference"] = "FP64 oracle, same network / weights / wavelet table"
    return rep


def make_relight_inputs(rank: int):
    from neural_wavelet_prt_demo_b200 import netconfig, synth
    desc = netconfig.parse(netconfig.CONFIG_LARGE)
    w = synth.make_weights(desc, seed=0, hash_scale=1e-4, param_round="fp16")
    gb = synth.make_gbuffer(WIDTH, HEIGHT, seed=1 + rank)
    faces = synth.make_env_faces(desc.face_size, seed=2)
    return desc, w, gb, faces


def cpu_relight_rate(desc, w, gb, idx, st, budget_s: float):
    """Oracle FP32 relight on a contiguous block of pixels sized to ~budget_s of host time."""
    from oracle import oracle as O
    b = O.Bound(desc, w, gb)
    threads = O.max_threads()
    mid = gb.n // 2
    n = 256
    t0 = time.perf_counter()
    O.relight_f32(b, idx, st, px_begin=mid, px_end=mid + n, n_threads=threads)
    dt = time.perf_counter() - t0
    n2 = int(min(gb.n - mid, max(n, n * budget_s / max(dt, 1e-6))))
    t0 = time.perf_counter()
    O.relight_f32(b, idx, st, px_begin=mid, px_end=mid + n2, n_threads=threads)
    dt = time.perf_counter() - t0
    return n2 * len(idx) / dt, threads, n2, dt


# ---------------------------------------------------------------------------- ours

def run_ours(args):
    import torch
    import torch.distributed as dist
    from neural_wavelet_prt_demo_b200 import engine as eng
    from neural_wavelet_prt_demo_b200.sharding import max_over_ranks

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        # a short timeout: ranks waiting on a failed peer end with an error instead of hanging
        # (the longest stretch without a collective is a rank-0 host phase of ~20 s)
        import datetime
        dist.init_process_group("nccl", device_id=dev, timeout=datetime.timedelta(seconds=300))

    if args.workload == "sh1080":
        return run_sh(args, rank, world, local, dev)
    if args.workload == "haar":
        return run_haar(args, rank, world, local, dev)
    if args.workload == "tonemap":
        return run_tonemap(args, rank, world, local, dev)
    if args.workload == "shvertex":
        return run_shvertex(args, rank, world, local, dev)
    if args.workload == "serve":
        return run_serve(args, rank, world, local, dev)
    if args.workload == "sweep":
        return run_sweep(args, rank, world, local, dev)

    desc, w, gb, faces = make_relight_inputs(rank)
    e = eng.RenderEngine(netconfig_json(), device=local)
    e.loadWeights(w)
    env_id = e.addEnvironmentMap(eng.EnvironmentMap(faces), K=K_WAVELETS)
    idx, st = e.envWavelets(env_id)
    fr = eng.FullFrame.from_gbuffer(gb, dev)
    e.setFrame(0, fr)
    N = WIDTH * HEIGHT
    evals = N * K_WAVELETS

    precision = args.precision
    if precision == "auto":
        try:
            e.TCNNPass_p1(0)
            e.TCNNPass_p2(env_id, 0, eng.RenderConfig(precision="bf16"))
            e.TCNNSync()
            precision = "bf16"
        except eng.NwprtError:
            precision = "fp32"
    cfg = eng.RenderConfig(precision=precision)
    stream = torch.cuda.current_stream()

    def step():
        e.TCNNPass_p1(0)
        e.TCNNPass_p2(env_id, 0, cfg)

    def timed(step_fn, steps, warmup, kernel_events=None):
        for _ in range(warmup):
            step_fn()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            step_fn()
        b.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ms = max_over_ranks(a.elapsed_time(b), device=dev)
        return ms / steps

    # ---- device-resident throughput (value) with live per-launch kernel timing
    kev = []

    def step_k():
        e.TCNNPass_p1(0)
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        e.TCNNPass_p2(env_id, 0, cfg)
        s1.record(stream)
        kev.append((s0, s1))

    sampler = ClockSampler(local)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler.start()
    ms_step = timed(step_k, args.steps, 0)
    clocks = sampler.stop()
    kernel_ms = sum(x.elapsed_time(y) for x, y in kev) / len(kev)
    value = world * evals / (ms_step / 1e3)
    acc_sel = torch.from_numpy(np.concatenate([np.arange(s, s + ACC_RUN)
                                               for s in accuracy_sample_starts(N)])).to(dev)

    def sampled_output():
        return fr.fbPredictedIndirect[acc_sel][:, :3].double().cpu().numpy()

    acc_outputs = {precision: sampled_output()}

    # ---- end to end through the public API with host buffers.  Every step copies its frame's
    # G-buffer from pinned host memory and reads both outputs back.  Two device frames
    # alternate: a step's host->device copy and the previous step's device->host read run on a
    # copy stream while the relight of the other frame runs on the compute stream.
    pin = lambda t: t.cpu().pin_memory()
    in_names = ("fbFirstHitPos", "fbworldNormal", "fbFirstHitReflecDir", "fbRoughness", "fbFirstHitKd",
                "fbFirstHitKs", "fbDirectDenoised", "fbEnvironmentMapFlag")
    out_names = ("fbPredictedIndirect", "fbPredictedIndirectWithDirect")
    host_in = {n: pin(getattr(fr, n)) for n in in_names}
    frames_e2e = [fr, eng.FullFrame.from_gbuffer(gb, dev)]
    e.setFrame(1, frames_e2e[1])
    host_out = [{n: torch.empty_like(getattr(fr, n), device="cpu").pin_memory() for n in out_names}
                for _ in range(2)]
    h2d = sum(t.numel() * t.element_size() for t in host_in.values())
    d2h = sum(t.numel() * t.element_size() for t in host_out[0].values())
    up_stream, down_stream = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    computed = [None, None]  # event: the last relight of slot s finished (its inputs are free)
    read = [None, None]      # event: the last read-back of slot s finished (its outputs are free)

    def run_e2e(n_steps):
        for i in range(n_steps):
            s_ = i % 2
            F = frames_e2e[s_]
            with torch.cuda.stream(up_stream):
                if computed[s_] is not None:
                    up_stream.wait_event(computed[s_])
                for n, t in host_in.items():
                    getattr(F, n).copy_(t, non_blocking=True)
                loaded = torch.cuda.Event()
                loaded.record(up_stream)
            stream.wait_event(loaded)
            if read[s_] is not None:
                stream.wait_event(read[s_])
            e.TCNNPass_p1(s_)
            e.TCNNPass_p2(env_id, s_, cfg)
            done = torch.cuda.Event()
            done.record(stream)
            computed[s_] = done
            with torch.cuda.stream(down_stream):
                down_stream.wait_event(done)
                for n, t in host_out[s_].items():
                    t.copy_(getattr(F, n), non_blocking=True)
                rb = torch.cuda.Event()
                rb.record(down_stream)
                read[s_] = rb
        stream.wait_stream(down_stream)  # the last read-back is inside the timed region

    n_e2e = max(3, args.steps // 2)
    run_e2e(2)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ea.record(stream)
    run_e2e(n_e2e)
    eb.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(ea.elapsed_time(eb), device=dev) / n_e2e
    ok = all(torch.equal(host_out[s_][n], getattr(frames_e2e[s_], n).cpu()) for s_ in range(2) for n in out_names)
    e2e = {"value": world * evals / (ms_e2e / 1e3), "unit": "evals/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e,
           "pipeline": "2 frames; uploads and read-backs on their own streams overlap the other frame's relight",
           "readback_matches_device": ok}

    # ---- the same step replayed from a CUDA graph (TCNNPass_p1 + TCNNPass_p2 captured once)
    graph = None
    if args.graph_steps > 0:
        gr = e.captureRelight(env_id, 0, cfg)
        msg = timed(gr.replay, args.graph_steps, 2)
        graph = {"value": world * evals / (msg / 1e3), "unit": "evals/s", "ms_per_step": msg}
        del gr

    # ---- the plain FP32 drop-in path, same workload (for the served/plain ratio)
    plain = None
    if precision != "fp32" and args.fp32_steps > 0:
        cfg32 = eng.RenderConfig(precision="fp32")

        def step32():
            e.TCNNPass_p1(0)
            e.TCNNPass_p2(env_id, 0, cfg32)

        ms32 = timed(step32, args.fp32_steps, 1)
        plain = {"value": world * evals / (ms32 / 1e3), "unit": "evals/s", "ms_per_step": ms32}
        acc_outputs["fp32"] = sampled_output()

    # ---- the FP8 (E4M3) form of the same step, scales from a seeded calibration batch
    fp8 = None
    if precision == "bf16" and args.fp8_steps > 0:
        from neural_wavelet_prt_demo_b200 import synth
        cal = eng.FullFrame.from_gbuffer(synth.make_gbuffer(256, 256, seed=7), dev)
        e.setFrame(1, cal)
        e.TCNNPass_p1(1)
        e.calibrateFP8(env_id, 1)
        cfg8 = eng.RenderConfig(precision="fp8")

        def step8():
            e.TCNNPass_p1(0)
            e.TCNNPass_p2(env_id, 0, cfg8)

        ms8 = timed(step8, args.fp8_steps, 1)
        fp8 = {"value": world * evals / (ms8 / 1e3), "unit": "evals/s", "ms_per_step": ms8,
               "calibration": "256x256 G-buffer seed 7, same env map",
               "served": False, "why_not_served": "below the 45 dB PSNR bar (see accuracy)"}
        acc_outputs["fp8_e4m3"] = sampled_output()

    # ---- roofline of the dominant kernel (the fused relight)
    peaks, peak_src = load_peaks()
    flops = desc.flops_per_eval() * evals
    achieved = flops / (kernel_ms / 1e3) / 1e12
    if precision == "bf16":
        peak = peaks["bf16_tflops"]
        peak_sus = peaks.get("bf16_tflops_sustained")
        # DRAM bytes per launch from one ncu capture of this kernel on the same 1920x1080 frame
        # (dram__bytes_read.sum + dram__bytes_write.sum = 337.0 + 63.3 MB at K=8); the kernel
        # reads each pixel's inputs and writes its outputs once, so the traffic does not depend
        # on K and scales with the pixel count.
        traffic = 400.3e6 * N / (1920 * 1080)
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": traffic,
                "traffic_source": "ncu dram bytes of relight_tc_kernel, 1920x1080 K=8 capture, K-independent",
                "peak_source": f"{peak_src} bf16 burst (cuBLAS 8192^3 GEMM, best of 10)",
                "peak_sustained": peak_sus,
                "frac_of_sustained": achieved / peak_sus if peak_sus else None}
    else:
        peak = 148 * 128 * 2 * 1.965e9 / 1e12
        roof = {"bound": "fp32-simt", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": None,
                "peak_source": "nominal FP32 CUDA-core peak (148 SM x 128 FMA/clk x 1965 MHz)"}
    roof["kernel_ms"] = kernel_ms
    roof["algorithmic_flops_per_launch"] = flops
    if precision != "fp32":
        # the tensor-core plan folds out_prd's linear output layer into cmp_net's first layer
        op_in_last, op_out = desc.op_layers()[-1]
        roof["executed_flops_per_eval"] = desc.flops_per_eval() - 2 * op_in_last * op_out

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, n_px, dt = cpu_relight_rate(desc, w, gb, idx, st, args.cpu_seconds)
        cpu = {"value": rate, "unit": "evals/s", "cores": cores, "kind": "port",
               "sample": f"{n_px} contiguous pixels x K={K_WAVELETS} through the FP32 oracle ({dt:.1f} s)"}

    e.close()
    accuracy = accuracy_report(desc, w, gb, idx, st, acc_outputs) if rank == 0 else None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": precision,
            "data": "synthetic: seeded G-buffer, log-normal env map, random-init FP16-rounded weights",
            "config": relight_config(world, h2d),
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": 2 * args.steps,
            "clocks": clocks, "accuracy": accuracy, "plain_fp32": plain, "fp8_e4m3": fp8,
            "cuda_graph": graph,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def netconfig_json():
    from neural_wavelet_prt_demo_b200 import netconfig
    return netconfig.to_json(netconfig.CONFIG_LARGE)


# ---------------------------------------------------------------------------- SH workload

def run_sh(args, rank, world, local, dev):
    import torch
    import torch.distributed as dist
    from neural_wavelet_prt_demo_b200 import engine as eng, synth
    N = WIDTH * HEIGHT
    g = torch.Generator(device=dev).manual_seed(rank)
    l = torch.floor(torch.sqrt(torch.arange(81, device=dev, dtype=torch.float32))).clamp_min(1)
    T = torch.randn((N, 81), generator=g, device=dev) / (l * l)
    faces = torch.from_numpy(synth.make_env_faces(128, seed=0)).to(dev)
    L = eng.sh_project(faces)
    out = torch.empty((N, 4), device=dev)
    for _ in range(args.warmup):
        eng.sh_dot(T, L, out=out)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        eng.sh_dot(T, L, out=out)
    b.record()
    torch.cuda.synchronize()
    from neural_wavelet_prt_demo_b200.sharding import max_over_ranks
    ms = max_over_ranks(a.elapsed_time(b), device=dev) / args.steps
    bytes_ = N * 81 * 4 + N * 16 + 81 * 12
    peaks, src = load_peaks()
    gbs = bytes_ / (ms / 1e3) / 1e9
    if rank == 0:
        print(json.dumps({"metric": "SH dot GB/s at 1080p (81 coeffs)", "value": gbs * world, "unit": "GB/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                          "data": "synthetic", "config": {"workload": "sh_dot 1920x1080x81"},
                          "roofline": {"bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                                       "frac": gbs / peaks["hbm_gbs"], "traffic": None},
                          "gpu_launches": args.steps}), flush=True)
    if world > 1:
        dist.destroy_process_group()


SHV_VERTICES, SHV_PX = 100_000, 1920 * 1080


def run_shvertex(args, rank, world, local, dev):
    """Full SH path without the ray tracer: 100k mesh vertices with 81x81 transfer matrices
    (2.6 GB), per-vertex SH shading, then the barycentric colour of every 1080p pixel."""
    import torch
    import torch.distributed as dist
    from neural_wavelet_prt_demo_b200 import engine as eng, netconfig, synth
    from neural_wavelet_prt_demo_b200.sharding import max_over_ranks
    from oracle import oracle as O
    V, n = SHV_VERTICES, 81
    g = torch.Generator(device=dev).manual_seed(rank)
    l = torch.floor(torch.sqrt(torch.arange(n, device=dev, dtype=torch.float32))).clamp_min(1)
    T = torch.randn((V, n, n), generator=g, device=dev) / (l[None, :, None] * l[None, None, :])
    brdf = torch.randn((V, n, 3), generator=g, device=dev) / (l * l)[None, :, None]
    L = torch.randn((n, 3), generator=g, device=dev) / (l * l)[:, None]
    tri = torch.randint(0, V, (SHV_PX, 3), generator=g, device=dev, dtype=torch.int32)
    uv = torch.rand((SHV_PX, 2), generator=g, device=dev) * 0.5
    e = eng.RenderEngine(netconfig.to_json(netconfig.CONFIG_SMALL), device=local)
    vc = torch.empty((V, 3), device=dev)
    px = torch.empty((SHV_PX, 4), device=dev)

    def step():
        eng.sh_vertex_radiance(T, brdf, L, out=vc)
        e.shInterpolate(vc, tri, uv, out=px)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    a, b, m = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    clk = ClockSampler(local)
    clk.start()
    a.record()
    kv = []
    for _ in range(args.steps):
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        eng.sh_vertex_radiance(T, brdf, L, out=vc)
        s1.record()
        e.shInterpolate(vc, tri, uv, out=px)
        kv.append((s0, s1))
    b.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(a.elapsed_time(b), device=dev) / args.steps
    kms = sum(x.elapsed_time(y) for x, y in kv) / len(kv)
    vbytes = V * (n * n * 4 + n * 12 + 12)
    gbs = vbytes / (kms / 1e3) / 1e9
    peaks, psrc = load_peaks()
    if rank == 0:
        k = 64
        ok = bool(np.array_equal(vc[:k].cpu().numpy().view(np.uint32),
                                 O.sh_vertex_radiance(T[:k].cpu().numpy(), brdf[:k].cpu().numpy(),
                                                      L.cpu().numpy()).view(np.uint32)))
        print(json.dumps({"metric": "SH vertex path: vertices/s (100k vertices, 81x81 T, + 1080p interpolation)",
                          "value": world * V / (ms / 1e3), "unit": "vertices/s", "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                          "config": {"workload": f"sh_vertex_radiance {V}x{n}x{n} + sh_interpolate {SHV_PX} px",
                                     "l2": "2.6 GB of transfer matrices per step vs 126 MB L2"},
                          "roofline": {"bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                                       "frac": gbs / peaks["hbm_gbs"], "traffic": None, "peak_source": psrc,
                                       "kernel": "sh_vertex_kernel", "kernel_ms": kms},
                          "parity_bit_exact_64_vertices": ok, "clocks": clocks, "gpu_launches": 2 * args.steps}),
              flush=True)
        if not ok:
            raise SystemExit("sh_vertex_radiance differs from the oracle")
    e.close()
    if world > 1:
        dist.destroy_process_group()


TONEMAP_FRAMES = 16


def run_tonemap(args, rank, world, local, dev):
    """Final-colour pass over TONEMAP_FRAMES 1080p relit frames in one launch (533 MB of float4
    in, 133 MB of RGBA8 out: larger than L2)."""
    import torch
    import torch.distributed as dist
    from neural_wavelet_prt_demo_b200 import engine as eng
    from neural_wavelet_prt_demo_b200.sharding import max_over_ranks
    from oracle import oracle as O
    n = TONEMAP_FRAMES * 1920 * 1080
    g = torch.Generator(device=dev).manual_seed(rank)
    src = torch.rand((n, 4), generator=g, device=dev) * 1.2
    out = torch.empty(n, dtype=torch.int32, device=dev)
    for _ in range(args.warmup):
        eng.tonemap_srgb(src, out=out)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(local)
    clk.start()
    a.record()
    for _ in range(args.steps):
        eng.tonemap_srgb(src, out=out)
    b.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(a.elapsed_time(b), device=dev) / args.steps
    gbs = n * 20 / (ms / 1e3) / 1e9
    peaks, psrc = load_peaks()
    if rank == 0:
        k = 65536
        ok = bool(np.array_equal(out[:k].cpu().numpy().view(np.uint32), O.tonemap_srgb(src[:k].cpu().numpy())))
        print(json.dumps({"metric": "final-colour pass GB/s (16 x 1080p float4 -> RGBA8)", "value": gbs * world,
                          "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f32", "data": "synthetic uniform radiance",
                          "config": {"workload": f"tonemap_srgb {n} px", "l2": "667 MB per launch vs 126 MB L2"},
                          "roofline": {"bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                                       "frac": gbs / peaks["hbm_gbs"], "traffic": None, "peak_source": psrc},
                          "parity_bit_exact_65536_px": ok, "clocks": clocks, "gpu_launches": args.steps}),
              flush=True)
        if not ok:
            raise SystemExit("tonemap differs from the oracle")
    if world > 1:
        dist.destroy_process_group()


HAAR_MAPS, HAAR_S, HAAR_K = 1024, 64, 300


def run_haar(args, rank, world, local, dev):
    """Batched Haar transform + top-K: HAAR_MAPS 6x64x64 env maps per launch (302 MB of
    faces, larger than L2), K=300, plus the latency of a single-map launch."""
    import torch
    import torch.distributed as dist
    from neural_wavelet_prt_demo_b200 import engine as eng, synth
    from neural_wavelet_prt_demo_b200.sharding import max_over_ranks
    from oracle import oracle as O
    g = torch.Generator(device=dev).manual_seed(rank)
    # log-normal(0, 1.5) radiance, the env-map distribution of the relight workloads
    faces = torch.exp(1.5 * torch.randn((HAAR_MAPS, 6, HAAR_S, HAAR_S, 3), generator=g, device=dev))
    for _ in range(args.warmup):
        eng.haar_topk(faces, HAAR_K)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(local)
    clk.start()
    a.record()
    for _ in range(args.steps):
        idx, st = eng.haar_topk(faces, HAAR_K)
    b.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(a.elapsed_time(b), device=dev) / args.steps
    one = faces[:1].contiguous()
    for _ in range(3):
        eng.haar_topk(one, HAAR_K)
    torch.cuda.synchronize()
    a.record()
    for _ in range(20):
        eng.haar_topk(one, HAAR_K)
    b.record()
    torch.cuda.synchronize()
    single_us = a.elapsed_time(b) / 20 * 1e3
    per_map = 6 * HAAR_S * HAAR_S * 3 * 4 + HAAR_K * 16
    gbs = HAAR_MAPS * per_map / (ms / 1e3) / 1e9
    peaks, src = load_peaks()
    ok = True
    if rank == 0:
        # parity spot check on a few maps, then the oracle timed on the host cores
        sub = faces[:4].cpu().numpy()
        ridx, rst = O.haar_topk(sub, HAAR_K)
        ok = bool(np.array_equal(ridx, idx[:4].cpu().numpy()) and
                  np.array_equal(rst.view(np.uint32), st[:4].cpu().numpy().view(np.uint32)))
        cpu = None
        if not args.no_cpu_baseline:
            host = faces[:64].cpu().numpy()
            threads = O.max_threads()
            t0 = time.perf_counter()
            O.haar_topk(host, HAAR_K, n_threads=threads)
            dt = time.perf_counter() - t0
            cpu = {"value": 64 * per_map / dt / 1e9, "unit": "GB/s", "cores": threads, "kind": "port",
                   "sample": "64 maps of the same batch, oracle Haar + top-K on all host threads"}
        print(json.dumps({"metric": "Haar + top-K GB/s (1024 6x64x64 env maps, K=300)", "value": gbs * world,
                          "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f32", "data": "synthetic: log-normal(0,1.5) env maps",
                          "config": {"workload": f"haar_topk {HAAR_MAPS}x6x{HAAR_S}x{HAAR_S}x3 K={HAAR_K}",
                                     "l2": "inputs 302 MB vs 126 MB L2 (no flush)"},
                          "roofline": {"bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                                       "frac": gbs / peaks["hbm_gbs"], "traffic": None,
                                       "peak_source": src},
                          "single_map_us": single_us, "parity_bit_exact_4_maps": ok,
                          "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": args.steps}), flush=True)
    if world > 1:
        dist.destroy_process_group()
    if not ok:
        raise SystemExit("haar_topk differs from the oracle")


# ---------------------------------------------------------------------------- serving stream

def _serve_rig(cfg, face_size, dev, seed=0):
    import torch
    from neural_wavelet_prt_demo_b200 import engine as eng, netconfig, serve, synth
    desc = netconfig.parse(cfg)
    w = synth.make_weights(desc, seed=seed, hash_scale=1e-4,
                           param_round="fp16" if cfg is netconfig.CONFIG_LARGE else "fp32")
    e = eng.RenderEngine(cfg, device=dev.index or 0)
    e.loadWeights(w)
    frames = []
    for i, (W, H) in enumerate(serve.RESOLUTIONS):
        fr = eng.FullFrame.from_gbuffer(synth.make_gbuffer(W, H, seed=200 + i), dev)
        e.setFrame(i, fr)
        e.TCNNPass_p1(i)
        frames.append(fr)
    base = [torch.from_numpy(synth.make_env_faces(face_size, seed=300, index=j)).to(dev) for j in range(8)]
    torch.cuda.synchronize()
    return e, frames, base


def _measure_rate(e, frames, base, precision):
    """Steady-state evals/s of one 1080p K=300 relight (sizes the scheduling quantum)."""
    import torch
    from neural_wavelet_prt_demo_b200 import engine as eng
    env = e.addEnvironmentFaces(base[0], 300)
    fr = frames[3]
    n = fr.width * fr.height
    out, out2 = torch.empty((n, 4), device=base[0].device), torch.empty((n, 4), device=base[0].device)
    cfg = eng.RenderConfig(precision=precision)
    e.relightRanges([(env, 3, out, out2, 0, n)], cfg)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    e.relightRanges([(env, 3, out, out2, 0, n)], cfg)
    b.record()
    torch.cuda.synchronize()
    e.releaseEnvironmentMap(env)
    return n * 300 / (a.elapsed_time(b) / 1e3)


def run_serve(args, rank, world, local, dev):
    """Config-4 serving stream: Poisson arrivals, mixed resolution / K / env maps (40% new,
    60% rotations of resident maps), budget admission, continuous batching.  Reports
    throughput and p50/p99 latency (overall, and for frames up to 720p vs larger ones) of the
    served BF16 path, the same for a small (config-0) network, and the plain FP32 serial
    baseline on a prefix of the stream.

    Every rank serves the SAME stream: with N GPUs it is split by the dispatcher (requests
    placed by estimated backlog, frames of >= 1080p at K=300 split into row bands gathered at
    their owner with NCCL point-to-point transfers), so N only changes how fast the fixed
    stream is served ("strong" scaling)."""
    import torch
    import torch.distributed as dist
    from neural_wavelet_prt_demo_b200 import dispatch, netconfig, serve
    out = {}
    sampler = ClockSampler(local)
    nets = [("served_bf16", netconfig.CONFIG_LARGE, 64), ("served_bf16_small_net", netconfig.CONFIG_SMALL, 32)]
    if args.serve_nets == "large":
        nets = nets[:1]
    elif args.serve_nets == "small":
        nets = nets[1:]
    channels = dispatch.PairChannels(world) if world > 1 else None
    clocks = None
    for name, cfg, S in nets:
        e, frames, base = _serve_rig(cfg, S, dev)
        rate = _measure_rate(e, frames, base, "bf16")
        if world > 1:  # every rank plans with the same estimate
            t = torch.tensor([rate], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MIN)
            rate = float(t.item())
        reqs = serve.make_stream(args.serve_requests, args.serve_rate, seed=0, face_size=S)
        kw = dict(precision="bf16", budget_bytes=150 << 30, quantum_ms=args.serve_quantum_ms, est_evals_per_s=rate,
                  max_active=args.serve_max_active or None, order=args.serve_order,
                  max_in_flight=max(1, args.serve_in_flight))
        frame_px = [f.width * f.height for f in frames]
        first = clocks is None
        if first:
            sampler.start()
        if world > 1:
            torch.cuda.synchronize()
            dist.barrier()
            mine = dispatch.serve_distributed(e, frames, base, reqs, rank, world, channels, dev, rate,
                                              server_kwargs=kw)
            local_reqs = mine.pop("local")
            owned = [r for r in local_reqs if r.owner == rank or not r.split]
            mine["classes_local"] = [(frame_px[r.res], r.latency * 1e3) for r in owned if r.status == "done"]
            all_s = [None] * world
            dist.all_gather_object(all_s, mine)
            st = dispatch.combine_summaries(all_s)
            cls = {}
            for cname, pick in (("small", lambda n: n <= serve.SMALL_CLASS_MAX_PX),
                                ("large", lambda n: n > serve.SMALL_CLASS_MAX_PX)):
                lat = [l for s_ in all_s for (n, l) in s_["classes_local"] if pick(n)]
                cls[cname] = {"done": len(lat), "p50_ms": serve.percentile(lat, 50), "p99_ms": serve.percentile(lat, 99)}
            st["classes"] = cls
        else:
            srv = serve.RelightServer(e, frames, base, **kw)
            st = srv.run(reqs)
            st.update({"quanta": srv.quanta, "max_concurrent": srv.max_active,
                       "classes": serve.class_latency(reqs, frame_px)})
        if first:
            clocks = sampler.stop()
        st.update({"kernel_evals_per_s_1080p": rate,
                   "offered_evals_per_s": sum(frame_px[r.res] * r.K for r in reqs) / reqs[-1].arrival})
        out[name] = st
        if name == "served_bf16" and args.serve_serial_prefix > 0 and world == 1:
            m = args.serve_serial_prefix
            prefix = serve.make_stream(m, args.serve_rate, seed=0, face_size=S)
            st2 = serve.RelightServer(e, frames, base, precision="bf16", quantum_ms=args.serve_quantum_ms,
                                      est_evals_per_s=rate).run(prefix)
            out["served_bf16_prefix"] = st2
            prefix = serve.make_stream(m, args.serve_rate, seed=0, face_size=S)
            out["serial_fp32_prefix"] = serve.serve_serial(e, frames, base, prefix, precision="fp32")
        e.close()
        del frames, base
        torch.cuda.empty_cache()
    if rank == 0:
        s_ = out.get("served_bf16") or out["served_bf16_small_net"]
        line = {"metric": f"p99 relight latency, {args.serve_requests} requests Poisson {args.serve_rate:g}/s",
                "value": s_["p99_ms"], "unit": "ms", "n_gpus": world, "steps": 1, "warmup": 0,
                "ms_per_step": s_["makespan_s"] * 1e3, "higher_is_better": False, "scaling": "strong",
                "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
                "config": {"workload": "serving stream: resolutions {256^2, 512^2, 720p, 1080p, 1440p}, "
                                       "K in {64,128,300}, 40% new 6x64x64 env maps, 60% rotations, "
                                       f"150 GB admission budget, {args.serve_quantum_ms:g} ms quanta, "
                                       f"order {args.serve_order}",
                           "networks": args.serve_nets,
                           "parallelism": f"request-dp{world} with row-band splits" if world > 1 else "1 GPU"},
                "clocks": clocks, **out}
        print(json.dumps(line), flush=True)
    if channels is not None:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------- precision sweep

def run_sweep(args, rank, world, local, dev):
    """Config-3 precision sweep: the 1080p frame relit at K in {128, 300, 512} in BF16, FP8
    (E4M3, per-layer scales) and FP32; per K, throughput and max / mean relative error and
    PSNR against the FP64 oracle of the same network and weights on a pixel sample spread
    over the frame.  The FP8 scales come from one seeded calibration batch (a separate
    256x256 synthetic G-buffer relit with the K=300 env map) and stay fixed for every K."""
    import torch
    from neural_wavelet_prt_demo_b200 import engine as eng
    from oracle import oracle as O
    desc, w, gb, faces = make_relight_inputs(rank)
    e = eng.RenderEngine(netconfig_json(), device=local)
    e.loadWeights(w)
    fr = eng.FullFrame.from_gbuffer(gb, dev)
    e.setFrame(0, fr)
    e.TCNNPass_p1(0)
    b = O.Bound(desc, w, gb)
    N = gb.n
    # sample: args.sweep_px pixels in 16 contiguous runs spread over the frame
    runs, per = 16, max(1, args.sweep_px // 16)
    starts = [int(i * (N - per) / (runs - 1)) for i in range(runs)]
    res = {}
    from neural_wavelet_prt_demo_b200 import synth
    cal = eng.FullFrame.from_gbuffer(synth.make_gbuffer(256, 256, seed=7), dev)
    e.setFrame(1, cal)
    e.TCNNPass_p1(1)
    cal_env = e.addEnvironmentMap(eng.EnvironmentMap(faces), K=300)
    amax = e.calibrateFP8(cal_env, 1)
    e.releaseEnvironmentMap(cal_env)
    for K in (128, 300, 512):
        env = e.addEnvironmentMap(eng.EnvironmentMap(faces), K=K)
        idx, st = e.envWavelets(env)
        ref = np.concatenate([O.relight_f64(b, idx, st, px_begin=s, px_end=s + per) for s in starts])
        sel = np.concatenate([np.arange(s, s + per) for s in starts])
        row = {}
        for prec in ("bf16", "fp8", "fp32"):
            cfg = eng.RenderConfig(precision=prec)
            e.TCNNPass_p2(env, 0, cfg)
            torch.cuda.synchronize()
            a, bb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            e.TCNNPass_p2(env, 0, cfg)
            bb.record()
            torch.cuda.synchronize()
            ms = a.elapsed_time(bb)
            got = fr.fbPredictedIndirect[torch.from_numpy(sel).to(dev)][:, :3].double().cpu().numpy()
            floor = 1e-6 * np.abs(ref).max()
            rel = np.abs(got - ref) / np.maximum(np.abs(ref), floor)
            mse = float(np.mean((got - ref) ** 2))
            row[prec] = {"ms": ms, "evals_per_s": N * K / (ms / 1e3),
                         "max_rel_err": float(rel.max()), "mean_rel_err": float(rel.mean()),
                         "psnr_db": 10 * np.log10(np.abs(ref).max() ** 2 / mse) if mse > 0 else float("inf")}
        row["fp8_e4m3"] = row.pop("fp8")
        res[f"K{K}"] = row
    e.close()
    if rank == 0:
        print(json.dumps({"metric": "precision sweep at 1920x1080 vs FP64 oracle", "value": res["K300"]["bf16"]["psnr_db"],
                          "unit": "dB (BF16 PSNR at K=300)", "n_gpus": world, "higher_is_better": True,
                          "data": "synthetic", "config": {"workload": "relight 1920x1080, K in {128,300,512}",
                                                          "oracle_pixels_per_K": runs * per,
                                                          "fp8_calibration": "256x256 G-buffer seed 7, K=300",
                                                          "fp8_layer_amax": [float(x) for x in amax]},
                          "sweep": res}),
              flush=True)


# ---------------------------------------------------------------------------- reference arm

def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    from neural_wavelet_prt_demo_b200 import netconfig
    desc, w, gb, faces = make_relight_inputs(0)
    idx, st = O.haar_topk(faces, K_WAVELETS)
    per_step = max(1.0, 150.0 / (args.steps + args.warmup))
    rate0, cores, n_px, _ = cpu_relight_rate(desc, w, gb, idx, st, per_step)
    b = O.Bound(desc, w, gb)
    mid = gb.n // 2
    for _ in range(args.warmup):
        O.relight_f32(b, idx, st, px_begin=mid, px_end=mid + n_px, n_threads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.relight_f32(b, idx, st, px_begin=mid, px_end=mid + n_px, n_threads=cores)
    dt = (time.perf_counter() - t0) / args.steps
    rate = n_px * K_WAVELETS / dt
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": relight_config(world, sum(a.nbytes for a in gb.arrays())),
            "cpu_baseline": {"value": rate, "unit": "evals/s", "cores": cores, "kind": "port",
                             "sample": f"{n_px} contiguous pixels of the frame x K={K_WAVELETS} per step, "
                                       "FP32 oracle (the reference's relight math restated; tiny-cuda-nn "
                                       "absent), scaled to evals/s"},
            "e2e": {"value": rate, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def launch_ranks(n: int) -> None:
    """Re-executes this command under torch.distributed.run with one process per GPU when
    --gpus N > 1 is given without a launcher; a launcher whose world size differs from N
    is an error (a run must never report fewer GPUs than it was asked for)."""
    if "WORLD_SIZE" in os.environ:
        world = int(os.environ["WORLD_SIZE"])
        if world != n:
            sys.exit(f"bench.py: --gpus {n} but the launcher started {world} ranks")
        return
    if n <= 1:
        return
    import socket
    with socket.socket() as s_:
        s_.bind(("127.0.0.1", 0))
        port = s_.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__),
           *sys.argv[1:]]
    os.execv(sys.executable, cmd)


def main():
    args = parse_args()
    if args.gpus < 1:
        sys.exit("bench.py: --gpus must be >= 1")
    if args.impl == "ours" and "WORLD_SIZE" not in os.environ and args.gpus > 1:
        import torch
        if torch.cuda.device_count() < args.gpus:
            sys.exit(f"bench.py: --gpus {args.gpus} but {torch.cuda.device_count()} CUDA devices are visible")
    launch_ranks(args.gpus)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

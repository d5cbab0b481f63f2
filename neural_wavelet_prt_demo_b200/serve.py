"""Continuous-batching relight server.

Requests of mixed resolution, K and env map arrive over time.  The server keeps the
network weights and the G-buffers of every resolution resident in HBM, admits requests
while a device-memory budget allows (their output buffers and env tables), and feeds the
GPU fixed-size *quanta* of work: each quantum is one ``nwprt_relight_ranges`` launch that
packs 128-pixel-aligned pixel ranges of several admitted requests, earliest deadline first
(``order="edf"``, the default: a deadline proportional to each request's own size, so small
requests are not queued behind large ones), in arrival order (``order="fifo"``) or smallest
remaining work first (``order="srpt"``).  Requests that arrive while
quanta are running join the next quantum, and two quanta are kept in flight so the GPU does
not idle while the host forms the next one.

Each request's env map is either new cubemap faces (Haar + top-K on the GPU) or a
rotation of a resident map (``env_rotate`` then Haar + top-K), stream-ordered ahead of
the request's first quantum.  The reference renders one frame at a time behind a 2-frame
ping-pong (Renderer/OutputVisualizer.cpp:61-126); this generalises that overlap to many
concurrent requests.

Failures stay with the request that caused them.  A request with malformed fields (no such
frame, K out of range, faces of the wrong shape, a non-finite rotation) is refused at
admission with status "error"; so is one whose set-up raises (an allocation failure, for
instance).  If a quantum's launch fails, its ranges are relaunched one request at a time and
only the requests that still fail are ended.  An optional ``fault`` hook injects such
failures on the host for testing: it is called with (request, stage) at "arrive" (return
"drop" to lose the request in transit: status "dropped"), "admit" and "launch" (raise to
fail the request there).  No failure is ever injected on the GPU.

``plan_quantum`` / ``Admission`` / ``validate_request`` are pure host logic (tested on CPU);
``RelightServer`` drives the GPU.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable, Deque, Dict, List, Optional, Sequence, Tuple

import numpy as np

TILE = 128          # pixels per tensor-core tile; quanta split requests on tile boundaries
OUT_BYTES_PER_PX = 32  # two float4 outputs


# ---------------------------------------------------------------------------- requests

@dataclass
class Request:
    rid: int
    arrival: float            # seconds after the stream starts
    res: int                  # index of the resident frame (resolution)
    K: int                    # wavelets
    env_kind: str             # "new" (faces given) or "rot" (rotation of a resident env map)
    faces: Optional[np.ndarray] = None   # [6,S,S,3] for "new"
    base_env: int = -1                   # resident env index for "rot"
    R: Optional[np.ndarray] = None       # 3x3 rotation for "rot"
    # a row band of the frame: pixels [px_lo, px_hi) (px_hi <= 0: to the end of the frame);
    # multi-GPU serving splits large requests into one band per rank (dispatch.py)
    px_lo: int = 0
    px_hi: int = 0
    owner: int = 0            # rank that reports the request (and gathers its bands)
    split: bool = False       # one band of a request split across ranks
    # filled by the server (max_queue_s: longest a request may wait for admission)
    n_px: int = 0
    next_px: int = 0
    status: str = "pending"   # pending -> queued -> active -> done | rejected | timeout | error | dropped
    t_admit: float = math.nan
    t_done: float = math.nan
    env_id: int = -1
    bytes_held: int = 0
    outputs: Tuple = ()

    @property
    def remaining_evals(self) -> int:
        return (self.n_px - self.next_px) * self.K

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


def validate_request(r: Request, n_res: int, face_size: int, n_base: int) -> None:
    """Raises ValueError when the request cannot be served as given."""
    if not math.isfinite(r.arrival):
        raise ValueError(f"request {r.rid}: arrival time is not finite")
    if not 0 <= r.res < n_res:
        raise ValueError(f"request {r.rid}: no resident frame {r.res}")
    if not 1 <= r.K <= min(1024, 6 * face_size * face_size):
        raise ValueError(f"request {r.rid}: K={r.K} outside [1, {min(1024, 6 * face_size * face_size)}]")
    if r.env_kind == "new":
        if r.faces is None or np.shape(r.faces) != (6, face_size, face_size, 3):
            raise ValueError(f"request {r.rid}: env faces must be [6, {face_size}, {face_size}, 3]")
    elif r.env_kind == "rot":
        if not 0 <= r.base_env < n_base:
            raise ValueError(f"request {r.rid}: no resident env map {r.base_env}")
        R = None if r.R is None else np.asarray(r.R, np.float64)
        if R is None or R.shape != (3, 3) or not np.all(np.isfinite(R)):
            raise ValueError(f"request {r.rid}: rotation must be a finite 3x3 matrix")
    else:
        raise ValueError(f"request {r.rid}: unknown env kind {r.env_kind!r}")


def request_bytes(n_px: int, K: int, face_size: int, enc_dims: int) -> int:
    """Device bytes a request holds while admitted: outputs, env table, rotated faces."""
    return n_px * OUT_BYTES_PER_PX + K * (4 + 12 + 4 * enc_dims) + 6 * face_size * face_size * 12


class Admission:
    """Admits queued requests first-come first-served while the byte budget allows."""

    def __init__(self, budget_bytes: int):
        self.budget = int(budget_bytes)
        self.used = 0

    def fits(self, nbytes: int) -> bool:
        return self.used + nbytes <= self.budget

    def take(self, nbytes: int) -> None:
        if not self.fits(nbytes):
            raise RuntimeError("admission over budget")
        self.used += nbytes

    def give(self, nbytes: int) -> None:
        self.used -= nbytes
        assert self.used >= 0


def deadline(r: Request, evals_per_s: float, slack: float = 4.0, floor_s: float = 0.016) -> float:
    """Target completion time of a request for earliest-deadline-first packing: its arrival
    plus `slack` times its own service time alone (pixels x K at `evals_per_s`), and never
    less than `floor_s` -- small requests get tight deadlines, large ones loose ones."""
    px = (r.n_px - max(0, r.px_lo)) if r.n_px else 0
    return r.arrival + max(floor_s, slack * px * r.K / evals_per_s)


def plan_quantum(active: Sequence[Request], quantum_evals: int, order: str = "srpt",
                 evals_per_s: float = 1e10) -> List[Tuple[Request, int, int]]:
    """Chunks for one launch: requests in order of least remaining work ("srpt"), of
    arrival ("fifo") or of deadline ("edf", see ``deadline``), each chunk a 128-pixel-aligned
    range, until the quantum is full.  Always makes progress: the first request gets at
    least one tile even if that alone exceeds the quantum."""
    if order not in ("srpt", "fifo", "edf"):
        raise ValueError(f"unknown quantum order {order!r}")
    if order == "srpt":
        key = lambda r: (r.remaining_evals, r.rid)
    elif order == "fifo":
        key = lambda r: (r.arrival, r.rid)
    else:
        key = lambda r: (deadline(r, evals_per_s), r.rid)
    plan = []
    used = 0
    for r in sorted((r for r in active if r.next_px < r.n_px), key=key):
        room = quantum_evals - used
        if room <= 0 and plan:
            break
        tiles = max(1, room // (TILE * r.K))
        end = min(r.n_px, r.next_px + tiles * TILE)
        if end <= r.next_px:
            continue
        plan.append((r, r.next_px, end))
        used += (end - r.next_px) * r.K
    return plan


def percentile(xs: Sequence[float], q: float) -> float:
    if not len(xs):
        return math.nan
    return float(np.percentile(np.asarray(xs, np.float64), q))


# ---------------------------------------------------------------------------- stream

RESOLUTIONS = [(256, 256), (512, 512), (1280, 720), (1920, 1080), (2560, 1440)]
KS = [64, 128, 300]


def random_rotation(g: np.random.Generator) -> np.ndarray:
    """Uniform rotation from a uniform unit quaternion (Shoemake's method)."""
    u1, u2, u3 = g.uniform(size=3)
    q = np.array([math.sqrt(1 - u1) * math.sin(2 * math.pi * u2), math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
                  math.sqrt(u1) * math.sin(2 * math.pi * u3), math.sqrt(u1) * math.cos(2 * math.pi * u3)])
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]], np.float32)


def make_stream(n: int, rate: float, seed: int = 0, face_size: int = 64, p_new: float = 0.4,
                n_base_envs: int = 8, resolutions=RESOLUTIONS, ks=KS) -> List[Request]:
    """The serving workload: Poisson arrivals at `rate`/s, resolution and K uniform,
    `p_new` new log-normal env maps, the rest random rotations of resident maps."""
    from .synth import make_env_faces
    g = np.random.Generator(np.random.PCG64([seed, 77]))
    t = 0.0
    out = []
    for i in range(n):
        t += g.exponential(1.0 / rate)
        res = int(g.integers(len(resolutions)))
        K = int(ks[int(g.integers(len(ks)))])
        if g.uniform() < p_new:
            faces = make_env_faces(face_size, seed=seed, index=1000 + i)
            out.append(Request(i, t, res, K, "new", faces=faces))
        else:
            out.append(Request(i, t, res, K, "rot", base_env=int(g.integers(n_base_envs)), R=random_rotation(g)))
    return out


# ---------------------------------------------------------------------------- GPU server

class LocalCompletion:
    """What happens when a request's last quantum has run: on one GPU, it is done.  The
    multi-GPU dispatcher (dispatch.BandGather) replaces it so that bands of split requests
    are gathered before the request counts as done."""

    def admitted(self, r: "Request") -> None:
        pass

    def finished(self, r: "Request") -> bool:
        """The request's local work has run; True if it is complete now."""
        return True

    def failed(self, r: "Request") -> None:
        """The request ended without its local work (refused, timed out or failed)."""

    def poll(self) -> List["Request"]:
        """Requests that completed since the last call through events outside this server."""
        return []

    def outstanding(self) -> bool:
        return False


class _HostEvent:
    """Stand-in for a CUDA event when the server drives a CPU engine (tests)."""

    def record(self, stream=None):
        pass

    def synchronize(self):
        pass


class RelightServer:
    """Serves a list of requests in real time on one GPU through one RenderEngine."""

    def __init__(self, engine, frames, base_faces, precision: str = "bf16", budget_bytes: int = 150 << 30,
                 quantum_ms: float = 12.0, est_evals_per_s: float = 9e9, max_queue_s: float = math.inf,
                 max_in_flight: int = 2, keep_outputs: bool = False,
                 fault: Optional[Callable[[Request, str], Optional[str]]] = None,
                 max_active: Optional[int] = None, order: str = "edf", completion=None):
        import torch
        self.torch = torch
        self.e = engine
        self.frames = frames            # resident FullFrame per resolution index (TCNNPass_p1 done)
        self.base_faces = base_faces    # device faces of the resident env maps, [6,S,S,3] each
        from .engine import RenderConfig
        self.cfg = RenderConfig(precision=precision)
        self.adm = Admission(budget_bytes)
        self.rate = est_evals_per_s
        self.quantum = int(est_evals_per_s * quantum_ms / 1e3)
        self.max_queue_s = max_queue_s
        self.max_in_flight = max_in_flight
        # admission also stops at max_active admitted requests (None: the byte budget alone)
        self.max_active_cap = max_active
        self.order = order  # quantum packing order: "srpt" (least remaining work) or "fifo"
        self.keep_outputs = keep_outputs
        self.fault = fault
        self.completion = completion or LocalCompletion()
        self.on_gpu = frames[0].fbPredictedIndirect.is_cuda
        self.stream = torch.cuda.current_stream() if self.on_gpu else None
        info = engine.networkInfo()
        self.face_size, self.enc_dims = info.face_size, info.enc_dims
        self.quanta = 0
        self.max_active = 0
        # pinned staging buffers for new env maps, reused round robin (a pinned allocation per
        # request costs milliseconds of host time, which the launch loop cannot spare); each
        # buffer's event marks its last upload as done before the buffer is overwritten
        # output buffers of retired requests, per resolution, handed to the next admitted
        # request of that resolution (with hundreds of requests admitted, fresh frame-sized
        # allocations fall through the caching allocator to cudaMalloc)
        self._out_pool: Dict[int, List] = {}
        self._staging: List = []
        self._staging_ev: List = []
        self._staging_next = 0

    def _prepare(self, r: Request) -> None:
        """Output buffers and the env wavelet table, stream-ordered before its first quantum."""
        torch = self.torch
        fr = self.frames[r.res]
        # outputs are indexed by absolute pixel: a band's buffer covers the whole frame, which
        # also lets a split request's owner receive the other ranks' bands into it
        pool = self._out_pool.setdefault(r.res, [])
        if pool:
            ind, wd = pool.pop()
        else:
            ind = torch.empty((fr.width * fr.height, 4), dtype=torch.float32, device=fr.fbPredictedIndirect.device)
            wd = torch.empty_like(ind)
        if r.env_kind == "new":
            host = torch.from_numpy(np.ascontiguousarray(r.faces, np.float32))
            if self.on_gpu:
                # through pinned memory: a copy from pageable memory may wait for the stream,
                # i.e. for the launches already queued
                faces = self._upload_pinned(host, ind.device)
            else:
                faces = host.to(ind.device)
        elif r.env_kind == "rot":
            from .engine import env_rotate
            faces = env_rotate(self.base_faces[r.base_env], r.R)
        else:
            raise ValueError(f"unknown env kind {r.env_kind!r}")
        r.env_id = self.e.addEnvironmentFaces(faces, r.K)
        r.outputs = (ind, wd, faces)

    STAGING_BUFFERS = 32
    ADMIT_SLICE_S = 0.002  # host time spent admitting before a free launch slot is filled

    def _upload_pinned(self, host, device):
        """Copies host faces to a new device tensor through the reused pinned staging pool."""
        torch = self.torch
        i = self._staging_next
        self._staging_next = (i + 1) % self.STAGING_BUFFERS
        if i >= len(self._staging):
            self._staging.append(torch.empty(host.shape, dtype=torch.float32, pin_memory=True))
            self._staging_ev.append(None)
        buf = self._staging[i]
        if buf.shape != host.shape:
            buf = self._staging[i] = torch.empty(host.shape, dtype=torch.float32, pin_memory=True)
            self._staging_ev[i] = None
        if self._staging_ev[i] is not None:
            self._staging_ev[i].synchronize()  # the upload 32 requests ago: long complete
        buf.copy_(host)
        faces = buf.to(device, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(self.stream)
        self._staging_ev[i] = ev
        return faces

    def _end_failed(self, r: Request, t: float) -> None:
        """Ends a request that failed after admission: returns its budget and env table."""
        r.status, r.t_done = "error", t
        self.completion.failed(r)
        if r.bytes_held:
            self.adm.give(r.bytes_held)
            r.bytes_held = 0
        if r.env_id >= 0:
            try:
                self.e.releaseEnvironmentMap(r.env_id)
            except Exception:
                pass  # an env id the request itself corrupted
            r.env_id = -1
        r.outputs = ()

    def _launch(self, ranges_by_req: List[Tuple[Request, Tuple]]) -> List[Request]:
        """One relight launch for the quantum; if it fails, one launch per request.  Returns
        the requests whose ranges failed even alone."""
        try:
            self.e.relightRanges([rg for _, rg in ranges_by_req], self.cfg)
            return []
        except Exception:
            failed = []
            for r, rg in ranges_by_req:
                try:
                    self.e.relightRanges([rg], self.cfg)
                except Exception:
                    failed.append(r)
            return failed

    def _retire(self, r: Request, t: float) -> None:
        """A request whose work (and gather) is complete: returns its budget and env table."""
        r.status, r.t_done = "done", t
        self.adm.give(r.bytes_held)
        r.bytes_held = 0
        self.e.releaseEnvironmentMap(r.env_id)
        r.env_id = -1
        if not self.keep_outputs:
            # the request's last launch has completed (its event was waited for)
            if r.outputs:
                self._out_pool.setdefault(r.res, []).append((r.outputs[0], r.outputs[1]))
            r.outputs = ()

    def _refuse(self, r: Request, status: str, t: float) -> None:
        r.status, r.t_done = status, t
        self.completion.failed(r)

    def run(self, requests: List[Request], realtime: bool = True, t0: Optional[float] = None) -> Dict:
        """Serves `requests` (arrival times in seconds after t0, default: now)."""
        torch = self.torch
        pending: Deque[Request] = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        queue: Deque[Request] = deque()
        active: List[Request] = []
        gathering: List[Request] = []
        in_flight: Deque[Tuple] = deque()
        for r in requests:
            ok = isinstance(r.res, (int, np.integer)) and 0 <= r.res < len(self.frames)
            full = self.frames[r.res].width * self.frames[r.res].height if ok else 0
            r.n_px = min(r.px_hi, full) if r.px_hi > 0 else full
            r.next_px = max(0, r.px_lo)
            r.status = "pending"
        t0 = time.perf_counter() if t0 is None else t0
        now = lambda: time.perf_counter() - t0
        finished = 0
        total = len(requests)
        busy_ms = 0.0  # device time of the relight launches
        host = {"admit": 0.0, "plan": 0.0, "launch": 0.0, "wait": 0.0}  # host seconds per phase
        starved = 0  # launches issued with nothing left queued on the GPU
        # transfers of refused or failed bands may still be queued once every request has
        # ended here: the loop runs until the completion has nothing outstanding either
        while finished < total or self.completion.outstanding():
            for r in self.completion.poll():
                gathering.remove(r)
                self._retire(r, now())
                finished += 1
            t = now() if realtime else math.inf
            while pending and pending[0].arrival <= t:
                r = pending.popleft()
                if self.fault is not None and self.fault(r, "arrive") == "drop":
                    self._refuse(r, "dropped", now())
                    finished += 1
                    continue
                r.status = "queued"
                queue.append(r)
            # admission (FCFS under the byte budget; over-budget and stale requests are refused)
            t_ph = time.perf_counter()
            while queue and (self.max_active_cap is None or len(active) < self.max_active_cap):
                # a launch slot is free and work is admitted: launch before admitting more, so a
                # burst of arrivals does not leave the GPU without queued work
                if (active and len(in_flight) < self.max_in_flight
                        and time.perf_counter() - t_ph > self.ADMIT_SLICE_S):
                    break
                r = queue[0]
                try:
                    validate_request(r, len(self.frames), self.face_size, len(self.base_faces))
                except ValueError:
                    queue.popleft()
                    self._refuse(r, "error", now())
                    finished += 1
                    continue
                fr = self.frames[r.res]
                nbytes = request_bytes(fr.width * fr.height, r.K, self.face_size, self.enc_dims)
                if nbytes > self.adm.budget:
                    queue.popleft()
                    self._refuse(r, "rejected", now())
                    finished += 1
                    continue
                if not self.adm.fits(nbytes):
                    if realtime and now() - r.arrival > self.max_queue_s:
                        queue.popleft()
                        self._refuse(r, "timeout", now())
                        finished += 1
                        continue
                    break
                queue.popleft()
                try:
                    if self.fault is not None:
                        self.fault(r, "admit")
                    self._prepare(r)
                except Exception:
                    self._end_failed(r, now())
                    finished += 1
                    continue
                self.adm.take(nbytes)
                r.bytes_held = nbytes
                r.status, r.t_admit = "active", now()
                self.completion.admitted(r)
                active.append(r)
            self.max_active = max(self.max_active, len(active))
            host["admit"] += time.perf_counter() - t_ph
            if active and len(in_flight) < self.max_in_flight:
                t_ph = time.perf_counter()
                plan = plan_quantum(active, self.quantum, self.order, self.rate)
                host["plan"] += time.perf_counter() - t_ph
                launch = []
                for r, b, e in plan:
                    try:
                        if self.fault is not None:
                            self.fault(r, "launch")
                    except Exception:
                        active.remove(r)
                        self._end_failed(r, now())
                        finished += 1
                        continue
                    launch.append((r, (r.env_id, r.res, r.outputs[0], r.outputs[1], b, e), e))
                if not launch:
                    continue
                t_ph = time.perf_counter()
                if self.on_gpu:
                    torch.cuda.nvtx.range_push(f"quantum {self.quanta}: {len(launch)} requests")
                    ev0 = torch.cuda.Event(enable_timing=True)
                    ev0.record(self.stream)
                    if self.quanta and (not in_flight or in_flight[-1][1].query()):
                        starved += 1
                else:
                    ev0 = None
                failed = self._launch([(r, rg) for r, rg, _ in launch])
                if self.on_gpu:
                    torch.cuda.nvtx.range_pop()
                for r in failed:
                    active.remove(r)
                    self._end_failed(r, now())
                    finished += 1
                for r, _, e in launch:
                    if r.status == "active":
                        r.next_px = e
                ev = torch.cuda.Event(enable_timing=True) if self.on_gpu else _HostEvent()
                ev.record(self.stream)
                done_now = [r for r, _, _ in launch if r.status == "active" and r.next_px >= r.n_px]
                for r in done_now:
                    active.remove(r)
                in_flight.append((ev0, ev, done_now))
                self.quanta += 1
                host["launch"] += time.perf_counter() - t_ph
                continue
            if in_flight:
                ev0, ev, done_now = in_flight.popleft()
                t_ph = time.perf_counter()
                ev.synchronize()
                host["wait"] += time.perf_counter() - t_ph
                if ev0 is not None:
                    busy_ms += ev0.elapsed_time(ev)
                t = now()
                for r in done_now:
                    if self.completion.finished(r):
                        self._retire(r, t)
                        finished += 1
                    else:
                        r.status = "gathering"
                        gathering.append(r)
                continue
            if pending or self.completion.outstanding():
                if realtime and pending:
                    dt = pending[0].arrival - now()
                    if dt > 0:
                        time.sleep(min(dt, 0.002))
                elif self.completion.outstanding():
                    time.sleep(0.0002)
                continue
            if queue:  # nothing active, nothing in flight, but the head does not fit: cannot happen
                raise RuntimeError("admission stalled")
        self.e.TCNNSync()
        out = summarize(requests, now())
        if self.on_gpu and out["makespan_s"] > 0:
            # share of the run the GPU spent in relight launches (the rest: idle or env set-up)
            out["relight_busy_frac"] = busy_ms / 1e3 / out["makespan_s"]
            out["host_s"] = {k: round(v, 3) for k, v in host.items()}
            out["launches_after_idle"] = starved
        return out


# latency classes of the serving stream: resolutions up to 1280x720, and larger ones
SMALL_CLASS_MAX_PX = 1280 * 720


def class_latency(requests: Sequence[Request], frame_px: Sequence[int]) -> Dict:
    """p50 / p99 of the finished requests per class (small: <= 720p frames, large: above)."""
    out = {}
    for name, pick in (("small", lambda n: n <= SMALL_CLASS_MAX_PX), ("large", lambda n: n > SMALL_CLASS_MAX_PX)):
        lat = [r.latency * 1e3 for r in requests if r.status == "done" and pick(frame_px[r.res])]
        out[name] = {"done": len(lat), "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99)}
    return out


def summarize(requests: Sequence[Request], makespan: float) -> Dict:
    done = [r for r in requests if r.status == "done"]
    lat = [r.latency * 1e3 for r in done]
    evals = sum((r.n_px - max(0, r.px_lo)) * r.K for r in done)
    return {
        "requests": len(requests),
        "done": len(done),
        "rejected": sum(r.status == "rejected" for r in requests),
        "timeout": sum(r.status == "timeout" for r in requests),
        "error": sum(r.status == "error" for r in requests),
        "dropped": sum(r.status == "dropped" for r in requests),
        "makespan_s": makespan,
        "evals_per_s": evals / makespan if makespan > 0 else math.nan,
        "p50_ms": percentile(lat, 50),
        "p99_ms": percentile(lat, 99),
        "max_ms": max(lat) if lat else math.nan,
    }


def serve_serial(engine, frames, base_faces, requests: List[Request], precision: str = "fp32",
                 realtime: bool = True) -> Dict:
    """Baseline: one request at a time in arrival order, each a whole-frame relight."""
    import torch
    from .engine import RenderConfig, env_rotate
    cfg = RenderConfig(precision=precision)
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0
    for r in sorted(requests, key=lambda r: (r.arrival, r.rid)):
        if realtime:
            while now() < r.arrival:
                time.sleep(min(r.arrival - now(), 0.002))
        fr = frames[r.res]
        r.n_px = fr.width * fr.height
        if r.env_kind == "new":
            faces = torch.from_numpy(np.ascontiguousarray(r.faces, np.float32)).to(fr.fbPredictedIndirect.device)
        else:
            faces = env_rotate(base_faces[r.base_env], r.R)
        env = engine.addEnvironmentFaces(faces, r.K)
        out = torch.empty((r.n_px, 4), dtype=torch.float32, device=faces.device)
        out2 = torch.empty_like(out)
        engine.relightRanges([(env, r.res, out, out2, 0, r.n_px)], cfg)
        torch.cuda.synchronize()
        r.status, r.t_done = "done", now()
        r.outputs = (out, out2, faces)
        engine.releaseEnvironmentMap(env)
    engine.TCNNSync()
    return summarize(requests, now())

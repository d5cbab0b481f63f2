"""Multi-GPU serving: one process, one library context and one ``RelightServer`` per GPU.

The relight path has no collective on its data path (pixels and requests are independent
given the resident weights, G-buffers and env tables), so GPUs split *work*:

* Placement (``sharding.assign_online``): every rank derives the same plan from the request
  stream alone.  A request goes to the rank whose estimated backlog lets it start first; a
  request of at least ``split_min_evals`` pixel*wavelet evaluations (a 1080p or 1440p frame at
  K=300) is split into one row band per rank, so that one large frame is relit by every GPU
  at once and its latency shrinks with the number of GPUs.
* Each rank serves its own requests and its band of every split request with the
  single-GPU server (continuous batching, byte-budget admission, two launches in flight);
  each band is written into that rank's own HBM.
* Gather (``BandGather``): a finished band goes to the request's owner with point-to-point
  sends (NCCL on GPUs, gloo on CPU) -- never by a load from a peer's memory.  Per pair of
  ranks, sends and receives are posted in request-id order, so every send meets its receive
  (NCCL requires the same order on both sides).  A band whose rank refused or failed it is
  still sent, with a failure flag, and an owner that refused or failed its own part still
  receives every band (into scratch memory), so a failure never leaves a send unmatched.
  The owner reports the request when its own band and all received bands are complete.

The reference renders on one GPU (Renderer/OptixBackend.h:90); its only split is the
per-row loop over four streams inside TCNNPass_p2 (Renderer/tinycudann/tcnn.cu:127-134).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Optional, Sequence, Tuple

from .serve import LocalCompletion, Request, RelightServer, percentile
from .sharding import assign_online, request_cost, row_band

# a 1080p frame at K=300 (6.2e8 evaluations) and everything larger is split across ranks
DEFAULT_SPLIT_MIN_EVALS = 1920 * 1080 * 300


def plan_stream(requests: Sequence[Request], frame_dims: Sequence[Tuple[int, int]], world: int,
                evals_per_s: float, split_min_evals: Optional[int] = DEFAULT_SPLIT_MIN_EVALS
                ) -> List[Tuple[int, bool]]:
    """(owner, split) for every request, in the order given (sorted by arrival here)."""
    order = sorted(range(len(requests)), key=lambda i: (requests[i].arrival, requests[i].rid))
    arrivals = [requests[i].arrival for i in order]
    costs = [request_cost(*frame_dims[requests[i].res], requests[i].K) for i in order]
    heights = [frame_dims[requests[i].res][1] for i in order]
    placed = assign_online(arrivals, costs, world, evals_per_s, split_min_evals, heights)
    out: List[Tuple[int, bool]] = [(0, False)] * len(requests)
    for i, p in zip(order, placed):
        out[i] = p
    return out


def local_requests(requests: Sequence[Request], plan: Sequence[Tuple[int, bool]],
                   frame_dims: Sequence[Tuple[int, int]], rank: int, world: int) -> List[Request]:
    """This rank's work: the whole requests placed on it, and its row band of every split
    request (pixels [row_begin * W, row_end * W) of the frame)."""
    mine = []
    for r, (owner, split) in zip(requests, plan):
        if split:
            W, H = frame_dims[r.res]
            b, e = row_band(H, rank, world)
            mine.append(dataclasses.replace(r, px_lo=b * W, px_hi=e * W, owner=owner, split=True))
        elif owner == rank:
            mine.append(dataclasses.replace(r, owner=owner, split=False))
    return mine


class _Transfer:
    """A posted send or receive that can be polled.  NCCL's work objects report completion
    through a CUDA event (``is_completed``); gloo's complete only inside ``wait``, so on CPU
    ranks a helper thread waits and raises a flag."""

    def __init__(self, work, threaded: bool):
        self.work = work
        self.ok = True
        self.flag = None
        if threaded:
            import threading
            self.flag = threading.Event()
            threading.Thread(target=self._wait, daemon=True).start()

    def _wait(self):
        try:
            self.work.wait()
        except Exception:
            self.ok = False
        finally:
            self.flag.set()

    def is_completed(self) -> bool:
        return self.flag.is_set() if self.flag is not None else self.work.is_completed()


class PairChannels:
    """One process group per direction of every pair of ranks, for the band transfers.

    Point-to-point operations of one communicator run in order (NCCL); if rank a's send to
    b and b's send to a shared a communicator, a send posted before a receive on both sides
    could wait on each other forever.  With one communicator per direction, the only order
    that matters is the one ``BandGather`` keeps: request-id order, on both ends.  Every rank
    must construct this at the same point (process-group creation is collective)."""

    def __init__(self, world: int):
        import torch.distributed as dist
        self.dist = dist
        self.threaded = dist.get_backend() == "gloo"
        self.groups = {}
        for a in range(world):
            for b in range(a + 1, world):
                self.groups[(a, b)] = dist.new_group([a, b])
                self.groups[(b, a)] = dist.new_group([a, b])

    def isend(self, t, src: int, dst: int) -> _Transfer:
        return _Transfer(self.dist.isend(t, dst=dst, group=self.groups[(src, dst)]), self.threaded)

    def irecv(self, t, src: int, dst: int) -> _Transfer:
        return _Transfer(self.dist.irecv(t, src=src, group=self.groups[(src, dst)]), self.threaded)


class BandGather(LocalCompletion):
    """Completion of split requests across ranks (see the module docstring).

    ``channels`` provides isend(t, src, dst) / irecv(t, src, dst) on a per-direction
    communicator (``PairChannels``)."""

    def __init__(self, rank: int, world: int, parts: Sequence[Request], frame_dims, channels, device):
        import torch
        self.torch = torch
        self.rank, self.world, self.ch, self.device = rank, world, channels, device
        self.frame_dims = frame_dims
        splits = sorted((r for r in parts if r.split), key=lambda r: r.rid)
        self.req = {r.rid: r for r in splits}
        # sends this rank makes, per destination owner, in request-id order
        self.send_order: Dict[int, List[int]] = {}
        # receives this rank makes as owner, per source rank, in request-id order
        self.recv_order: Dict[int, List[int]] = {}
        for r in splits:
            if r.owner == self.rank:
                for src in range(world):
                    if src != rank:
                        self.recv_order.setdefault(src, []).append(r.rid)
            else:
                self.send_order.setdefault(r.owner, []).append(r.rid)
        self.send_next = {d: 0 for d in self.send_order}
        self.recv_next = {s_: 0 for s_ in self.recv_order}
        self.send_ready: Dict[int, bool] = {}   # rid -> this rank's band outcome (True = ran)
        self.recv_ready: Dict[int, bool] = {}   # rid -> owner part outcome (True = admitted)
        self.sends: List[Tuple[Request, list, tuple]] = []   # in flight: (request, works, buffers)
        self.recvs: Dict[int, List[Tuple[list, object, tuple]]] = {}  # rid -> [(works, flag, buffers)]
        self.local: Dict[int, bool] = {}       # owner: rid -> own band ran (True) or ended (False)
        self.band_failures: Dict[int, int] = {}

    def _band(self, r: Request, src: int) -> Tuple[int, int]:
        W, H = self.frame_dims[r.res]
        b, e = row_band(H, src, self.world)
        return b * W, e * W

    def _scratch(self, n: int):
        return self.torch.zeros((n, 4), dtype=self.torch.float32, device=self.device)

    def _post(self) -> None:
        for d, order in self.send_order.items():
            while self.send_next[d] < len(order) and order[self.send_next[d]] in self.send_ready:
                rid = order[self.send_next[d]]
                r, ok = self.req[rid], self.send_ready.pop(rid)
                lo, hi = self._band(r, self.rank)
                if ok and r.outputs:
                    ind, wd = r.outputs[0][lo:hi], r.outputs[1][lo:hi]
                else:
                    ind, wd = self._scratch(hi - lo), self._scratch(hi - lo)
                flag = self.torch.tensor([1 if ok else 0], dtype=self.torch.int32, device=self.device)
                bufs = (ind, wd, flag)
                self.sends.append((r, [self.ch.isend(t, self.rank, d) for t in bufs], bufs))
                self.send_next[d] += 1
        for src, order in self.recv_order.items():
            while self.recv_next[src] < len(order) and order[self.recv_next[src]] in self.recv_ready:
                rid = order[self.recv_next[src]]
                r = self.req[rid]
                lo, hi = self._band(r, src)
                if self.recv_ready[rid] and r.outputs:
                    ind, wd = r.outputs[0][lo:hi], r.outputs[1][lo:hi]
                else:
                    ind, wd = self._scratch(hi - lo), self._scratch(hi - lo)
                flag = self.torch.zeros(1, dtype=self.torch.int32, device=self.device)
                bufs = (ind, wd, flag)
                self.recvs.setdefault(rid, []).append(([self.ch.irecv(t, src, self.rank) for t in bufs], flag, bufs))
                self.recv_next[src] += 1
        # an owner outcome is kept until every source has posted its receive
        for rid in [x for x in self.recv_ready if len(self.recvs.get(x, ())) == self.world - 1]:
            del self.recv_ready[rid]

    # ---- LocalCompletion interface
    def admitted(self, r: Request) -> None:
        if r.split and r.owner == self.rank:
            self.recv_ready[r.rid] = True
            self._post()

    def finished(self, r: Request) -> bool:
        if not r.split:
            return True
        if r.owner != self.rank:
            self.send_ready[r.rid] = True      # done once its sends are
        else:
            self.local[r.rid] = True           # done once every band has arrived
        self._post()
        return False

    def failed(self, r: Request) -> None:
        if not r.split:
            return
        if r.owner != self.rank:
            self.send_ready[r.rid] = False     # the band still goes out, flagged as failed
        else:
            if r.rid not in self.recvs:
                self.recv_ready[r.rid] = False  # receive into scratch memory
            self.local[r.rid] = False
        self._post()

    def poll(self) -> List[Request]:
        out, still = [], []
        for r, works, bufs in self.sends:
            if all(w.is_completed() for w in works):
                if r.status == "gathering":
                    out.append(r)
            else:
                still.append((r, works, bufs))
        self.sends = still
        for rid in list(self.recvs):
            parts = self.recvs[rid]
            if len(parts) < self.world - 1 or rid not in self.local:
                continue
            if not all(w.is_completed() for works, _, _ in parts for w in works):
                continue
            del self.recvs[rid]
            r = self.req[rid]
            bad = sum(int(flag.item()) == 0 or not all(w.ok for w in works) for works, flag, _ in parts)
            if self.local.pop(rid) and r.status == "gathering":
                if bad:
                    self.band_failures[rid] = bad
                out.append(r)
        return out

    def outstanding(self) -> bool:
        return bool(self.sends) or bool(self.recvs) or bool(self.send_ready) or any(
            self.send_next[d] < len(o) for d, o in self.send_order.items())


def serve_distributed(engine, frames, base_faces, requests: Sequence[Request], rank: int, world: int,
                      channels, device, evals_per_s: float,
                      split_min_evals: Optional[int] = DEFAULT_SPLIT_MIN_EVALS,
                      server_kwargs: Optional[dict] = None, realtime: bool = True) -> Dict:
    """Serves the stream with every rank's share of it (call on every rank at the same time,
    after a barrier; ``channels``: a ``PairChannels`` built on every rank).  Returns this
    rank's summary plus the latencies of the requests it owns (``latency_ms``) and
    ``local``: its Request copies (outputs kept if the server keeps them)."""
    frame_dims = [(f.width, f.height) for f in frames]
    plan = plan_stream(requests, frame_dims, world, evals_per_s, split_min_evals)
    mine = local_requests(requests, plan, frame_dims, rank, world)
    gather = BandGather(rank, world, mine, frame_dims, channels, device)
    srv = RelightServer(engine, frames, base_faces, completion=gather, **(server_kwargs or {}))
    summ = srv.run(mine, realtime=realtime)
    for r in mine:  # a split request with a band that failed on another rank failed as a whole
        if gather.band_failures.get(r.rid) and r.owner == rank:
            r.status = "error"
    owned = [r for r in mine if r.owner == rank or not r.split]
    done = [r for r in owned if r.status == "done"]
    summ["latency_ms"] = [r.latency * 1e3 for r in done]
    summ["owned"] = len(owned)
    summ["owned_done"] = len(done)
    summ["evals_done"] = sum(request_cost(*frame_dims[r.res], r.K) for r in done)
    summ["split_requests"] = sum(1 for _, s in plan if s)
    summ["local"] = mine
    return summ


def combine_summaries(summaries: Sequence[Dict], makespan_s: Optional[float] = None) -> Dict:
    """Whole-job figures from every rank's ``serve_distributed`` summary."""
    lat = [x for s in summaries for x in s["latency_ms"]]
    span = makespan_s if makespan_s is not None else max(s["makespan_s"] for s in summaries)
    evals = sum(s["evals_done"] for s in summaries)
    return {"ranks": len(summaries), "done": sum(s["owned_done"] for s in summaries),
            "requests": sum(s["owned"] for s in summaries), "split_requests": summaries[0]["split_requests"],
            "makespan_s": span, "evals_per_s": evals / span if span > 0 else math.nan,
            "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99), "max_ms": max(lat) if lat else math.nan}

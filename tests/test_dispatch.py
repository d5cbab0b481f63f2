"""Multi-GPU serving (neural_wavelet_prt_demo_b200/dispatch.py) end to end on CPU ranks.

Two gloo processes run the real dispatcher and the real serving loop; only the relight is
a stand-in (``FakeEngine``), which writes a value that depends on the env map's contents, K
and the pixel alone, so a frame assembled from bands of two ranks can be checked exactly.
Covered: the placement is the same on every rank, every request ends exactly once, split
requests are gathered whole at their owner, and failures injected on the host (a band that
fails at launch on one rank, an owner refusing its own part at admission) end those
requests without leaving any transfer unmatched."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from neural_wavelet_prt_demo_b200 import dispatch, serve, sharding

FRAMES = [(16, 8), (32, 16), (48, 24)]
FACE = 4


class FakeFrame:
    def __init__(self, w, h):
        self.width, self.height = w, h
        self.fbPredictedIndirect = torch.zeros((w * h, 4))


class FakeInfo:
    face_size, enc_dims = FACE, 16


class FakeEngine:
    def __init__(self):
        self.envs = {}
        self.next = 0

    def networkInfo(self):
        return FakeInfo()

    def addEnvironmentFaces(self, faces, K):
        self.envs[self.next] = (float(faces.double().sum()), K)
        self.next += 1
        return self.next - 1

    def releaseEnvironmentMap(self, env):
        self.envs.pop(env)

    def relightRanges(self, ranges, cfg=None):
        for env, frame, ind, wd, b, e in ranges:
            ind[b:e] = expected(self.envs[env][0], self.envs[env][1], frame, torch.arange(b, e))
            wd[b:e] = ind[b:e] + 1.0

    def TCNNSync(self):
        pass


def expected(fsum, K, frame, px):
    px = px.to(torch.float32)
    return torch.stack([px, torch.full_like(px, float(K)), torch.full_like(px, float(frame)),
                        torch.full_like(px, fsum % 1000.0)], dim=1)


def make_requests():
    return serve.make_stream(40, rate=4000.0, seed=3, face_size=FACE, p_new=1.0, resolutions=FRAMES, ks=[4, 8])


SPLIT_MIN = 32 * 16 * 8   # the two larger frames at K=8 are split


def _worker(rank, world, port, faults, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        channels = dispatch.PairChannels(world)
        frames = [FakeFrame(w, h) for w, h in FRAMES]
        reqs = make_requests()
        fault = None
        if rank in faults:
            def fault(r, stage, mine=tuple(faults[rank])):
                if ("drop", r.rid) in mine and stage == "arrive":
                    return "drop"
                if (stage, r.rid) in mine:
                    raise RuntimeError("injected")
                return None
        dist.barrier()
        summ = dispatch.serve_distributed(
            FakeEngine(), frames, [], reqs, rank, world, channels, "cpu", evals_per_s=1e6, split_min_evals=SPLIT_MIN,
            server_kwargs=dict(precision="fp32", keep_outputs=True, quantum_ms=1.0, est_evals_per_s=2e6,
                               fault=fault))
        bad = []
        owned = {}
        for r in summ["local"]:
            if r.split and r.owner != rank:
                continue
            owned[r.rid] = r.status
            if r.status != "done":
                continue
            W, H = FRAMES[r.res]
            want = expected(float(torch.from_numpy(r.faces).double().sum()), r.K, r.res, torch.arange(W * H))
            got = r.outputs[0]
            if r.split and not torch.equal(got, want):
                bad.append(r.rid)
            if not r.split and not torch.equal(got[:W * H], want):
                bad.append(r.rid)
        plan = dispatch.plan_stream(reqs, FRAMES, world, 1e6, SPLIT_MIN)
        out = [None] * world
        dist.all_gather_object(out, (owned, bad, plan, summ["owned_done"]))
        if rank == 0:
            q.put(out)
    finally:
        dist.destroy_process_group()


def _run(faults):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, faults, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = q.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=60)
    for p in procs:
        assert p.exitcode == 0
    return res


def test_assign_online_is_deterministic_and_splits_large_requests():
    reqs = make_requests()
    a = dispatch.plan_stream(reqs, FRAMES, 2, 1e6, SPLIT_MIN)
    b = dispatch.plan_stream(list(reversed(reqs)), FRAMES, 2, 1e6, SPLIT_MIN)[::-1]
    assert a == b
    assert any(s for _, s in a) and any(not s for _, s in a)
    for r, (owner, split) in zip(reqs, a):
        assert split == (sharding.request_cost(*FRAMES[r.res], r.K) >= SPLIT_MIN)
    # one rank: nothing is split
    assert not any(s for _, s in dispatch.plan_stream(reqs, FRAMES, 1, 1e6, SPLIT_MIN))


def test_local_requests_cover_every_pixel_of_split_requests():
    reqs = make_requests()
    plan = dispatch.plan_stream(reqs, FRAMES, 3, 1e6, SPLIT_MIN)
    parts = [dispatch.local_requests(reqs, plan, FRAMES, r, 3) for r in range(3)]
    for r, (owner, split) in zip(reqs, plan):
        W, H = FRAMES[r.res]
        mine = [p for rank in range(3) for p in parts[rank] if p.rid == r.rid]
        if split:
            spans = sorted((p.px_lo, p.px_hi) for p in mine)
            assert spans[0][0] == 0 and spans[-1][1] == W * H
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
        else:
            assert len(mine) == 1 and mine[0].px_hi == 0


def test_two_ranks_serve_and_gather():
    out = _run({})
    owned = {}
    for o, bad, plan, _ in out:
        assert not bad, bad
        for rid, st in o.items():
            assert rid not in owned, f"request {rid} owned twice"
            owned[rid] = st
    assert out[0][2] == out[1][2]                      # same plan on both ranks
    assert sorted(owned) == list(range(40))
    assert all(st == "done" for st in owned.values()), owned
    assert sum(1 for _, s in out[0][2] if s) >= 5      # split requests were exercised


def test_injected_failures_end_only_their_requests():
    reqs = make_requests()
    plan = dispatch.plan_stream(reqs, FRAMES, 2, 1e6, SPLIT_MIN)
    split = [r.rid for r, (o, s) in zip(reqs, plan) if s]
    # rank 1's band of a request owned by rank 0 fails at launch; rank 1, owner of another
    # split request, fails its own part at admission
    rid_band = next(rid for rid in split if plan[rid][0] == 0)
    rid_owner = next(rid for rid in split if plan[rid][0] == 1)
    # rank 0 loses its band of the earliest split request rank 1 owns (dropped in transit):
    # the band still goes out, flagged, ahead of rank 0's later bands for rank 1
    rid_drop = next(rid for rid in split if plan[rid][0] == 1 and rid != rid_owner)
    out = _run({1: [("launch", rid_band), ("admit", rid_owner)], 0: [("drop", rid_drop)]})
    owned = {}
    for o, bad, _, _ in out:
        assert not bad
        owned.update(o)
    assert sorted(owned) == list(range(40))
    not_done = sorted(rid for rid, st in owned.items() if st != "done")
    assert not_done == sorted([rid_band, rid_owner, rid_drop]), not_done

"""CPU tests of the serving policy: quantum planning, admission, the request stream."""
import math

import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import serve


def _req(rid, n_px, K, next_px=0):
    r = serve.Request(rid, 0.0, 0, K, "rot")
    r.n_px, r.next_px = n_px, next_px
    return r


def test_quantum_is_tile_aligned_srpt_and_bounded():
    active = [_req(0, 1920 * 1080, 300), _req(1, 256 * 256, 64), _req(2, 512 * 512, 128, next_px=128 * 100)]
    q = 50_000_000
    plan = serve.plan_quantum(active, q)
    assert [r.rid for r, _, _ in plan] == [1, 2, 0]          # least remaining work first
    for r, b, e in plan:
        assert b == r.next_px and e > b
        assert b % serve.TILE == 0 and (e % serve.TILE == 0 or e == r.n_px)
    used = sum((e - b) * r.K for r, b, e in plan)
    assert used <= q


def test_quantum_fifo_order_follows_arrival():
    active = [_req(0, 1920 * 1080, 300), _req(1, 256 * 256, 64), _req(2, 512 * 512, 128)]
    for r, t in zip(active, (0.5, 0.2, 0.1)):
        r.arrival = t
    plan = serve.plan_quantum(active, 10 ** 12, order="fifo")
    assert [r.rid for r, _, _ in plan] == [2, 1, 0]          # earliest arrival first
    plan = serve.plan_quantum(active, 10 ** 12)
    assert [r.rid for r, _, _ in plan] == [1, 2, 0]          # default: least remaining work first
    with pytest.raises(ValueError):
        serve.plan_quantum(active, 10 ** 12, order="lifo")


def test_quantum_always_progresses_and_finishes_requests():
    r = _req(0, 1000, 300)
    plans = 0
    while r.next_px < r.n_px:
        plan = serve.plan_quantum([r], quantum_evals=1)      # smaller than one tile
        assert len(plan) == 1
        _, b, e = plan[0]
        assert e - b == min(serve.TILE, r.n_px - b)
        r.next_px = e
        plans += 1
    assert plans == math.ceil(1000 / serve.TILE)
    assert serve.plan_quantum([r], 10 ** 9) == []


def test_admission_budget():
    a = serve.Admission(100)
    assert a.fits(60)
    a.take(60)
    assert not a.fits(41) and a.fits(40)
    with pytest.raises(RuntimeError):
        a.take(41)
    a.give(60)
    assert a.used == 0


def test_request_bytes_counts_outputs_and_env_table():
    assert serve.request_bytes(100, 10, 64, 32) == 100 * 32 + 10 * (4 + 12 + 128) + 6 * 64 * 64 * 12


def test_stream_is_seeded_poisson_with_the_configured_mix():
    reqs = serve.make_stream(2000, 120.0, seed=0, face_size=4)
    assert [r.rid for r in reqs] == list(range(2000))
    gaps = np.diff([0.0] + [r.arrival for r in reqs])
    assert abs(gaps.mean() - 1 / 120) < 0.1 / 120
    frac_new = np.mean([r.env_kind == "new" for r in reqs])
    assert abs(frac_new - 0.4) < 0.05
    assert {r.K for r in reqs} == {64, 128, 300}
    assert {r.res for r in reqs} == set(range(5))
    for r in reqs[:50]:
        if r.env_kind == "rot":
            assert np.allclose(r.R @ r.R.T, np.eye(3), atol=1e-5) and abs(np.linalg.det(r.R) - 1) < 1e-5
    again = serve.make_stream(20, 120.0, seed=0, face_size=4)
    assert [(r.arrival, r.res, r.K, r.env_kind) for r in again] == [(r.arrival, r.res, r.K, r.env_kind) for r in reqs[:20]]


def test_summary_percentiles():
    reqs = [serve.Request(i, 0.0, 0, 1, "rot") for i in range(100)]
    for i, r in enumerate(reqs):
        r.status, r.t_done, r.n_px = "done", (i + 1) / 1000.0, 1
    s = serve.summarize(reqs, 1.0)
    assert s["done"] == 100 and abs(s["p50_ms"] - 50.5) < 1e-9 and abs(s["p99_ms"] - 99.01) < 1e-9


def test_validate_request_refuses_malformed_fields():
    g = np.random.default_rng(0)
    good_new = serve.Request(0, 0.0, 1, 64, "new", faces=np.zeros((6, 8, 8, 3), np.float32))
    good_rot = serve.Request(1, 0.0, 0, 300, "rot", base_env=2, R=serve.random_rotation(g))
    for r in (good_new, good_rot):
        serve.validate_request(r, n_res=2, face_size=8, n_base=3)
    bad = [
        serve.Request(2, 0.0, 2, 64, "rot", base_env=0, R=np.eye(3)),            # no such frame
        serve.Request(3, 0.0, 0, 0, "rot", base_env=0, R=np.eye(3)),             # K = 0
        serve.Request(4, 0.0, 0, 385, "rot", base_env=0, R=np.eye(3)),           # K > 6*8*8
        serve.Request(5, 0.0, 0, 64, "new", faces=np.zeros((6, 4, 4, 3))),       # wrong face size
        serve.Request(6, 0.0, 0, 64, "rot", base_env=3, R=np.eye(3)),            # no such env map
        serve.Request(7, 0.0, 0, 64, "rot", base_env=0, R=np.full((3, 3), np.nan)),
        serve.Request(8, 0.0, 0, 64, "blur"),
        serve.Request(9, math.nan, 0, 64, "rot", base_env=0, R=np.eye(3)),
    ]
    for r in bad:
        with pytest.raises(ValueError):
            serve.validate_request(r, n_res=2, face_size=8, n_base=3)


def test_edf_packs_small_requests_ahead_of_large_ones():
    """Earliest deadline first: a deadline of arrival + 4x the request's own service time
    (at least 16 ms), so a small request that arrives just after a large one goes first."""
    big = serve.Request(0, 0.000, 0, 300, "new")
    small = serve.Request(1, 0.001, 0, 64, "new")
    for r, n in ((big, 2560 * 1440), (small, 256 * 256)):
        r.n_px, r.next_px = n, 0
    rate = 5e10
    assert serve.deadline(small, rate) == pytest.approx(0.001 + 0.016)
    assert serve.deadline(big, rate) == pytest.approx(4 * 2560 * 1440 * 300 / rate)
    plan = serve.plan_quantum([big, small], quantum_evals=int(rate * 0.012), order="edf", evals_per_s=rate)
    assert plan[0][0] is small and plan[0][1:] == (0, 256 * 256)
    assert plan[1][0] is big and (plan[1][2] - plan[1][1]) % serve.TILE == 0
    fifo = serve.plan_quantum([big, small], quantum_evals=int(rate * 0.012), order="fifo")
    assert fifo[0][0] is big


def test_class_latency_splits_at_720p():
    frames = [256 * 256, 1280 * 720, 1920 * 1080]
    reqs = []
    for i, (res, lat) in enumerate([(0, 0.004), (1, 0.010), (2, 0.030), (2, 0.050)]):
        r = serve.Request(i, 0.0, res, 64, "new")
        r.status, r.t_done = "done", lat
        reqs.append(r)
    c = serve.class_latency(reqs, frames)
    assert c["small"]["done"] == 2 and c["large"]["done"] == 2
    assert c["small"]["p50_ms"] == pytest.approx(7.0) and c["large"]["p50_ms"] == pytest.approx(40.0)


class _PoolFrame:
    def __init__(self, w, h):
        import torch
        self.width, self.height = w, h
        self.fbPredictedIndirect = torch.zeros((w * h, 4))


class _PoolEngine:
    """Stand-in relight that checks no two live requests ever write the same output buffer."""

    class _Info:
        face_size, enc_dims = 4, 16

    def __init__(self):
        self.live = {}      # env id -> id of the output buffer its request writes
        self.next = 0
        self.violations = 0

    def networkInfo(self):
        return self._Info()

    def addEnvironmentFaces(self, faces, K):
        self.next += 1
        return self.next - 1

    def releaseEnvironmentMap(self, env):
        self.live.pop(env, None)

    def relightRanges(self, ranges, cfg=None):
        for env, frame, ind, wd, b, e in ranges:
            owner = self.live.setdefault(env, id(ind))
            if owner != id(ind) or any(o == id(ind) for k, o in self.live.items() if k != env):
                self.violations += 1
            ind[b:e] = float(env)
            wd[b:e] = float(env) + 1.0

    def TCNNSync(self):
        pass


def test_output_buffers_are_reused_and_never_shared_by_live_requests():
    """Retired requests hand their output buffers to later requests of the same resolution
    (no fresh frame-sized allocation per request), and no two live requests share one.  A
    request holds its buffers from admission until its last launch has completed: with at most
    two admitted and two launches in flight, at most six pairs per resolution are ever made."""
    frames_wh = [(16, 8), (32, 16), (48, 24)]
    frames = [_PoolFrame(w, h) for w, h in frames_wh]
    reqs = serve.make_stream(60, rate=1e5, seed=5, face_size=4, p_new=1.0, resolutions=frames_wh, ks=[4, 8])
    eng = _PoolEngine()
    srv = serve.RelightServer(eng, frames, [], precision="fp32", quantum_ms=1.0, est_evals_per_s=2e5, max_active=2)
    out = srv.run(reqs, realtime=False)
    assert out["done"] == len(reqs)
    assert eng.violations == 0
    for res in range(len(frames_wh)):
        pool = srv._out_pool.get(res, [])
        n_res = sum(1 for r in reqs if r.res == res)
        assert 1 <= len(pool) <= 6 and 2 * len(pool) < n_res, (res, len(pool), n_res)

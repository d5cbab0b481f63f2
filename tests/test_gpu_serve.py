"""GPU tests of the serving path: env-map rotation parity, pixel-range relights and the
continuous-batching server (results inside the mix equal results relit alone, bitwise;
admission under a memory budget; rejection, timeout and error paths)."""
import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import netconfig, serve, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _eng():
    from neural_wavelet_prt_demo_b200 import engine
    return engine


def test_env_rotate_bit_exact_and_identity(cuda):
    import torch
    eng = _eng()
    g = np.random.default_rng(0)
    for S in (1, 8, 64, 128):
        faces = synth.make_env_faces(S, seed=S)
        tf = torch.from_numpy(faces).to(cuda)
        assert torch.equal(eng.env_rotate(tf, np.eye(3)), tf)
        for _ in range(3):
            R = serve.random_rotation(g)
            got = eng.env_rotate(tf, R).cpu().numpy()
            assert np.array_equal(got.view(np.uint32), O.env_rotate(faces, R).view(np.uint32))
    # axis permutations land texels on texels exactly
    R = np.array([[0, 0, 1], [0, 1, 0], [-1, 0, 0]], np.float32)
    faces = synth.make_env_faces(16, seed=3)
    got = eng.env_rotate(torch.from_numpy(faces).to(cuda), R).cpu().numpy()
    assert np.array_equal(got, O.env_rotate(faces, R))
    with pytest.raises(eng.NwprtError):
        eng.env_rotate(torch.from_numpy(faces).to(cuda), np.full((3, 3), np.nan))


@pytest.fixture(scope="module")
def rig(cuda):
    import torch
    eng = _eng()
    desc = netconfig.parse(netconfig.CONFIG_LARGE)
    w = synth.make_weights(desc, seed=0, hash_scale=0.5, param_round="fp16")
    e = eng.RenderEngine(netconfig.CONFIG_LARGE)
    e.loadWeights(w)
    sizes = [(64, 48), (100, 37), (128, 128)]
    frames = []
    for i, (W, H) in enumerate(sizes):
        fr = eng.FullFrame.from_gbuffer(synth.make_gbuffer(W, H, seed=50 + i, flag_prob=0.9), cuda)
        e.setFrame(i, fr)
        e.TCNNPass_p1(i)
        frames.append(fr)
    base = [torch.from_numpy(synth.make_env_faces(64, seed=60, index=j)).to(cuda) for j in range(3)]
    yield e, frames, base
    e.close()


def _requests(n, seed=0, spacing=0.003):
    g = np.random.default_rng(seed)
    out = []
    for i in range(n):
        res, K = int(g.integers(3)), int(g.choice([16, 64, 100, 300]))
        if g.uniform() < 0.4:
            out.append(serve.Request(i, i * spacing, res, K, "new",
                                     faces=synth.make_env_faces(64, seed=seed, index=500 + i)))
        else:
            out.append(serve.Request(i, i * spacing, res, K, "rot", base_env=int(g.integers(3)),
                                     R=serve.random_rotation(g)))
    return out


def _solo(e, frames, base, r):
    import torch
    eng = _eng()
    fr = frames[r.res]
    faces = (torch.from_numpy(r.faces).to(fr.fbPredictedIndirect.device) if r.env_kind == "new"
             else eng.env_rotate(base[r.base_env], r.R))
    env = e.addEnvironmentFaces(faces, r.K)
    n = fr.width * fr.height
    out, out2 = torch.empty((n, 4), device=faces.device), torch.empty((n, 4), device=faces.device)
    e.relightRanges([(env, r.res, out, out2, 0, n)], eng.RenderConfig(precision="bf16"))
    e.TCNNSync()
    e.releaseEnvironmentMap(env)
    return out, out2


def test_pixel_ranges_compose_to_the_whole_frame(rig):
    import torch
    e, frames, base = rig
    eng = _eng()
    r = _requests(1, seed=4)[0]
    r.res = 2
    ref, ref2 = _solo(e, frames, base, r)
    faces = (torch.from_numpy(r.faces).cuda() if r.env_kind == "new" else eng.env_rotate(base[r.base_env], r.R))
    env = e.addEnvironmentFaces(faces, r.K)
    n = frames[2].width * frames[2].height
    out, out2 = torch.zeros((n, 4), device="cuda"), torch.zeros((n, 4), device="cuda")
    cuts = [0, 128, 128 * 37, 128 * 90, n]
    e.relightRanges([(env, 2, out, out2, cuts[i], cuts[i + 1]) for i in range(len(cuts) - 1)],
                    eng.RenderConfig(precision="bf16"))
    e.TCNNSync()
    assert torch.equal(out, ref) and torch.equal(out2, ref2)
    with pytest.raises(eng.NwprtError):
        e.relightRanges([(env, 2, out, out2, 0, n + 1)], eng.RenderConfig(precision="bf16"))
    e.releaseEnvironmentMap(env)


def test_served_results_equal_solo_results(rig):
    import torch
    e, frames, base = rig
    reqs = _requests(14, seed=1)
    srv = serve.RelightServer(e, frames, base, precision="bf16", quantum_ms=0.05, est_evals_per_s=9e9,
                              keep_outputs=True)
    stats = srv.run(reqs)
    assert stats["done"] == len(reqs), stats
    assert srv.quanta > len(reqs)          # requests were split across several launches
    for r in reqs:
        ind, wd = _solo(e, frames, base, r)
        assert torch.equal(r.outputs[0], ind), r.rid
        assert torch.equal(r.outputs[1], wd), r.rid
        assert r.latency >= 0


def test_budget_admits_one_request_at_a_time(rig):
    e, frames, base = rig
    reqs = _requests(6, seed=2, spacing=0.0)
    for r in reqs:
        r.res, r.K = 2, 300
    one = serve.request_bytes(frames[2].width * frames[2].height, 300, 64, 32)
    srv = serve.RelightServer(e, frames, base, budget_bytes=one + one // 2, quantum_ms=0.2)
    stats = srv.run(reqs)
    assert stats["done"] == 6 and srv.max_active == 1


def test_admission_cap_limits_concurrency_and_keeps_results(rig):
    import torch
    e, frames, base = rig
    reqs = _requests(10, seed=5, spacing=0.0)
    srv = serve.RelightServer(e, frames, base, precision="bf16", quantum_ms=0.05, est_evals_per_s=9e9,
                              keep_outputs=True, max_active=2)
    stats = srv.run(reqs)
    assert stats["done"] == len(reqs), stats
    assert srv.max_active <= 2
    for r in reqs[:4]:
        ind, _ = _solo(e, frames, base, r)
        assert torch.equal(r.outputs[0], ind), r.rid


def test_rejection_timeout_and_error_paths(rig):
    e, frames, base = rig
    reqs = _requests(5, seed=3, spacing=0.0)
    # a request larger than the whole budget is refused; the others are served
    small = serve.request_bytes(frames[0].width * frames[0].height, 300, 64, 32)
    for r in reqs:
        r.res = 0
    reqs[2].res = 2
    srv = serve.RelightServer(e, frames, base, budget_bytes=small, quantum_ms=0.2)
    stats = srv.run(reqs)
    assert reqs[2].status == "rejected" and stats["rejected"] == 1 and stats["done"] == 4
    # malformed env map (wrong face size) fails that request only
    reqs = _requests(4, seed=5, spacing=0.0)
    reqs[1].env_kind, reqs[1].faces = "new", synth.make_env_faces(16, seed=1)
    stats = serve.RelightServer(e, frames, base, quantum_ms=0.2).run(reqs)
    assert reqs[1].status == "error" and stats["done"] == 3
    # a queue deadline of zero with room for one request at a time times the rest out
    reqs = _requests(5, seed=6, spacing=0.0)
    for r in reqs:
        r.res, r.K = 2, 300
    one = serve.request_bytes(frames[2].width * frames[2].height, 300, 64, 32)
    stats = serve.RelightServer(e, frames, base, budget_bytes=one, quantum_ms=0.2, max_queue_s=0.0).run(reqs)
    assert stats["timeout"] >= 1 and stats["done"] >= 1 and stats["done"] + stats["timeout"] == 5


def test_more_ranges_than_one_launch_carries(rig):
    """A batch of more requests than one launch's job table (256) is split into several
    launches; the pieces still compose to the whole-frame relight bit for bit."""
    import torch
    e, frames, base = rig
    eng = _eng()
    fr = frames[2]
    n = fr.width * fr.height                      # 128 x 128 = 16384 px
    env = e.addEnvironmentFaces(base[0], 64)
    whole, whole2 = torch.empty((n, 4), device="cuda"), torch.empty((n, 4), device="cuda")
    e.relightRanges([(env, 2, whole, whole2, 0, n)], eng.RenderConfig(precision="bf16"))
    cuts = list(range(0, n, 48)) + [n]            # 342 ranges, most not tile-aligned
    out, out2 = torch.zeros((n, 4), device="cuda"), torch.zeros((n, 4), device="cuda")
    e.relightRanges([(env, 2, out, out2, cuts[i], cuts[i + 1]) for i in range(len(cuts) - 1)],
                    eng.RenderConfig(precision="bf16"))
    e.TCNNSync()
    assert len(cuts) - 1 > 256
    assert torch.equal(out, whole) and torch.equal(out2, whole2)
    e.releaseEnvironmentMap(env)


def test_injected_faults_stay_with_their_requests(rig):
    """Host-side fault injection: a request lost in transit, one malformed request, an
    allocation failure at set-up, a failure detected at launch, and a request whose env id
    is corrupted so that its quantum's launch raises.  Each ends alone; every other request
    is served and equals its solo result, and the whole budget is returned."""
    import torch
    e, frames, base = rig
    reqs = _requests(10, seed=9, spacing=0.0)
    reqs[2].K = 0                                   # malformed: refused at admission

    def fault(r, stage):
        if stage == "arrive" and r.rid == 1:
            return "drop"
        if stage == "admit" and r.rid == 3:
            raise MemoryError("simulated allocation failure")
        if stage == "launch" and r.rid == 4:
            raise RuntimeError("simulated corrupt request")
        if stage == "launch" and r.rid == 6:
            r.env_id = 10_000                       # the batched launch fails; isolation ends r 6 only
        return None

    srv = serve.RelightServer(e, frames, base, quantum_ms=0.05, est_evals_per_s=9e9, keep_outputs=True,
                              fault=fault)
    stats = srv.run(reqs)
    status = {r.rid: r.status for r in reqs}
    assert status[1] == "dropped" and status[2] == "error" and status[3] == "error"
    assert status[4] == "error" and status[6] == "error"
    assert stats["dropped"] == 1 and stats["error"] == 4 and stats["done"] == 5
    assert srv.adm.used == 0
    for r in reqs:
        if r.status == "done":
            ind, wd = _solo(e, frames, base, r)
            assert torch.equal(r.outputs[0], ind) and torch.equal(r.outputs[1], wd), r.rid


@pytest.mark.parametrize("order", ["edf", "fifo", "srpt"])
def test_packing_orders_keep_results(rig, order):
    import torch
    e, frames, base = rig
    reqs = _requests(10, seed=7)
    srv = serve.RelightServer(e, frames, base, precision="bf16", quantum_ms=0.05, est_evals_per_s=9e9,
                              keep_outputs=True, order=order)
    stats = srv.run(reqs)
    assert stats["done"] == len(reqs), stats
    for r in reqs:
        ind, _ = _solo(e, frames, base, r)
        assert torch.equal(r.outputs[0], ind), (order, r.rid)
    cls = serve.class_latency(reqs, [f.width * f.height for f in frames])
    assert cls["small"]["done"] == len(reqs)


def test_dispatcher_on_one_gpu(rig):
    """The multi-GPU dispatcher at world size 1: every request placed on rank 0, none split,
    results equal to the same requests relit alone."""
    import torch
    from neural_wavelet_prt_demo_b200 import dispatch
    e, frames, base = rig
    reqs = _requests(8, seed=9)
    summ = dispatch.serve_distributed(e, frames, base, reqs, 0, 1, None, "cuda", evals_per_s=9e9,
                                      server_kwargs=dict(precision="bf16", quantum_ms=0.05, est_evals_per_s=9e9,
                                                         keep_outputs=True))
    assert summ["owned_done"] == len(reqs) and summ["split_requests"] == 0
    for r in summ["local"]:
        ind, _ = _solo(e, frames, base, r)
        assert torch.equal(r.outputs[0], ind), r.rid


def test_env_slots_are_reused_and_grown(rig):
    """Env slots hold 1,024 wavelets and are reused in stream order; a table larger than every
    released slot gets a new one (no device-wide synchronisation).  Tables registered in any
    order read back intact, and the grown slots relight as the FP32 oracle does."""
    import torch
    e, frames, base = rig
    eng = _eng()
    desc = netconfig.parse(netconfig.CONFIG_LARGE)
    w = synth.make_weights(desc, seed=0, hash_scale=0.5, param_round="fp16")
    b = O.Bound(desc, w, synth.make_gbuffer(64, 48, seed=50, flag_prob=0.9))
    g = np.random.default_rng(9)
    n, px = 64 * 48, 128
    for K in (64, 1024, 1500, 16, 2000, 300):
        idx = g.choice(desc.n_coeffs, K, replace=False).astype(np.int32)
        st = g.lognormal(0.0, 1.0, size=(K, 3)).astype(np.float32)
        env = e.addEnvironmentMap(eng.EnvironmentMap(top_coefficients=idx, top_strength=st))
        gi, gs = e.envWavelets(env)
        assert np.array_equal(gi, idx) and np.array_equal(gs, st), K
        if K > 1024:
            out, out2 = torch.zeros((n, 4), device="cuda"), torch.zeros((n, 4), device="cuda")
            e.relightRanges([(env, 0, out, out2, 0, px)], eng.RenderConfig(precision="fp32"))
            e.TCNNSync()
            ref, _ = O.relight_f32(b, idx, st, px_begin=0, px_end=px)
            got = out[:px, :3].cpu().numpy()
            r = ref[:px, :3]
            rel = np.abs(got - r) / np.maximum(np.abs(r), 1e-6 * np.abs(r).max())
            assert float(rel.max()) <= 1e-5, (K, float(rel.max()))
        e.releaseEnvironmentMap(env)

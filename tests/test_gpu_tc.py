"""GPU tests of the tcgen05 BF16 relight path through the C ABI.

Accuracy bar (the served form): PSNR >= 45 dB against the FP64 oracle of the same
network and weights, per image.  Batching bar: every request's result inside a mixed
batch is bitwise identical to the same request relit alone."""
import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import netconfig, synth
from oracle import oracle as O
from tests.helpers import make_case, psnr, rel_err

pytestmark = pytest.mark.gpu

PSNR_MIN = 45.0


def _eng():
    from neural_wavelet_prt_demo_b200 import engine
    return engine


def relight(case, precision="bf16", kahan=True, clamp=True):
    eng = _eng()
    e = eng.RenderEngine(case.cfg)
    e.loadWeights(case.weights)
    e.addEnvironmentMap(eng.EnvironmentMap(top_coefficients=case.idx, top_strength=case.strength))
    fr = eng.FullFrame.from_gbuffer(case.gbuf)
    e.setFrame(0, fr)
    e.TCNNPass_p1(0)
    e.TCNNPass_p2(0, 0, eng.RenderConfig(precision=precision, kahan=kahan, clamp_terms=clamp))
    e.TCNNSync()
    out = fr.fbPredictedIndirect.cpu().numpy(), fr.fbPredictedIndirectWithDirect.cpu().numpy()
    e.close()
    return out


@pytest.mark.parametrize("cfg,w,h,K,hs", [
    (netconfig.CONFIG_LARGE, 64, 40, 64, 1e-4),
    (netconfig.CONFIG_LARGE, 48, 30, 300, 1e-4),
    (netconfig.CONFIG_LARGE, 32, 20, 512, 1e-4),
    (netconfig.CONFIG_LARGE, 16, 8, 1024, 1e-4),
    (netconfig.CONFIG_LARGE, 33, 17, 29, 0.5),
    (netconfig.CONFIG_SMALL, 128, 128, 64, 1e-4),
    (netconfig.CONFIG_SMALL, 31, 9, 17, 0.5),
], ids=["large-k64", "large-k300", "large-k512", "large-k1024", "large-ragged-hash", "small-config0",
       "small-ragged"])
def test_bf16_psnr_vs_fp64(cuda, cfg, w, h, K, hs):
    case = make_case(cfg, w, h, K, seed=K, hash_scale=hs, flag_prob=0.9,
                     param_round="fp16" if cfg is netconfig.CONFIG_LARGE else "fp32")
    ind, wd = relight(case)
    r64 = O.relight_f64(case.bound, case.idx, case.strength)
    p = psnr(ind[:, :3], r64)
    assert p >= PSNR_MIN, (p, rel_err(ind[:, :3], r64))
    assert np.all(ind[:, 3] == 1.0) and np.all(wd[:, 3] == 1.0)
    off = case.gbuf.flag == 0
    assert np.all(ind[off, :3] == 0)
    assert np.allclose(wd[:, :3], ind[:, :3] + case.gbuf.direct[:, :3], rtol=0, atol=0)


def test_bf16_when_every_layer_matters(cuda):
    """In the random-init networks the 13 aux values entering cmp_net's first layer dominate
    the output, so rounding in the four tensor-core layers before them barely shows.  With the
    aux block of that layer scaled by 1e-3, the wavelet-dependent path carries the output (an
    operand-rounding model of this network gives 41-46 dB with E4M3 in any single layer): BF16
    must still clear the bar there, and the FP32 drop-in must still match the FP32 oracle."""
    case = make_case(netconfig.CONFIG_LARGE, 48, 30, 300, seed=11, hash_scale=0.5, flag_prob=0.9,
                     param_round="fp16")
    n_in, n_out = case.desc.cn_layers()[0]
    m = case.desc.op_out  # cmp_net's input: out_prd's outputs, then the aux block
    w0 = case.weights.cmp_net[:n_in * n_out].reshape(n_out, n_in)
    w0[:, m:] *= np.float32(1e-3)
    case.bound = O.Bound(case.desc, case.weights, case.gbuf)
    ind, _ = relight(case)
    r64 = O.relight_f64(case.bound, case.idx, case.strength)
    p = psnr(ind[:, :3], r64)
    assert p >= PSNR_MIN, (p, rel_err(ind[:, :3], r64))
    ind32, _ = relight(case, precision="fp32")
    r32, _ = O.relight_f32(case.bound, case.idx, case.strength)
    assert rel_err(ind32[:, :3], r32[:, :3])[0] <= 1e-5


def test_bf16_single_pixel_single_wavelet(cuda):
    case = make_case(netconfig.CONFIG_LARGE, 1, 1, 1, seed=3, hash_scale=0.5)
    ind, _ = relight(case)
    r64 = O.relight_f64(case.bound, case.idx, case.strength)
    assert abs(ind[0, :3] - r64[0]).max() <= 2e-2 * max(abs(r64).max(), 1e-6)


def test_bf16_kahan_and_clamp_options(cuda):
    case = make_case(netconfig.CONFIG_LARGE, 40, 20, 96, seed=8, hash_scale=0.5)
    ind, _ = relight(case, kahan=False, clamp=False)
    r64 = O.relight_f64(case.bound, case.idx, case.strength, clamp=False)
    assert psnr(ind[:, :3], r64) >= 40.0     # unclamped sums cancel: a looser bar


def test_bf16_deterministic(cuda):
    case = make_case(netconfig.CONFIG_LARGE, 64, 64, 48, seed=2, hash_scale=0.5)
    a, _ = relight(case)
    b, _ = relight(case)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_batch_result_equals_solo_result(cuda):
    """Continuous-batching property: requests of mixed size, K and env map relit together
    in one device pass give the same bits as each request relit alone."""
    import torch
    eng = _eng()
    desc = netconfig.parse(netconfig.CONFIG_LARGE)
    w = synth.make_weights(desc, seed=0, hash_scale=0.5, param_round="fp16")
    e = eng.RenderEngine(netconfig.CONFIG_LARGE)
    e.loadWeights(w)
    sizes = [(37, 11), (128, 3), (64, 64), (5, 1)]
    Ks = [64, 300, 128, 7]
    frames, envs = [], []
    for i, ((W, H), K) in enumerate(zip(sizes, Ks)):
        gb = synth.make_gbuffer(W, H, seed=100 + i, flag_prob=0.8)
        fr = eng.FullFrame.from_gbuffer(gb)
        e.setFrame(i, fr)
        e.TCNNPass_p1(i)
        frames.append(fr)
        envs.append(e.addEnvironmentMap(eng.EnvironmentMap(synth.make_env_faces(64, seed=7, index=i)), K=K))
    cfg = eng.RenderConfig(precision="bf16")
    solo = []
    for i, fr in enumerate(frames):
        e.TCNNPass_p2(envs[i], i, cfg)
        e.TCNNSync()
        solo.append(fr.fbPredictedIndirect.clone())
    outs = [(torch.zeros_like(f.fbPredictedIndirect), torch.zeros_like(f.fbPredictedIndirect)) for f in frames]
    e.relightBatch([(envs[i], i, outs[i][0], outs[i][1]) for i in range(len(frames))], cfg)
    e.TCNNSync()
    for i in range(len(frames)):
        assert torch.equal(outs[i][0], solo[i]), i
    e.close()

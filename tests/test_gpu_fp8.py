"""GPU tests of the FP8 (E4M3, per-layer scales) tensor-core relight through the C ABI.

FP8 keeps 4 significant bits per operand against BF16's 8, so its error is about 16x
(24 dB) larger; the bar here is PSNR >= FP8_PSNR_MIN against the FP64 oracle of the same
network and weights.  Scales are calibrated once and then fixed, so results are
deterministic and a request gives the same bits alone and inside a batch."""
import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import netconfig, synth
from oracle import oracle as O
from tests.helpers import make_case, psnr, rel_err

pytestmark = pytest.mark.gpu

FP8_PSNR_MIN = 30.0


def _eng():
    from neural_wavelet_prt_demo_b200 import engine
    return engine


def _rig(case):
    eng = _eng()
    e = eng.RenderEngine(case.cfg)
    e.loadWeights(case.weights)
    env = e.addEnvironmentMap(eng.EnvironmentMap(top_coefficients=case.idx, top_strength=case.strength))
    fr = eng.FullFrame.from_gbuffer(case.gbuf)
    e.setFrame(0, fr)
    e.TCNNPass_p1(0)
    return e, env, fr


def _run(e, env, fr, precision="fp8"):
    eng = _eng()
    e.TCNNPass_p2(env, 0, eng.RenderConfig(precision=precision))
    e.TCNNSync()
    return fr.fbPredictedIndirect.cpu().numpy().copy(), fr.fbPredictedIndirectWithDirect.cpu().numpy().copy()


def test_fp8_needs_calibration(cuda):
    eng = _eng()
    case = make_case(netconfig.CONFIG_LARGE, 16, 8, 16, seed=1, hash_scale=0.5)
    e, env, fr = _rig(case)
    with pytest.raises(eng.NwprtError) as ex:
        e.TCNNPass_p2(env, 0, eng.RenderConfig(precision="fp8"))
    assert ex.value.status == 5  # NWPRT_NOT_READY
    with pytest.raises(eng.NwprtError):
        e.fp8Calibration()
    with pytest.raises(eng.NwprtError):
        e.calibrateFP8(env, 0, 5, 5)  # empty range
    e.close()


@pytest.mark.parametrize("cfg,w,h,K,hs", [
    (netconfig.CONFIG_LARGE, 64, 40, 64, 1e-4),
    (netconfig.CONFIG_LARGE, 48, 30, 300, 1e-4),
    (netconfig.CONFIG_LARGE, 33, 17, 29, 0.5),
    (netconfig.CONFIG_SMALL, 128, 128, 64, 1e-4),
    (netconfig.CONFIG_SMALL, 31, 9, 17, 0.5),
], ids=["large-k64", "large-k300", "large-ragged-hash", "small-config0", "small-ragged"])
def test_fp8_psnr_vs_fp64(cuda, cfg, w, h, K, hs):
    case = make_case(cfg, w, h, K, seed=K, hash_scale=hs, flag_prob=0.9,
                     param_round="fp16" if cfg is netconfig.CONFIG_LARGE else "fp32")
    e, env, fr = _rig(case)
    amax = e.calibrateFP8(env, 0)
    desc = netconfig.parse(cfg)
    # the 3-wide output layer runs in FP32, and out_prd's linear output layer is folded into
    # cmp_net's first layer
    n_tc_layers = len(desc.op_layers()) + len(desc.cn_layers()) - 2
    assert np.all(np.isfinite(amax)) and np.all(amax >= 0) and amax[0] > 0
    assert len(amax) == n_tc_layers + 1
    ind, wd = _run(e, env, fr)
    bf, _ = _run(e, env, fr, "bf16")
    e.close()
    r64 = O.relight_f64(case.bound, case.idx, case.strength)
    p8, pb = psnr(ind[:, :3], r64), psnr(bf[:, :3], r64)
    print(f"fp8 PSNR {p8:.1f} dB (bf16 {pb:.1f} dB), rel err {rel_err(ind[:, :3], r64)}")
    assert p8 >= FP8_PSNR_MIN, (p8, pb)
    assert np.all(ind[:, 3] == 1.0) and np.all(wd[:, 3] == 1.0)
    off = case.gbuf.flag == 0
    assert np.all(ind[off, :3] == 0)
    assert np.allclose(wd[:, :3], ind[:, :3] + case.gbuf.direct[:, :3], rtol=0, atol=0)


def test_fp8_calibration_reproducible_and_deterministic(cuda):
    case = make_case(netconfig.CONFIG_LARGE, 64, 32, 48, seed=2, hash_scale=0.5)
    e, env, fr = _rig(case)
    a1 = e.calibrateFP8(env, 0, 0, 1024)
    x1, _ = _run(e, env, fr)
    a2 = e.calibrateFP8(env, 0, 0, 1024)
    x2, _ = _run(e, env, fr)
    assert np.array_equal(a1, a2)
    assert np.array_equal(x1.view(np.uint32), x2.view(np.uint32))
    # a different calibration range gives other scales; the results stay close
    a3 = e.calibrateFP8(env, 0)
    x3, _ = _run(e, env, fr)
    e.close()
    assert np.all(a3 >= a1)  # the whole frame contains the first 1024 pixels
    r64 = O.relight_f64(case.bound, case.idx, case.strength)
    assert psnr(x3[:, :3], r64) >= FP8_PSNR_MIN


def test_fp8_batch_result_equals_solo_result(cuda):
    import torch
    eng = _eng()
    desc = netconfig.parse(netconfig.CONFIG_LARGE)
    w = synth.make_weights(desc, seed=0, hash_scale=0.5, param_round="fp16")
    e = eng.RenderEngine(netconfig.CONFIG_LARGE)
    e.loadWeights(w)
    sizes, Ks = [(37, 11), (128, 3), (64, 64)], [64, 300, 7]
    frames, envs = [], []
    for i, ((W, H), K) in enumerate(zip(sizes, Ks)):
        fr = eng.FullFrame.from_gbuffer(synth.make_gbuffer(W, H, seed=100 + i, flag_prob=0.8))
        e.setFrame(i, fr)
        e.TCNNPass_p1(i)
        frames.append(fr)
        envs.append(e.addEnvironmentMap(eng.EnvironmentMap(synth.make_env_faces(64, seed=7, index=i)), K=K))
    e.calibrateFP8(envs[2], 2)
    cfg = eng.RenderConfig(precision="fp8")
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
    # a weight load drops the calibration
    e.loadWeights(w)
    with pytest.raises(eng.NwprtError):
        e.TCNNPass_p2(envs[0], 0, cfg)
    e.close()

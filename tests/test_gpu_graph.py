"""GPU test of the relight pass captured in a CUDA graph: a replay reads the frame's
G-buffer tensors as they are at replay time and gives the same bits as the eager pass."""
import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import netconfig, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg,precision", [(netconfig.CONFIG_LARGE, "bf16"), (netconfig.CONFIG_SMALL, "fp32")])
def test_captured_relight_replays_on_new_inputs(cuda, cfg, precision):
    import torch
    from neural_wavelet_prt_demo_b200 import engine as eng
    desc = netconfig.parse(cfg)
    e = eng.RenderEngine(cfg)
    e.loadWeights(synth.make_weights(desc, seed=3, hash_scale=0.5))
    env = e.addEnvironmentMap(eng.EnvironmentMap(synth.make_env_faces(desc.face_size, seed=4)), K=48)
    W, H = 70, 33
    frame = eng.FullFrame.from_gbuffer(synth.make_gbuffer(W, H, seed=1, flag_prob=0.8))
    e.setFrame(0, frame)
    rc = eng.RenderConfig(precision=precision)
    g = e.captureRelight(env, 0, rc)
    first = frame.fbPredictedIndirect.clone()
    frame.fbPredictedIndirect.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(frame.fbPredictedIndirect, first)
    # new G-buffer contents in the same tensors; the replay must see them
    other = eng.FullFrame.from_gbuffer(synth.make_gbuffer(W, H, seed=2, flag_prob=0.8))
    for name in ("fbFirstHitPos", "fbworldNormal", "fbFirstHitReflecDir", "fbRoughness", "fbFirstHitKd",
                 "fbFirstHitKs", "fbDirectDenoised", "fbEnvironmentMapFlag"):
        getattr(frame, name).copy_(getattr(other, name))
    g.replay()
    torch.cuda.synchronize()
    e.setFrame(1, other)
    e.TCNNPass_p1(1)
    e.TCNNPass_p2(env, 1, rc)
    e.TCNNSync()
    assert not torch.equal(other.fbPredictedIndirect, first)
    assert torch.equal(frame.fbPredictedIndirect, other.fbPredictedIndirect)
    assert torch.equal(frame.fbPredictedIndirectWithDirect, other.fbPredictedIndirectWithDirect)
    del g
    e.close()

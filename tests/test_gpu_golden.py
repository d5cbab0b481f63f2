"""The GPU path through the C ABI against the committed known answers (tests/golden/*.npz).

- Haar + top-K: indices and strength bits equal the fixture's.
- FP32 drop-in: equal to the FP32 oracle's fixture within 1e-5 relative (bit-exact on
  config 0), and within 1e-5 of the FP32 relight fed with the reference's own remap rows
  (prt::waveletDataCopy, utils_kernels.h:7-49): the drop-in's gap to the reference's
  arithmetic, not only to this build's oracle.
- BF16 tensor-core path: PSNR >= 45 dB against the FP64 fixture.
- SH projection within 1e-5 of the FP64 fixture's largest coefficient; SH dot bit-exact."""
import numpy as np
import pytest
import torch

from tests.golden import make_golden as G
from tests.helpers import bits_equal, err_stats, load_golden, rel_err

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5


def _relight(case, fx, precision):
    from neural_wavelet_prt_demo_b200 import engine as eng
    desc, w, gb, faces = G.relight_inputs(case)
    e = eng.RenderEngine(case["cfg"])
    try:
        e.loadWeights(w)
        env = e.addEnvironmentMap(eng.EnvironmentMap(faces), K=case["K"])
        idx, st = e.envWavelets(env)
        fr = eng.FullFrame.from_gbuffer(gb)
        e.setFrame(0, fr)
        e.TCNNPass_p1(0)
        px = fx["px"]
        runs = G.contiguous_runs(px) if "runs" in case else [(0, gb.n)]
        ranges = [(env, 0, fr.fbPredictedIndirect, fr.fbPredictedIndirectWithDirect, s, en) for s, en in runs]
        e.relightRanges(ranges, eng.RenderConfig(precision=precision))
        e.TCNNSync()
        out = fr.fbPredictedIndirect[torch.from_numpy(px).to(fr.fbPredictedIndirect.device)].cpu().numpy()
        return idx, st, out
    finally:
        e.close()


@pytest.mark.parametrize("name,case", [("cfg0", G.CFG0), ("cfg2", G.CFG2)])
def test_golden_relight_fp32(cuda, name, case):
    fx = load_golden(name)
    idx, st, out = _relight(case, fx, "fp32")
    assert np.array_equal(idx, fx["topk_idx"])
    assert bits_equal(st, fx["topk_strength"])
    mx, _ = rel_err(out[:, :3], fx["fp32_indirect"][:, :3])
    assert mx <= FP32_TOL, mx
    if name == "cfg0":
        assert bits_equal(out, fx["fp32_indirect"])
    gap, mean_gap = rel_err(out[:, :3], fx["fp32_refrows_indirect"][:, :3])
    print(f"{name}: FP32 drop-in vs the reference's remap rows: max rel {gap:.2e}, mean {mean_gap:.2e}")
    assert gap <= FP32_TOL, gap


@pytest.mark.parametrize("name,case", [("cfg0", G.CFG0), ("cfg2", G.CFG2)])
def test_golden_relight_bf16(cuda, name, case):
    from neural_wavelet_prt_demo_b200 import engine as eng
    fx = load_golden(name)
    try:
        _, _, out = _relight(case, fx, "bf16")
    except eng.NwprtError as ex:
        if ex.status == eng._lib.UNSUPPORTED:
            pytest.skip("network not supported by the tensor-core path")
        raise
    s = err_stats(out[:, :3], fx["fp64_rgb"])
    print(name, "BF16 vs FP64 fixture", s)
    assert s["psnr_db"] >= 45.0, s


def test_golden_sh(cuda):
    from neural_wavelet_prt_demo_b200 import engine as eng
    fx = load_golden("cfg1")
    c = G.CFG1
    faces = G.synth.make_env_faces(c["face_size"], seed=c["env_seed"])
    T = G.synth.make_sh_transport(c["n_px"], seed=c["t_seed"])
    L = eng.sh_project(torch.from_numpy(faces).to(cuda)).cpu().numpy().astype(np.float64)
    assert np.abs(L - fx["L_f64"]).max() <= 1e-5 * np.abs(fx["L_f64"]).max()
    L32 = torch.from_numpy(fx["L_f64"].astype(np.float32)).to(cuda)
    out = eng.sh_dot(torch.from_numpy(T).to(cuda), L32).cpu().numpy()
    assert bits_equal(out, fx["sh_dot_f32"])

"""GPU tests of the tensor-core relight on networks outside the two standard shapes.

The kernel is specialised at compile time for the two standard layer sequences (config 0
and config 2); every other supported network runs its generic form, which reads the layer
sequence from the plan at run time.  These networks take that form: other hidden-layer
counts, 32-wide out_prd layers, 16 hash features with a deeper out_prd.  Same bars as the
standard shapes: BF16 PSNR >= 45 dB against the FP64 oracle, FP8 >= 30 dB, and the FP32
drop-in (its generic kernel) within 1e-5 of the FP32 oracle, in fact bit-identical."""
import copy

import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import netconfig
from oracle import oracle as O
from tests.helpers import make_case, psnr, rel_err

pytestmark = pytest.mark.gpu

PSNR_MIN = 45.0
FP8_PSNR_MIN = 30.0
FP32_TOL = 1e-5


def _variant(base, **changes):
    cfg = copy.deepcopy(base)
    for path, value in changes.items():
        block, key = path.split("__")
        cfg[block][key] = value
    return cfg


NETS = {
    # out_prd 32->64->64->64 (2 hidden), cmp_net (64||16)->64->64->3: five tensor-core layers
    "large-2x2": _variant(netconfig.CONFIG_LARGE, out_prd__n_hidden_layers=2, cmp_net__n_hidden_layers=2),
    # 32-wide out_prd: hidden and output layers of width 32 (one-half accumulator epilogues)
    "large-op32": _variant(netconfig.CONFIG_LARGE, out_prd__n_neurons=32, out_prd__n_output_dims=32),
    # 16 hash features with a hidden out_prd layer, and a deeper cmp_net
    "small-deep": _variant(netconfig.CONFIG_SMALL, out_prd__n_hidden_layers=1, cmp_net__n_hidden_layers=3),
}


def _eng():
    from neural_wavelet_prt_demo_b200 import engine
    return engine


def _relight(case, precision, calibrate=False):
    eng = _eng()
    e = eng.RenderEngine(case.cfg)
    e.loadWeights(case.weights)
    env = e.addEnvironmentMap(eng.EnvironmentMap(top_coefficients=case.idx, top_strength=case.strength))
    fr = eng.FullFrame.from_gbuffer(case.gbuf)
    e.setFrame(0, fr)
    e.TCNNPass_p1(0)
    if calibrate:
        e.calibrateFP8(env, 0)
    e.TCNNPass_p2(env, 0, eng.RenderConfig(precision=precision))
    e.TCNNSync()
    out = fr.fbPredictedIndirect.cpu().numpy(), fr.fbPredictedIndirectWithDirect.cpu().numpy()
    e.close()
    return out


@pytest.mark.parametrize("name", list(NETS))
def test_generic_plan_bf16_psnr(cuda, name):
    case = make_case(NETS[name], 40, 24, 72, seed=11, hash_scale=0.5, flag_prob=0.9)
    ind, wd = _relight(case, "bf16")
    r64 = O.relight_f64(case.bound, case.idx, case.strength)
    p = psnr(ind[:, :3], r64)
    assert p >= PSNR_MIN, (name, p, rel_err(ind[:, :3], r64))
    assert np.all(ind[:, 3] == 1.0) and np.all(wd[:, 3] == 1.0)
    assert np.all(ind[case.gbuf.flag == 0, :3] == 0)


@pytest.mark.parametrize("name", list(NETS))
def test_generic_plan_fp8_psnr(cuda, name):
    case = make_case(NETS[name], 40, 24, 72, seed=12, hash_scale=0.5, flag_prob=0.9)
    ind, _ = _relight(case, "fp8", calibrate=True)
    r64 = O.relight_f64(case.bound, case.idx, case.strength)
    assert psnr(ind[:, :3], r64) >= FP8_PSNR_MIN, name


@pytest.mark.parametrize("name", list(NETS))
def test_generic_plan_fp32_drop_in(cuda, name):
    # the generic FP32 kernel keeps the oracle's operation order: same bits, within 1e-5 a fortiori
    case = make_case(NETS[name], 24, 16, 40, seed=13, hash_scale=0.5)
    ind, wd = _relight(case, "fp32")
    rind, rwd = O.relight_f32(case.bound, case.idx, case.strength)
    assert rel_err(ind[:, :3], rind[:, :3])[0] <= FP32_TOL, name
    assert rel_err(wd[:, :3], rwd[:, :3])[0] <= FP32_TOL, name
    assert np.array_equal(ind.view(np.uint32), rind.view(np.uint32)), name

"""GPU parity of the relight path through the C ABI against the CPU oracle.

FP32 drop-in path: max relative error <= 1e-5 against the FP32 oracle (same operation
order; denominators floored at 1e-6 of the image maximum).  Engine entry points and
their error behaviour mirror the reference's RenderEngine."""
import os

import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import netconfig, synth
from oracle import oracle as O
from tests.helpers import make_case, rel_err

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5


def _eng():
    from neural_wavelet_prt_demo_b200 import engine
    return engine


def run_gpu(case, precision="fp32", clamp=True, kahan=True, K_env=None):
    eng = _eng()
    e = eng.RenderEngine(case.cfg)
    e.loadWeights(case.weights)
    e.addEnvironmentMap(eng.EnvironmentMap(top_coefficients=case.idx, top_strength=case.strength))
    fr = eng.FullFrame.from_gbuffer(case.gbuf)
    e.setFrame(0, fr)
    e.TCNNPass_p1(0)
    e.TCNNPass_p2(0, 0, eng.RenderConfig(precision=precision, clamp_terms=clamp, kahan=kahan))
    e.TCNNSync()
    out = fr.fbPredictedIndirect.cpu().numpy(), fr.fbPredictedIndirectWithDirect.cpu().numpy()
    e.close()
    return out


def check_fp32(case, clamp=True, kahan=True):
    ind, wd = run_gpu(case, clamp=clamp, kahan=kahan)
    rind, rwd = O.relight_f32(case.bound, case.idx, case.strength, clamp=clamp, kahan=kahan)
    mx, _ = rel_err(ind[:, :3], rind[:, :3])
    assert mx <= FP32_TOL, mx
    mx2, _ = rel_err(wd[:, :3], rwd[:, :3])
    assert mx2 <= FP32_TOL, mx2
    assert np.all(ind[:, 3] == 1.0) and np.all(wd[:, 3] == 1.0)
    return ind, rind


def test_fp32_config0_full_size(cuda):
    # 128x128, K=64 from a 6x32x32 cubemap, hash params U(-1e-4, 1e-4)
    case = make_case(netconfig.CONFIG_SMALL, 128, 128, 64, seed=0)
    ind, rind = check_fp32(case)
    # the drop-in path evaluates the oracle's exact operation sequence: same bits
    assert np.array_equal(ind.view(np.uint32), rind.view(np.uint32))


@pytest.mark.parametrize("w,h,K,flags", [(1, 1, 1, 1.0), (31, 17, 17, 0.6), (64, 33, 64, 1.0)])
def test_fp32_small_net_edges(cuda, w, h, K, flags):
    case = make_case(netconfig.CONFIG_SMALL, w, h, K, seed=w + K, hash_scale=0.5, flag_prob=flags)
    check_fp32(case)


@pytest.mark.parametrize("K,hs,rnd", [(300, 1e-4, "fp16"), (33, 0.5, "fp32"), (1, 0.5, "fp32")])
def test_fp32_large_net(cuda, K, hs, rnd):
    case = make_case(netconfig.CONFIG_LARGE, 40, 24, K, seed=K, hash_scale=hs, param_round=rnd)
    check_fp32(case)


def test_fp32_clamp_and_kahan_options(cuda):
    case = make_case(netconfig.CONFIG_SMALL, 24, 16, 40, seed=3, hash_scale=0.5, flag_prob=0.8)
    check_fp32(case, clamp=False, kahan=False)
    check_fp32(case, clamp=True, kahan=False)


def test_fp32_all_flags_false_gives_direct_only(cuda):
    case = make_case(netconfig.CONFIG_SMALL, 20, 10, 16, seed=4, flag_prob=0.0)
    ind, wd = run_gpu(case)
    assert np.all(ind[:, :3] == 0)
    assert np.array_equal(wd[:, :3], case.gbuf.direct[:, :3])


def test_fp32_deterministic(cuda):
    case = make_case(netconfig.CONFIG_LARGE, 32, 16, 64, seed=9, hash_scale=0.5)
    a = run_gpu(case)[0]
    b = run_gpu(case)[0]
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_engine_env_from_faces_matches_oracle_and_relights(cuda):
    eng = _eng()
    case = make_case(netconfig.CONFIG_SMALL, 16, 16, 64, seed=12, hash_scale=0.5)
    e = eng.RenderEngine(case.cfg)
    e.loadWeights(case.weights)
    assert not e.TCNNAvaliable()
    em = eng.EnvironmentMap(case.faces)
    eid = e.addEnvironmentMap(em, K=64)
    assert e.TCNNAvaliable()
    idx, st = e.envWavelets(eid)
    assert np.array_equal(idx, case.idx) and np.array_equal(st.view(np.uint32), case.strength.view(np.uint32))
    fr = eng.FullFrame.from_gbuffer(case.gbuf)
    e.setFrame(1, fr)
    e.TCNNPass_p1(1)
    e.TCNNPass_p2(eid, 1)
    e.TCNNSync()
    rind, _ = O.relight_f32(case.bound, case.idx, case.strength)
    assert rel_err(fr.fbPredictedIndirect.cpu().numpy()[:, :3], rind[:, :3])[0] <= FP32_TOL
    e.close()


def test_engine_two_frames_of_different_sizes(cuda):
    eng = _eng()
    c0 = make_case(netconfig.CONFIG_SMALL, 20, 12, 32, seed=21, hash_scale=0.5)
    gb1 = synth.make_gbuffer(7, 9, seed=99)
    e = eng.RenderEngine(c0.cfg)
    e.loadWeights(c0.weights)
    e.addEnvironmentMap(eng.EnvironmentMap(top_coefficients=c0.idx, top_strength=c0.strength))
    f0, f1 = eng.FullFrame.from_gbuffer(c0.gbuf), eng.FullFrame.from_gbuffer(gb1)
    e.setFrame(0, f0)
    e.setFrame(1, f1)
    e.TCNNPass_p1(0)
    e.TCNNPass_p1(1)
    e.TCNNPass_p2(0, 1)
    e.TCNNPass_p2(0, 0)
    e.TCNNSync()
    r0, _ = O.relight_f32(c0.bound, c0.idx, c0.strength)
    b1 = O.Bound(c0.desc, c0.weights, gb1)
    r1, _ = O.relight_f32(b1, c0.idx, c0.strength)
    assert rel_err(f0.fbPredictedIndirect.cpu().numpy()[:, :3], r0[:, :3])[0] <= FP32_TOL
    assert rel_err(f1.fbPredictedIndirect.cpu().numpy()[:, :3], r1[:, :3])[0] <= FP32_TOL
    e.close()


def test_engine_error_paths(cuda):
    import torch
    eng = _eng()
    case = make_case(netconfig.CONFIG_SMALL, 8, 8, 8, seed=1)
    e = eng.RenderEngine(case.cfg)
    fr = eng.FullFrame.from_gbuffer(case.gbuf)
    e.setFrame(0, fr)
    e.TCNNPass_p1(0)
    with pytest.raises(eng.NwprtError) as ei:           # weights missing
        e.addEnvironmentMap(eng.EnvironmentMap(top_coefficients=case.idx, top_strength=case.strength))
        e.TCNNPass_p2(0, 0)
    assert ei.value.status in (eng._lib.NOT_READY,)
    e.loadWeights(case.weights)
    with pytest.raises(eng.NwprtError):                  # frame 3 never prepared
        e.setFrame(3, fr)
        e.TCNNPass_p2(0, 3)
    with pytest.raises(eng.NwprtError) as ei:            # index outside 6*S*S (host check)
        e.addEnvironmentMap(eng.EnvironmentMap(top_coefficients=np.array([0, 6 * 32 * 32], np.int32),
                                               top_strength=np.ones((2, 3), np.float32)))
    assert ei.value.status == eng._lib.INVALID_ARG
    with pytest.raises(eng.NwprtError):                  # face size must match the network
        e.addEnvironmentMap(eng.EnvironmentMap(synth.make_env_faces(16)), K=8)
    bad = fr.fbPredictedIndirect.view(-1)[1:].clone()    # misaligned output
    with pytest.raises(eng.NwprtError):
        from neural_wavelet_prt_demo_b200 import _lib
        import ctypes as C
        s = _lib.lib().nwprt_relight(e._ctx, e.envIds[0], 0, None, C.c_void_p(bad.data_ptr() + 4),
                                     C.c_void_p(fr.fbPredictedIndirectWithDirect.data_ptr()), None)
        _lib.check(s, e._ctx)
    # device-side index check: an out-of-range index supplied in device memory
    idx_d = torch.tensor([3, 1 << 20], dtype=torch.int32, device=cuda)
    st_d = torch.ones((2, 3), dtype=torch.float32, device=cuda)
    from neural_wavelet_prt_demo_b200 import _lib
    import ctypes as C
    env = C.c_int(-1)
    _lib.check(_lib.lib().nwprt_env_from_wavelets(e._ctx, C.c_void_p(idx_d.data_ptr()),
                                                  C.c_void_p(st_d.data_ptr()), 2, 1, None, C.byref(env)), e._ctx)
    with pytest.raises(eng.NwprtError) as ei:
        e.TCNNSync()
    assert ei.value.status == eng._lib.INVALID_ARG
    e.TCNNSync()                                          # error word cleared
    e.close()


def test_init_tcnn_from_npy_directory(cuda, tmp_path):
    eng = _eng()
    case = make_case(netconfig.CONFIG_SMALL, 16, 8, 16, seed=5, hash_scale=0.5)
    np.save(tmp_path / "vtx_enc.npy", case.weights.hash_params)
    np.save(tmp_path / "out_prd.npy", case.weights.out_prd)
    np.save(tmp_path / "cmp_net.npy", case.weights.cmp_net)
    np.save(tmp_path / "wve_enc.npy", case.weights.wve_enc)
    (tmp_path / "config_comp.json").write_text(netconfig.to_json(case.cfg))
    e = eng.RenderEngine(case.cfg)
    e.initTCNN(str(tmp_path))
    info = e.networkInfo()
    assert info.enc_dims == case.desc.enc_dims and info.n_coeffs == case.desc.n_coeffs
    assert info.n_hash_params == case.desc.n_hash_params and info.flops_per_eval == case.desc.flops_per_eval()
    e.addEnvironmentMap(eng.EnvironmentMap(top_coefficients=case.idx, top_strength=case.strength))
    fr = eng.FullFrame.from_gbuffer(case.gbuf)
    e.setFrame(0, fr)
    e.TCNNPass_p1(0)
    e.TCNNPass_p2(0, 0)
    e.TCNNSync()
    rind, _ = O.relight_f32(case.bound, case.idx, case.strength)
    assert rel_err(fr.fbPredictedIndirect.cpu().numpy()[:, :3], rind[:, :3])[0] <= FP32_TOL
    with pytest.raises(eng.NwprtError) as ei:
        e.initTCNN(str(tmp_path / "missing"))
    assert ei.value.status == eng._lib.IO_ERROR
    e.close()

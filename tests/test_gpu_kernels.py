"""GPU parity of the env-map kernels through the C ABI: Haar + top-K (bit-exact),
SH projection (FP32 vs the FP64 oracle) and the SH dot product (bit-exact vs the FP32 oracle)."""
import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import synth
from oracle import oracle as O
from tests.helpers import bits_equal

pytestmark = pytest.mark.gpu


def _engine():
    from neural_wavelet_prt_demo_b200 import engine
    return engine


@pytest.mark.parametrize("S,K", [(1, 1), (1, 6), (2, 5), (4, 96), (8, 64), (8, 384), (16, 300), (32, 64),
                                 (32, 1024), (64, 1), (64, 300), (64, 512), (64, 1024)])
def test_haar_topk_bit_exact(cuda, S, K):
    import torch
    faces = np.stack([synth.make_env_faces(S, seed=S * 7 + K, index=e) for e in range(3)])
    idx, st = _engine().haar_topk(torch.from_numpy(faces).to(cuda), K)
    ridx, rst = O.haar_topk(faces, K)
    assert np.array_equal(idx.cpu().numpy(), ridx)
    assert np.array_equal(st.cpu().numpy().view(np.uint32), rst.view(np.uint32))


def test_haar_topk_ties_nan_inf_bit_exact(cuda):
    import torch
    S = 8
    g = np.random.default_rng(11)
    faces = g.integers(0, 3, size=(4, 6, S, S, 3)).astype(np.float32)  # many equal keys
    faces[0, 1, 3, 4] = np.nan
    faces[1, 2, 0, 0, 1] = np.inf
    faces[2, 5, 7, 7, 2] = -np.inf
    faces[3] = 1.0                                                     # all-constant faces
    for K in (1, 17, 64, 6 * S * S):
        idx, st = _engine().haar_topk(torch.from_numpy(faces).to(cuda), K)
        ridx, rst = O.haar_topk(faces, K)
        assert np.array_equal(idx.cpu().numpy(), ridx), K
        assert bits_equal(st.cpu().numpy(), rst), K


def test_haar_topk_large_batch(cuda):
    import torch
    S, K, E = 64, 300, 96
    faces = np.stack([synth.make_env_faces(S, seed=3, index=e) for e in range(E)])
    idx, st = _engine().haar_topk(torch.from_numpy(faces).to(cuda), K)
    ridx, rst = O.haar_topk(faces, K)
    assert np.array_equal(idx.cpu().numpy(), ridx)
    assert np.array_equal(st.cpu().numpy().view(np.uint32), rst.view(np.uint32))


@pytest.mark.parametrize("S,K", [(64, 300), (64, 1024), (32, 64), (8, 384), (4, 17), (2, 24), (1, 6)])
def test_haar_topk_batched_and_single_map_forms_agree(cuda, S, K):
    """Batches of 32 maps or more run the batched kernel (one CTA per map), single maps the
    cluster kernel (one CTA per face): both give the oracle's bits, ties and non-finite
    texels included."""
    import torch
    E = 40
    g = np.random.default_rng(S + K)
    faces = np.stack([synth.make_env_faces(S, seed=5, index=e) for e in range(E)])
    faces[3] = g.integers(0, 3, size=(6, S, S, 3)).astype(np.float32)   # many equal keys
    faces[7] = 1.0                                                      # constant map
    faces[9, 1, 0, 0, 0] = np.nan
    faces[11, 4, S - 1, S - 1, 2] = np.inf
    # the selection's shortcuts: winners packed into a few texel blocks (the per-block maxima
    # bound the threshold loosely), a dynamic range wider than the first pass's window (fewer
    # than K keys in it: the full passes run), all zeros, negative texels
    h = max(1, S // 4)
    faces[13, 2, :h, :h, :] *= 1e4
    faces[15, 0, 0, 0, :] = 1e30
    faces[17] = 0.0
    faces[19] = -faces[19]
    tf = torch.from_numpy(faces).to(cuda)
    idx, st = _engine().haar_topk(tf, K)
    ridx, rst = O.haar_topk(faces, K)
    assert np.array_equal(idx.cpu().numpy(), ridx)
    assert bits_equal(st.cpu().numpy(), rst)
    for e in (0, 3, 7, 9, 11, 13, 15, 17, E - 1):
        i1, s1 = _engine().haar_topk(tf[e:e + 1].contiguous(), K)
        assert np.array_equal(i1.cpu().numpy()[0], ridx[e]), e
        assert bits_equal(s1.cpu().numpy()[0], rst[e]), e


def test_haar_topk_rejects_bad_sizes(cuda):
    import torch
    eng = _engine()
    with pytest.raises(eng.NwprtError):
        eng.haar_topk(torch.zeros((6, 128, 128, 3), device=cuda), 8)
    with pytest.raises(eng.NwprtError):
        eng.haar_topk(torch.zeros((6, 16, 16, 3), device=cuda), 1025)
    with pytest.raises(eng.NwprtError):
        eng.haar_topk(torch.zeros((6, 2, 2, 3), device=cuda), 25)


@pytest.mark.parametrize("S", [1, 16, 64, 128])
def test_sh_project_vs_f64_oracle(cuda, S):
    import torch
    faces = synth.make_env_faces(S, seed=S)
    L = _engine().sh_project(torch.from_numpy(faces).to(cuda)).cpu().numpy().astype(np.float64)
    ref, ref_abs = O.sh_project_f64(faces)
    assert np.all(np.abs(L - ref) <= 1e-5 * ref_abs + 1e-7)


@pytest.mark.parametrize("N", [1, 127, 128, 1000, 4097, 128 * 300 + 5])
@pytest.mark.parametrize("abs_out", [True, False])
def test_sh_dot_bit_exact(cuda, N, abs_out):
    import torch
    T = synth.make_sh_transport(N, seed=N)
    L = np.random.default_rng(N).normal(size=(81, 3)).astype(np.float32)
    out = _engine().sh_dot(torch.from_numpy(T).to(cuda), torch.from_numpy(L).to(cuda), abs_out=abs_out)
    ref = O.sh_dot_f32(T, L, abs_out=abs_out)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_sh_dot_1080p_sampled(cuda):
    import torch
    N = 1920 * 1080
    g = torch.Generator(device=cuda).manual_seed(0)
    l = torch.floor(torch.sqrt(torch.arange(81, device=cuda, dtype=torch.float32))).clamp_min(1)
    T = torch.randn((N, 81), generator=g, device=cuda) / (l * l)
    L = torch.randn((81, 3), generator=g, device=cuda)
    out = _engine().sh_dot(T, L)
    rows = np.random.default_rng(0).choice(N, 4096, replace=False)
    ref = O.sh_dot_f32(T[rows].cpu().numpy(), L.cpu().numpy())
    assert np.array_equal(out[rows].cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_tonemap_bit_exact(cuda):
    import torch
    eng = _engine()
    g = np.random.default_rng(11)
    n = 300_001
    x = np.concatenate([g.uniform(0, 1.5, n * 2), 10.0 ** g.uniform(-7, 2, n * 2)]).astype(np.float32)
    src = x[: n * 4].reshape(n, 4).copy()
    src[:16, :3] = np.array([0, 0.5, 1, -1, np.nan, np.inf, -np.inf, 1e-8, 3e38, 0.18, 2, 1e-3, 0.04,
                             0.0031308, 0.99, 1.01], np.float32).reshape(16, 1)
    # every step of the byte function, +-8 ulps
    t = O.srgb_thresholds()[1:].view(np.int32)
    near = (t[:, None] + np.arange(-8, 9, dtype=np.int32)[None, :]).ravel().view(np.float32)
    src[16:16 + near.size // 3 * 1, :3] = np.resize(near, (near.size // 3 * 1, 3))
    got = eng.tonemap_srgb(torch.from_numpy(src).to(cuda)).cpu().numpy().view(np.uint32)
    assert np.array_equal(got, O.tonemap_srgb(src))
    with pytest.raises(ValueError):
        eng.tonemap_srgb(torch.zeros((4, 3), device=cuda))
    assert eng.tonemap_srgb(torch.zeros((0, 4), device=cuda)).numel() == 0


def test_final_pixel_colors_of_a_relit_frame(cuda):
    from neural_wavelet_prt_demo_b200 import netconfig
    from tests.helpers import make_case
    eng = _engine()
    case = make_case(netconfig.CONFIG_SMALL, 40, 24, 32, seed=4, hash_scale=0.5)
    e = eng.RenderEngine(case.cfg)
    e.loadWeights(case.weights)
    env = e.addEnvironmentMap(eng.EnvironmentMap(top_coefficients=case.idx, top_strength=case.strength))
    fr = eng.FullFrame.from_gbuffer(case.gbuf)
    e.setFrame(0, fr)
    e.TCNNPass_p1(0)
    e.TCNNPass_p2(env, 0, eng.RenderConfig(precision="fp32"))
    full = e.computeFinalPixelColors(0).cpu().numpy().view(np.uint32)
    ind = e.computeFinalPixelColors(0, "indirect").cpu().numpy().view(np.uint32)
    e.TCNNSync()
    assert np.array_equal(full, O.tonemap_srgb(fr.fbPredictedIndirectWithDirect.cpu().numpy()))
    assert np.array_equal(ind, O.tonemap_srgb(fr.fbPredictedIndirect.cpu().numpy()))
    with pytest.raises(ValueError):
        e.computeFinalPixelColors(0, "direct")
    e.close()


@pytest.mark.parametrize("V,n", [(1, 81), (37, 81), (1000, 81), (33, 9), (17, 1), (5, 4)])
def test_sh_vertex_radiance_bit_exact(cuda, V, n):
    import torch
    from neural_wavelet_prt_demo_b200 import synth
    eng = _engine()
    T, brdf, _, _ = synth.make_sh_mesh(V, 1, 81, seed=V)
    T, brdf = T[:, :n, :n].copy(), brdf[:, :n].copy()
    L = synth.make_sh_transport(3, 81, seed=5).T[:n].copy()
    got = eng.sh_vertex_radiance(*(torch.from_numpy(a).to(cuda) for a in (T, brdf, L))).cpu().numpy()
    assert np.array_equal(got.view(np.uint32), O.sh_vertex_radiance(T, brdf, L).view(np.uint32))


def test_sh_interpolate_bit_exact_and_bad_index(cuda):
    import torch
    from neural_wavelet_prt_demo_b200 import netconfig, synth
    eng = _engine()
    T, brdf, tri, uv = synth.make_sh_mesh(64, 50_000, 81, seed=3)
    L = synth.make_sh_transport(3, 81, seed=5).T.copy()
    vc = O.sh_vertex_radiance(T, brdf, L)
    tri[7] = [0, 64, 1]  # out of range
    e = eng.RenderEngine(netconfig.CONFIG_SMALL)
    got = e.shInterpolate(*(torch.from_numpy(a).to(cuda) for a in (vc, tri, uv))).cpu().numpy()
    ref, bad = O.sh_interpolate(vc, tri, uv)
    assert bad == 1 and np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    with pytest.raises(eng.NwprtError):
        e.TCNNSync()
    e.close()

"""CPU tests of the oracle: known answers, the numpy twin, and the reference's own kernels.

The reference ships no tests or golden data for this path; the oracle is pinned here by
(1) analytic known answers, (2) an independent numpy restatement, (3) the reference's
own utils_kernels.h compiled for the host (oracle/_ref), and (4) the committed fixtures of
tests/golden/ (checked in tests/test_golden.py).
"""
import math

import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import netconfig, synth
from oracle import oracle as O
from oracle import oracle_np as ON
from tests.helpers import make_case, rel_err


# ------------------------------------------------------------------ Haar + top-K

@pytest.mark.parametrize("S", [1, 2, 4, 16, 64])
def test_haar_constant_face_is_one_dc_coefficient(S):
    face = np.full((S, S, 3), 0.75, np.float32)
    c = O.haar_face(face)
    assert np.allclose(c[0, 0], 0.75 * S)
    c[0, 0] = 0
    assert not np.any(c)


@pytest.mark.parametrize("S", [2, 8, 32, 64])
def test_haar_is_orthonormal_and_invertible(S):
    face = synth.make_env_faces(S, seed=S)[0]
    c = O.haar_face(face)
    e_in, e_out = np.sum(face.astype(np.float64) ** 2), np.sum(c.astype(np.float64) ** 2)
    assert abs(e_in - e_out) <= 1e-5 * e_in
    back = O.haar_inverse_f64(c)
    assert np.allclose(back, face, rtol=1e-5, atol=1e-6 * np.abs(face).max())


@pytest.mark.parametrize("S,K,seed", [(1, 6, 0), (2, 5, 1), (8, 64, 2), (32, 64, 3), (64, 300, 4), (64, 1024, 5)])
def test_topk_matches_numpy_twin_bit_exact(S, K, seed):
    faces = synth.make_env_faces(S, seed=seed)
    idx, st = O.haar_topk(faces, K)
    idx2, st2 = ON.haar_topk(faces, K)
    assert np.array_equal(idx, idx2)
    assert np.array_equal(st.view(np.uint32), st2.view(np.uint32))
    for f in range(6):
        assert np.array_equal(O.haar_face(faces[f]).view(np.uint32), ON.haar_face(faces[f]).view(np.uint32))


def test_topk_order_is_key_desc_then_index_asc_with_ties_and_nonfinite():
    S = 16
    g = np.random.default_rng(7)
    faces = g.integers(0, 3, size=(6, S, S, 3)).astype(np.float32)  # many equal keys
    faces[1, 3, 4] = np.nan
    faces[2, 0, 0, 1] = np.inf
    K = 6 * S * S
    idx, st = O.haar_topk(faces, K)
    idx2, st2 = ON.haar_topk(faces, K)
    assert np.array_equal(idx, idx2)
    assert sorted(idx.tolist()) == list(range(K))  # a permutation when K = all
    keys = np.array([O.wavelet_key(*s) for s in st], np.float32)
    for a in range(K - 1):
        assert keys[a] > keys[a + 1] or (keys[a] == keys[a + 1] and idx[a] < idx[a + 1])


def test_topk_rejects_bad_k():
    with pytest.raises(ValueError):
        O.haar_topk(synth.make_env_faces(4, seed=0), 6 * 16 + 1)


# ------------------------------------------------------------------ SH

def test_sh_basis_known_values():
    c1 = math.sqrt(3.0 / (4.0 * math.pi))
    for d in ([0.0, 0.0, 1.0], [0.6, 0.0, 0.8], [0.0, -0.6, 0.8], [0.36, 0.48, 0.8]):
        Y = O.sh_eval_f64(d)
        assert abs(Y[0] - 0.28209479177387814) < 1e-14
        assert abs(Y[1] - (-c1 * d[1])) < 1e-13
        assert abs(Y[2] - (c1 * d[2])) < 1e-13
        assert abs(Y[3] - (-c1 * d[0])) < 1e-13


def test_sh_projection_of_a_basis_function_is_a_unit_vector():
    S = 64
    faces = np.zeros((6, S, S, 3), np.float32)
    # fill the cubemap with Y_6 (l=2, m=0) evaluated at each texel direction
    dirs = {0: lambda u, v: (1, v, u), 1: lambda u, v: (-1, v, -u), 2: lambda u, v: (u, 1, v),
            3: lambda u, v: (u, -1, -v), 4: lambda u, v: (u, v, -1), 5: lambda u, v: (-u, v, 1)}
    for f in range(6):
        for r in range(S):
            for c in range(S):
                u, v = 2 * (c + 0.5) / S - 1, 2 * (r + 0.5) / S - 1
                d = np.array(dirs[f](u, v), np.float64)
                d /= np.linalg.norm(d)
                faces[f, r, c, :] = O.sh_eval_f64(d)[6]
    L, _ = O.sh_project_f64(faces)
    assert abs(L[6, 0] - 1.0) < 2e-3
    others = np.delete(L[:, 0], 6)
    assert np.abs(others).max() < 2e-3


def test_sh_dot_f32_vs_f64():
    T = synth.make_sh_transport(1000, seed=3)
    L = np.random.default_rng(0).normal(size=(81, 3)).astype(np.float32)
    out = O.sh_dot_f32(T, L)
    ref = O.sh_dot_f64(T, L.astype(np.float64))
    assert np.allclose(out[:, :3], ref, rtol=1e-5, atol=1e-5 * np.abs(ref).max())
    assert np.all(out[:, 3] == 1.0)


# ------------------------------------------------------------------ relight

@pytest.mark.parametrize("cfg", [netconfig.CONFIG_SMALL, netconfig.CONFIG_LARGE], ids=["small", "large"])
def test_relight_c_f64_matches_numpy_twin(cfg):
    case = make_case(cfg, 12, 7, 24, seed=11, hash_scale=0.5, flag_prob=0.7)
    r64 = O.relight_f64(case.bound, case.idx, case.strength)
    rnp = ON.relight_f64(case.desc, case.weights, case.gbuf, case.idx, case.strength)
    assert np.abs(r64 - rnp).max() <= 1e-12 * np.abs(rnp).max()


@pytest.mark.parametrize("cfg", [netconfig.CONFIG_SMALL, netconfig.CONFIG_LARGE], ids=["small", "large"])
def test_relight_f32_close_to_f64(cfg):
    case = make_case(cfg, 16, 9, 40, seed=5, hash_scale=0.5)
    ind, wd = O.relight_f32(case.bound, case.idx, case.strength)
    r64 = O.relight_f64(case.bound, case.idx, case.strength)
    mx, _ = rel_err(ind[:, :3], r64)
    assert mx < 1e-3                                    # FP32 accuracy, per pixel
    assert np.abs(ind[:, :3] - r64).max() < 1e-5 * np.abs(r64).max()
    assert np.array_equal(wd[:, :3], ind[:, :3] + case.gbuf.direct[:, :3])
    assert np.all(ind[:, 3] == 1) and np.all(wd[:, 3] == 1)


def test_relight_flag_gates_and_clamp_option():
    case = make_case(netconfig.CONFIG_SMALL, 10, 10, 16, seed=2, hash_scale=0.5, flag_prob=0.5)
    ind, _ = O.relight_f32(case.bound, case.idx, case.strength)
    off = case.gbuf.flag == 0
    assert off.any() and np.all(ind[off, :3] == 0)
    assert np.all(ind[:, :3] >= 0)                      # clamped terms are non-negative
    ind2, _ = O.relight_f32(case.bound, case.idx, case.strength, clamp=False)
    assert np.any(ind2[~off, :3] < ind[~off, :3])


def test_hash_encoding_dense_and_hashed_levels_vs_numpy():
    case = make_case(netconfig.CONFIG_SMALL, 4, 4, 4, seed=9, hash_scale=1.0)
    pos = np.random.default_rng(1).uniform(-0.1, 1.1, size=(64, 3)).astype(np.float32)
    pos[0] = [1.0, 1.0, 1.0]
    pos[1] = [0.0, 0.0, 0.0]
    ref = ON.hash_encode_f64(case.desc, case.weights.hash_params, pos)
    for i in range(pos.shape[0]):
        c64 = O.hash_encode_f64(case.bound, pos[i])
        assert np.abs(c64 - ref[i]).max() < 1e-12
        c32 = O.hash_encode_f32(case.bound, pos[i])
        assert np.abs(c32 - ref[i]).max() < 1e-5


# ------------------------------------------------------------------ pinned against the reference's kernels

ref = pytest.mark.skipif(O.ref_lib() is None, reason="oracle/_ref not built (needs the reference tree)")


@ref
def test_remap_matches_reference_waveletDataCopy():
    case = make_case(netconfig.CONFIG_SMALL, 9, 5, 4, seed=4)
    r = O.ref_wavelet_data_copy(case.gbuf)
    mine = np.stack([O.remap_f32(case.bound, p) for p in range(case.gbuf.n)])
    for k in range(r.shape[1]):
        # 15 of 16 columns bit for bit; the roughness log (column 9) is the correctly
        # rounded one, which the C library's logf misses by 1 ulp in ~0.1% of inputs
        cols = [c for c in range(16) if c != 9]
        assert np.array_equal(r[:, k][:, cols].view(np.uint32), mine[:, cols].view(np.uint32))
        ulp = np.abs(r[:, k, 9].view(np.int32).astype(np.int64) - mine[:, 9].view(np.int32).astype(np.int64))
        assert ulp.max() <= 1


def test_series_log_is_correctly_rounded():
    import ctypes as C
    L = O.lib()
    L.orc_logf_series.restype = C.c_float
    L.orc_logf_series.argtypes = [C.c_float]
    g = np.random.default_rng(0)
    xs = np.concatenate([g.uniform(1, 26, 20000), 2.0 ** g.uniform(-120, 120, 5000)]).astype(np.float32)
    got = np.array([L.orc_logf_series(float(x)) for x in xs], np.float32)
    cr = np.log(xs.astype(np.float64)).astype(np.float32)
    assert np.array_equal(got.view(np.uint32), cr.view(np.uint32))
    assert np.isnan(L.orc_logf_series(-1.0)) and L.orc_logf_series(0.0) == -np.inf


@ref
def test_clamped_sum_matches_reference_computeResponse():
    gb = synth.make_gbuffer(7, 6, seed=8, flag_prob=0.6)
    g = np.random.default_rng(3)
    T = g.normal(size=(gb.n, 64, 3)).astype(np.float32)
    L = g.normal(size=(64, 3)).astype(np.float32)
    ind, wd = O.ref_compute_response(gb, T, L)
    s = np.zeros((gb.n, 3), np.float32)
    for k in range(64):  # the oracle's plain (kahan=0) clamped sum, k ascending
        s = s + np.maximum(L[k][None] * T[:, k], np.float32(0))
    s[gb.flag == 0] = 0
    assert np.array_equal(ind[:, :3], s)
    assert np.array_equal(wd[:, :3], s + gb.direct[:, :3])
    assert np.all(ind[:, 3] == 1) and np.all(wd[:, 3] == 1)


@ref
def test_embedding_gather_matches_reference_ptwise_mlt():
    # the reference hard-codes 64 wavelets and a 6*64*64 coefficient space (utils_kernels.h:121-126)
    case = make_case(netconfig.CONFIG_LARGE, 3, 2, 64, seed=6, hash_scale=0.5)
    D, n = case.desc.enc_dims, case.gbuf.n
    enc = np.stack([O.hash_encode_f32(case.bound, case.gbuf.pos[p, :3]) for p in range(n)])
    enc_fm = np.repeat(enc, 64, axis=0).T.copy()                  # [D, n*64], column = p*64 + k
    out = O.ref_ptwise_mlt(enc_fm, case.weights.wve_enc.ravel(), case.idx)
    mine = enc[:, None, :] * case.weights.wve_enc[:, case.idx].T[None]   # [n, 64, D] float32
    assert np.array_equal(out.T.reshape(n, 64, D), mine.astype(np.float32))


# ---------------------------------------------------------------- final-colour pass (tonemap)

def test_powf_series_matches_double_pow():
    """The series x^(1/2.4) rounds to the float nearest the float64 power (tie cases aside)."""
    g = np.random.default_rng(5)
    x = np.concatenate([g.uniform(0, 4, 4000), 10.0 ** g.uniform(-8, 3, 4000)]).astype(np.float32)
    y = np.float32(1.0) / np.float32(2.4)
    got = O.powf_series(x, y)
    ref = np.power(x.astype(np.float64), float(y)).astype(np.float32)
    ulps = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
    assert ulps.max() <= 1 and np.mean(ulps == 0) > 0.999


def test_tonemap_known_answers_and_edges():
    x = np.array([0, 0.5, 1, 1e-3, 0.18, 2.0, -1, np.nan, np.inf, -np.inf, 1e-8, 3e38], np.float32)
    src = np.stack([x, x, x, np.ones_like(x)], 1)
    t = O.tonemap_srgb(src)
    r = t & 255
    assert list(r) == [0, 188, 255, 1, 118, 255, 0, 0, 255, 0, 0, 255]
    assert np.all((t >> 24) == 255)
    assert np.all(((t >> 8) & 255) == r) and np.all(((t >> 16) & 255) == r)


def test_tonemap_against_float64_formula():
    """Bytes equal floor(255.9 * clamp(1.055 (x + 1e-6)^(1/2.4) - 0.055)) evaluated in float64,
    except where that value lies within float rounding of an integer."""
    g = np.random.default_rng(6)
    x = np.concatenate([g.uniform(0, 1.2, 20000), 10.0 ** g.uniform(-6, 1, 20000)]).astype(np.float32)
    src = np.stack([x, np.roll(x, 1), np.roll(x, 2), np.zeros_like(x)], 1)
    got = O.tonemap_srgb(src)
    for c in range(3):
        xc = src[:, c].astype(np.float64)
        f = np.clip(1.055 * np.power(xc + np.float64(np.float32(1e-6)), 1 / 2.4) - 0.055, 0, 1) * 255.9
        want = np.floor(f).astype(np.int64)
        byte = (got >> (8 * c)) & 255
        near = np.abs(f - np.round(f)) < 1e-4
        assert np.array_equal(byte[~near], want[~near])


def test_srgb_step_table_equals_formula_near_every_step():
    """The final-colour kernel maps a channel to the number of step thresholds at or below it;
    around every threshold (+-4096 ulps) that count equals the direct formula."""
    t = O.srgb_thresholds()
    assert np.all(np.diff(t[1:]) > 0) and t[1] > 0
    assert O.srgb_threshold_mismatches(t, 4096) == 0
    # between thresholds the byte is constant: spot-check the midpoints
    mid = ((t[1:-1].view(np.uint32).astype(np.uint64) + t[2:].view(np.uint32)) // 2).astype(np.uint32).view(np.float32)
    src = np.stack([mid, mid, mid, mid], 1)
    assert np.array_equal(O.tonemap_srgb(src) & 255, np.arange(1, 255, dtype=np.uint32))


# ---------------------------------------------------------------- per-vertex SH path

def test_sh_vertex_radiance_matches_float64():
    from neural_wavelet_prt_demo_b200 import synth
    T, brdf, tri, uv = synth.make_sh_mesh(20, 50, 81, seed=1)
    L = synth.make_sh_transport(3, 81, seed=2).T.copy()  # [81, 3]
    got = O.sh_vertex_radiance(T, brdf, L)
    ref = np.abs(np.einsum("vkj,jc,vkc->vc", T.astype(np.float64), L.astype(np.float64), brdf.astype(np.float64)))
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()
    # lower degree: the leading 4 or 9 coefficients
    for n in (1, 4, 9):
        g = O.sh_vertex_radiance(T[:, :n, :n].copy(), brdf[:, :n].copy(), L[:n].copy())
        r = np.abs(np.einsum("vkj,jc,vkc->vc", T[:, :n, :n].astype(np.float64), L[:n].astype(np.float64),
                             brdf[:, :n].astype(np.float64)))
        assert np.abs(g - r).max() <= 1e-5 * max(np.abs(r).max(), 1e-30)


def test_sh_interpolate_barycentric():
    vc = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    tri = np.array([[0, 1, 2], [0, 1, 2], [2, 1, 0], [0, 1, 5]], np.int32)
    uv = np.array([[0, 0], [0.25, 0.5], [1, 0], [0.5, 0.5]], np.float32)
    out, bad = O.sh_interpolate(vc, tri, uv)
    assert bad == 1
    assert np.array_equal(out[0], [1, 0, 0, 1]) and np.allclose(out[1], [0.25, 0.25, 0.5, 1])
    assert np.array_equal(out[2], [0, 1, 0, 1]) and np.array_equal(out[3], [0, 0, 0, 1])

"""Why FP8 E4M3 is not a served form: a numerical model of the tensor-core relight's operand
rounding on the config-2 network (1080p frame, K=300), against the FP64 network.

The model rounds what the kernel rounds -- the operand of every tensor-core layer (out_prd's
output layer folded into cmp_net's first layer, the aux block kept in BF16), FP32/FP64
accumulation, the 64->3 output layer in full precision -- and reports PSNR of the clamped
radiance sum over 256 random pixels.  It reproduces the GPU's measured figures (BF16 ~58 dB,
FP8 with per-layer scales ~36 dB), and shows that block scaling (one power-of-two scale per
32-element K block, the MXFP8 form of tcgen05.mma.kind::mxf8f6f4.block_scale) does not help:
E4M3 keeps 3 mantissa bits against BF16's 7, and the error is rounding, not range."""
import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import netconfig, synth
from oracle import oracle as O


def _round_mantissa(x, bits):
    m, e = np.frexp(x)
    return np.ldexp(np.round(m * 2.0 ** bits) / 2.0 ** bits, e)


def bf16(x):
    return _round_mantissa(x, 8)


def e4m3(x):
    """Round to E4M3: 3 mantissa bits, normal exponents down to -6 (subnormal steps 2^-9),
    saturated at 448; ties to even (np.round)."""
    a = np.abs(x)
    e = np.maximum(np.floor(np.log2(np.where(a > 0, a, 1.0))), -6)
    step = 2.0 ** (e - 3)
    return np.clip(np.round(x / step) * step, -448, 448)


def mx_blocks(x, block=32):
    """E4M3 with one power-of-two scale per `block` consecutive K elements (UE8M0)."""
    k = x.shape[-1]
    pad = (-k) % block
    xp = np.concatenate([x, np.zeros(x.shape[:-1] + (pad,))], -1) if pad else x
    blk = xp.reshape(x.shape[:-1] + (-1, block))
    amax = np.abs(blk).max(-1, keepdims=True)
    sc = 2.0 ** np.ceil(np.log2(np.where(amax > 0, amax, 1.0) / 448.0))
    return (e4m3(blk / sc) * sc).reshape(xp.shape)[..., :k]


@pytest.fixture(scope="module")
def net():
    desc = netconfig.parse(netconfig.CONFIG_LARGE)
    w = synth.make_weights(desc, seed=0, hash_scale=1e-4, param_round="fp16")
    gb = synth.make_gbuffer(1920, 1080, seed=1)
    idx, st = O.haar_topk(synth.make_env_faces(desc.face_size, seed=2), 300)
    b = O.Bound(desc, w, gb)

    def layers(flat, shapes):
        out, o = [], 0
        for n_in, n_out in shapes:
            out.append(flat[o:o + n_in * n_out].reshape(n_out, n_in).astype(np.float64))
            o += n_in * n_out
        return out

    wop, wcn = layers(w.out_prd, desc.op_layers()), layers(w.cmp_net, desc.cn_layers())
    m = wop[-1].shape[0]
    fold = wcn[0][:, :m] @ wop[-1]
    ops = wop[:-1] + [fold] + wcn[1:-1]          # the tensor-core layers
    emb = w.wve_enc.reshape(desc.enc_dims, -1).astype(np.float64)[:, idx].T
    pix = np.sort(np.random.default_rng(0).choice(gb.n, 256, replace=False))
    data = []
    for p in pix:
        row = O.remap_f32(b, int(p))
        data.append((O.hash_encode_f64(b, row[:3]), np.concatenate([row[3:16].astype(np.float64), np.ones(3)])))
    return ops, wcn[0][:, m:], wcn[-1], len(wop) - 1, emb, st.astype(np.float64), data


def _radiance(net, q_act, q_w):
    ops, w_aux, v_last, aux_layer, emb, st, data = net
    out = []
    for enc, aux in data:
        h = enc[None, :] * emb
        for li, W in enumerate(ops):
            z = q_act(h, li) @ q_w(W).T
            if li == aux_layer:
                z += bf16(aux)[None, :] @ bf16(w_aux).T
            h = np.maximum(z, 0)
        out.append(np.maximum((h @ v_last.T) * st, 0).sum(0))
    return np.array(out)


def _psnr(x, ref):
    return 10 * np.log10(np.abs(ref).max() ** 2 / np.mean((x - ref) ** 2))


def test_fp8_cannot_reach_the_45db_bar(net):
    ident = lambda x, *a: x
    ref = _radiance(net, ident, ident)
    # per-layer activation maxima of the exact network (the calibration the kernel performs)
    amax = []
    ops, w_aux, _, aux_layer, emb, _, data = net
    for li in range(len(ops)):
        m = 0.0
        for enc, aux in data[:64]:
            h = enc[None, :] * emb
            for lj in range(li):
                z = h @ ops[lj].T + (aux[None, :] @ w_aux.T if lj == aux_layer else 0)
                h = np.maximum(z, 0)
            m = max(m, float(np.abs(h).max()))
        amax.append(m)
    p_bf16 = _psnr(_radiance(net, lambda h, li: bf16(h), bf16), ref)
    per_layer = lambda h, li: e4m3(h * (240 / amax[li])) / (240 / amax[li])
    p_fp8 = _psnr(_radiance(net, per_layer, lambda W: e4m3(W * (240 / np.abs(W).max())) / (240 / np.abs(W).max())), ref)
    p_mx = _psnr(_radiance(net, lambda h, li: mx_blocks(h), mx_blocks), ref)
    print(f"model PSNR vs FP64: BF16 {p_bf16:.1f} dB, FP8 per-layer {p_fp8:.1f} dB, FP8 block-scaled {p_mx:.1f} dB")
    assert 55 <= p_bf16 <= 62        # the GPU measures 57.6-58.4 dB on this network
    assert 32 <= p_fp8 <= 39         # the GPU measures 35.2-36.0 dB
    assert p_mx < 40 and p_fp8 < 45 and p_mx < 45

"""Network description for the neural wavelet PRT relight path.

The reference builds its network from ``config_comp.json`` with the four keys
``vtx_enc`` / ``cmp_enc`` / ``out_prd`` / ``cmp_net``
(Renderer/tinycudann/prt_network.h:38-61).  That JSON and the tiny-cuda-nn
factories it feeds are not shipped with the reference, so this module pins the
meaning of every key we accept.  The same JSON text is parsed by the native
library (``csrc/config.cpp``) and by the CPU oracle driver; both derive
the same numbers from it with the formulas below.

Composite network (prt_network.h:73-154), per pixel p and selected wavelet k:

* ``vtx_enc``  multiresolution hash grid (Instant-NGP, Mueller et al. 2022) of
  the bbox-normalised first-hit position -> D = n_levels * n_features_per_level.
* wavelet embedding ``wve_enc``: E[D][n_coeffs], dimension-major, gathered at
  the wavelet's coefficient index (utils_kernels.h:110-127); cp = enc * E[:, idx_k].
* ``out_prd``  bias-free ReLU MLP  D -> n_neurons x n_hidden_layers -> n_output_dims
  (default 64, prt_network.h:50-52), linear output.
* ``cmp_enc``  identity encoding of the 13 auxiliary G-buffer values (rows 3..15
  of the 16-float input row, prt_globals.h:4-13) padded with ones to
  ``n_padded_dims`` so that the bias-free MLP sees a constant input.
* ``cmp_net``  bias-free ReLU MLP [out_prd || aux] -> n_neurons x n_hidden_layers -> 3.

Weight layout (our own, documented; the tcnn parameter layout is not available):
every dense layer is a row-major float32 matrix [out][in]; the layers of a
network are concatenated in evaluation order.  Hash-grid parameters are
float32 [sum_l T_l][F]; level l holds T_l = min(2**log2_hashmap_size, (N_l+1)**3)
entries with N_l = floor(base_resolution * per_level_scale**l).
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from typing import List

N_AUX_INPUTS = 13  # prt_globals.h:6 INPUT_AUX_SIZE


# Config 0: 128x128 parity network.  cmp_net is 42->64->64->3: its 42 inputs are
# out_prd's 26 outputs followed by the 16-wide padded aux encoding.
CONFIG_SMALL = {
    "vtx_enc": {"otype": "HashGrid", "n_levels": 8, "n_features_per_level": 2,
                "log2_hashmap_size": 16, "base_resolution": 16, "per_level_scale": 1.5},
    "cmp_enc": {"otype": "Identity", "n_padded_dims": 16},
    "out_prd": {"otype": "FullyFusedMLP", "activation": "ReLU", "output_activation": "None",
                "n_neurons": 64, "n_hidden_layers": 0, "n_output_dims": 26},
    "cmp_net": {"otype": "FullyFusedMLP", "activation": "ReLU", "output_activation": "None",
                "n_neurons": 64, "n_hidden_layers": 2},
    "wve_enc": {"face_size": 32},
}

# Config 2/3/4: 1080p network.  16 levels x 2 features, 2^19 table, 64-wide MLPs with
# 3 hidden layers: out_prd 32->64->64->64->64, cmp_net (64||16)->64->64->64->3.
CONFIG_LARGE = {
    "vtx_enc": {"otype": "HashGrid", "n_levels": 16, "n_features_per_level": 2,
                "log2_hashmap_size": 19, "base_resolution": 16, "per_level_scale": 1.5},
    "cmp_enc": {"otype": "Identity", "n_padded_dims": 16},
    "out_prd": {"otype": "FullyFusedMLP", "activation": "ReLU", "output_activation": "None",
                "n_neurons": 64, "n_hidden_layers": 3, "n_output_dims": 64},
    "cmp_net": {"otype": "FullyFusedMLP", "activation": "ReLU", "output_activation": "None",
                "n_neurons": 64, "n_hidden_layers": 3},
    "wve_enc": {"face_size": 64},
}


@dataclass
class NetDesc:
    n_levels: int
    n_features: int
    log2_table: int
    base_resolution: int
    per_level_scale: float
    aux_width: int
    op_neurons: int
    op_hidden: int
    op_out: int
    cn_neurons: int
    cn_hidden: int
    face_size: int
    level_res: List[int] = field(default_factory=list)
    level_size: List[int] = field(default_factory=list)
    level_offset: List[int] = field(default_factory=list)

    # ---- derived sizes -------------------------------------------------
    @property
    def enc_dims(self) -> int:
        return self.n_levels * self.n_features

    @property
    def n_coeffs(self) -> int:
        return 6 * self.face_size * self.face_size

    @property
    def cmp_in(self) -> int:
        return self.op_out + self.aux_width

    def op_layers(self):
        """(in, out) of every out_prd layer, evaluation order."""
        return _mlp_shapes(self.enc_dims, self.op_neurons, self.op_hidden, self.op_out)

    def cn_layers(self):
        return _mlp_shapes(self.cmp_in, self.cn_neurons, self.cn_hidden, 3)

    @property
    def n_hash_params(self) -> int:
        return sum(self.level_size) * self.n_features

    @property
    def n_op_params(self) -> int:
        return sum(i * o for i, o in self.op_layers())

    @property
    def n_cn_params(self) -> int:
        return sum(i * o for i, o in self.cn_layers())

    def flops_per_eval(self) -> int:
        """Multiply-add FLOPs per (pixel, wavelet) evaluation, aux layer-1 part hoisted.

        The aux columns of cmp_net's first layer are the same for all K wavelets of a
        pixel, so their product is a per-pixel cost and is not counted per eval.
        """
        f = sum(2 * i * o for i, o in self.op_layers())
        for li, (i, o) in enumerate(self.cn_layers()):
            if li == 0:
                i = self.op_out
            f += 2 * i * o
        return f


def _mlp_shapes(n_in: int, width: int, n_hidden: int, n_out: int):
    if n_hidden == 0:
        return [(n_in, n_out)]
    shapes = [(n_in, width)]
    shapes += [(width, width)] * (n_hidden - 1)
    shapes.append((width, n_out))
    return shapes


def level_layout(n_levels, base, scale, log2_table):
    res, size, off = [], [], []
    o = 0
    t = 1 << log2_table
    for l in range(n_levels):
        n = int(math.floor(base * math.pow(scale, l)))
        if n < 1:
            raise ValueError("hash grid level resolution must be >= 1")
        res.append(n)
        v = (n + 1) ** 3
        s = min(t, v)
        size.append(s)
        off.append(o)
        o += s
    return res, size, off


def parse(cfg) -> NetDesc:
    """Parse a config dict or JSON string; raise ValueError on anything unsupported."""
    if isinstance(cfg, (str, bytes)):
        cfg = json.loads(cfg)
    try:
        ve = cfg["vtx_enc"]
        ce = cfg.get("cmp_enc", {"otype": "Identity", "n_padded_dims": 16})
        op = cfg["out_prd"]
        cn = cfg["cmp_net"]
        we = cfg.get("wve_enc", {"face_size": 64})
    except KeyError as e:  # mirrors the reference's config.value(...) lookups
        raise ValueError(f"missing config key {e}") from None
    if ve.get("otype", "HashGrid") != "HashGrid":
        raise ValueError("vtx_enc.otype must be HashGrid")
    if ce.get("otype", "Identity") != "Identity":
        raise ValueError("cmp_enc.otype must be Identity")
    for name, net in (("out_prd", op), ("cmp_net", cn)):
        if net.get("activation", "ReLU") != "ReLU":
            raise ValueError(f"{name}.activation must be ReLU")
        if net.get("output_activation", "None") != "None":
            raise ValueError(f"{name}.output_activation must be None")
    d = NetDesc(
        n_levels=int(ve.get("n_levels", 16)),
        n_features=int(ve.get("n_features_per_level", 2)),
        log2_table=int(ve.get("log2_hashmap_size", 19)),
        base_resolution=int(ve.get("base_resolution", 16)),
        per_level_scale=float(ve.get("per_level_scale", 2.0)),
        aux_width=int(ce.get("n_padded_dims", 16)),
        op_neurons=int(op.get("n_neurons", 64)),
        op_hidden=int(op.get("n_hidden_layers", 2)),
        op_out=int(op.get("n_output_dims", 64)),
        cn_neurons=int(cn.get("n_neurons", 64)),
        cn_hidden=int(cn.get("n_hidden_layers", 2)),
        face_size=int(we.get("face_size", 64)),
    )
    if d.aux_width < N_AUX_INPUTS:
        raise ValueError("cmp_enc.n_padded_dims must be >= 13")
    if not (1 <= d.n_levels <= 32 and 1 <= d.n_features <= 8 and 1 <= d.log2_table <= 24):
        raise ValueError("hash grid dimensions out of range")
    if d.face_size < 1 or (d.face_size & (d.face_size - 1)):
        raise ValueError("wve_enc.face_size must be a power of two")
    d.level_res, d.level_size, d.level_offset = level_layout(
        d.n_levels, d.base_resolution, d.per_level_scale, d.log2_table)
    return d


def to_json(cfg: dict) -> str:
    return json.dumps(cfg, sort_keys=True)

"""CPU tests of the C-ABI boundary: the library loads, exports every declared symbol,
validates its inputs without a GPU, and the C++ shim compiles against it."""
import ctypes as C
import os
import re
import subprocess

import pytest

from neural_wavelet_prt_demo_b200 import _lib, netconfig

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "nwprt.h")).read()
    return sorted(set(re.findall(r"NWPRT_API\s+[\w\s\*]+?\b(nwprt_\w+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (nwprt_\w+)", out))
    assert set(declared_symbols()) <= exported
    assert all(s.startswith("nwprt_") for s in exported)   # nothing else leaks


def test_version_and_status_strings():
    L = _lib.lib()
    assert L.nwprt_abi_version() == 1
    for s in range(8):
        assert L.nwprt_status_string(s)


@pytest.mark.parametrize("text,status", [
    (b"{", _lib.INVALID_ARG),
    (b"[]", _lib.INVALID_ARG),
    (b'{"vtx_enc": {}}', _lib.INVALID_ARG),
    (b'{"vtx_enc": {"otype": "Frequency"}, "out_prd": {}, "cmp_net": {}}', _lib.UNSUPPORTED),
    (b'{"vtx_enc": {"n_levels": 99}, "out_prd": {}, "cmp_net": {}}', _lib.INVALID_ARG),
    (b'{"vtx_enc": {}, "out_prd": {"activation": "Tanh"}, "cmp_net": {}}', _lib.UNSUPPORTED),
    (b'{"vtx_enc": {}, "out_prd": {}, "cmp_net": {}, "wve_enc": {"face_size": 48}}', _lib.INVALID_ARG),
])
def test_create_rejects_bad_configs_with_a_message(text, status):
    ctx = C.c_void_p()
    s = _lib.lib().nwprt_create(text, 0, C.byref(ctx))
    assert s == status
    assert not ctx.value
    assert _lib.lib().nwprt_last_error(None)


def test_create_valid_config_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx = C.c_void_p()
    s = _lib.lib().nwprt_create(netconfig.to_json(netconfig.CONFIG_SMALL).encode(), 0, C.byref(ctx))
    assert s == _lib.CUDA_ERROR and not ctx.value


def test_null_arguments_are_rejected():
    L = _lib.lib()
    assert L.nwprt_create(None, 0, None) == _lib.INVALID_ARG
    assert L.nwprt_haar_topk(None, 1, 8, 4, None, None, None) == _lib.INVALID_ARG
    assert L.nwprt_sh_dot(None, 10, 81, None, 1, None, None) == _lib.INVALID_ARG
    assert L.nwprt_haar_topk(None, 1, 128, 4, None, None, None) == _lib.UNSUPPORTED
    assert L.nwprt_ready(None) == 0
    assert L.nwprt_sh_project_workspace_size(64) == 96 * 243 * 4


def test_cpp_shim_compiles_and_links(tmp_path):
    src = tmp_path / "shim.cpp"
    src.write_text(
        '#include "nwprt_engine.hpp"\n'
        "int main() {\n"
        "  nwprt::RenderEngine e(0);\n"
        "  nwprt::renderConfig cfg; cfg.precision = NWPRT_PREC_BF16;\n"
        "  try { e.createFromConfig(\"{\"); } catch (const std::runtime_error&) { return 0; }\n"
        "  return 1;\n"
        "}\n")
    exe = tmp_path / "shim"
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L", os.path.dirname(_lib.LIB_PATH), "-lnwprt",
                        "-Wl,-rpath," + os.path.dirname(_lib.LIB_PATH)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True)
    assert run.returncode == 0, run.stderr


def test_python_and_native_config_sizes_agree():
    # the native parser's derived sizes are reported through nwprt_get_network_info on the GPU
    # suite; here: the Python side's derived numbers used by tests and the bench
    d = netconfig.parse(netconfig.CONFIG_LARGE)
    assert d.flops_per_eval() == 53632
    assert d.enc_dims == 32 and d.n_coeffs == 24576 and d.cmp_in == 80
    s = netconfig.parse(netconfig.CONFIG_SMALL)
    assert s.cn_layers()[0] == (42, 64) and s.op_layers() == [(16, 26)]

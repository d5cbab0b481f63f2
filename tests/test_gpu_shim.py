"""The C++ drop-in shim (include/nwprt_engine.hpp) driven end to end on the GPU, the way the
reference's renderer calls its engine (Renderer/main.cpp:165-167, offlineRenderer.cpp:125-142):

    RenderEngine::initTCNN(model dir)            config_comp.json + the four weight .npy files
    Environment_Map(folder, name)                cube/<name>.hdr cross -> six faces
    RenderEngine::buildLights                    Haar + top-K on the GPU
    setFrameBuffers / TCNNPass_p1 / TCNNPass_p2 / TCNNSync on cudaMalloc'd G-buffers

A C++ program compiled against the header does all of it; its FP32 output must equal the
CPU oracle's for the same faces (read back from the .hdr), weights and G-buffer (the drop-in
is bit-exact against the FP32 oracle on this network), and its wavelet table must equal the
oracle's Haar + top-K."""
import os
import subprocess

import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import _lib, netconfig, synth
from neural_wavelet_prt_demo_b200.engine import EnvironmentMap, read_hdr
from oracle import oracle as O
from tests.helpers import bits_equal, write_hdr

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")

DRIVER = r'''
#include <cstdio>
#include <cuda_runtime.h>
#include "nwprt_engine.hpp"

static std::vector<char> slurp(const std::string& p) {
  FILE* f = std::fopen(p.c_str(), "rb");
  if (!f) throw std::runtime_error("cannot open " + p);
  std::fseek(f, 0, SEEK_END);
  const long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  std::vector<char> v(n);
  if (std::fread(v.data(), 1, n, f) != (size_t)n) throw std::runtime_error("short read " + p);
  std::fclose(f);
  return v;
}
static void* upload(const std::string& p) {
  std::vector<char> v = slurp(p);
  void* d = nullptr;
  if (cudaMalloc(&d, v.size()) != cudaSuccess) throw std::runtime_error("cudaMalloc");
  cudaMemcpy(d, v.data(), v.size(), cudaMemcpyHostToDevice);
  return d;
}

int main(int argc, char** argv) {
  // argv: model dir, env folder, env name, G-buffer dir, width, height, K, out dir
  try {
    const std::string gb = argv[4], out = argv[8];
    const int W = std::atoi(argv[5]), H = std::atoi(argv[6]), K = std::atoi(argv[7]);
    nwprt::RenderEngine engine(0);
    engine.initTCNN(argv[1]);
    std::vector<nwprt::Environment_Map> envs;
    envs.emplace_back(std::string(argv[2]), std::string(argv[3]));
    engine.buildLights(envs, K);
    if (!engine.TCNNAvaliable()) throw std::runtime_error("engine not available after buildLights");
    nwprt::FrameBuffers fb;
    fb.width = W;
    fb.height = H;
    fb.fbFirstHitPos = (const float*)upload(gb + "/pos.bin");
    fb.fbworldNormal = (const float*)upload(gb + "/normal.bin");
    fb.fbFirstHitReflecDir = (const float*)upload(gb + "/reflect.bin");
    fb.fbRoughness = (const float*)upload(gb + "/roughness.bin");
    fb.fbFirstHitKd = (const float*)upload(gb + "/kd.bin");
    fb.fbFirstHitKs = (const float*)upload(gb + "/ks.bin");
    fb.fbDirectDenoised = (const float*)upload(gb + "/direct.bin");
    fb.fbEnvironmentMapFlag = (const uint8_t*)upload(gb + "/flag.bin");
    const size_t n4 = (size_t)W * H * 4;
    cudaMalloc((void**)&fb.fbPredictedIndirect, n4 * sizeof(float));
    cudaMalloc((void**)&fb.fbPredictedIndirectWithDirect, n4 * sizeof(float));
    engine.setFrameBuffers(0, fb);
    nwprt::renderConfig cfg;  // FP32 drop-in, clamped Kahan sum: the reference's defaults
    engine.TCNNPass_p1(0);
    engine.TCNNPass_p2(0, 0, cfg);
    engine.TCNNSync();
    std::vector<float> ind(n4), wd(n4);
    cudaMemcpy(ind.data(), fb.fbPredictedIndirect, n4 * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(wd.data(), fb.fbPredictedIndirectWithDirect, n4 * sizeof(float), cudaMemcpyDeviceToHost);
    FILE* f = std::fopen((out + "/indirect.bin").c_str(), "wb");
    std::fwrite(ind.data(), sizeof(float), n4, f);
    std::fclose(f);
    f = std::fopen((out + "/with_direct.bin").c_str(), "wb");
    std::fwrite(wd.data(), sizeof(float), n4, f);
    std::fclose(f);
    f = std::fopen((out + "/idx.bin").c_str(), "wb");
    std::fwrite(envs[0].topWaveletCoefficients.data(), sizeof(int), envs[0].topWaveletCoefficients.size(), f);
    std::fclose(f);
    f = std::fopen((out + "/strength.bin").c_str(), "wb");
    std::fwrite(envs[0].topWaveletStrength.data(), sizeof(float), envs[0].topWaveletStrength.size(), f);
    std::fclose(f);
    // an unknown env id throws, as the reference's engine would on a bad index
    try {
      engine.TCNNPass_p2(5, 0, cfg);
      return 3;
    } catch (const std::runtime_error&) {
    }
    std::printf("ok\n");
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 2;
  }
}
'''


def test_cpp_engine_end_to_end(cuda, tmp_path):
    W, H, K = 64, 48, 64
    cfg = netconfig.CONFIG_SMALL
    desc = netconfig.parse(cfg)
    w = synth.make_weights(desc, seed=3, hash_scale=0.5)
    model = tmp_path / "model"
    model.mkdir()
    np.save(model / "vtx_enc.npy", w.hash_params)
    np.save(model / "out_prd.npy", w.out_prd)
    np.save(model / "cmp_net.npy", w.cmp_net)
    np.save(model / "wve_enc.npy", w.wve_enc)
    (model / "config_comp.json").write_text(netconfig.to_json(cfg))
    # env map: a seeded log-normal cubemap laid out as a 4x3 cross (top row first in the file)
    faces = synth.make_env_faces(desc.face_size, seed=4)
    S = desc.face_size
    cross = np.zeros((3 * S, 4 * S, 3), np.float32)
    for f, (cc, cr) in enumerate([(2, 1), (0, 1), (1, 2), (1, 0), (1, 1), (3, 1)]):
        for r in range(S):
            cross[3 * S - 1 - (cr * S + r), cc * S:(cc + 1) * S] = faces[f, r]
    env = tmp_path / "env"
    (env / "cube").mkdir(parents=True)
    write_hdr(env / "cube" / "studio.hdr", cross, rle=True)
    faces_file = EnvironmentMap.cross_to_faces(read_hdr(str(env / "cube" / "studio.hdr")))
    gb = synth.make_gbuffer(W, H, seed=5, flag_prob=0.8)
    gdir = tmp_path / "gb"
    gdir.mkdir()
    for name, a in zip(("pos", "normal", "reflect", "roughness", "kd", "ks", "direct", "flag"), gb.arrays()):
        np.ascontiguousarray(a).tofile(gdir / f"{name}.bin")
    src = tmp_path / "engine.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "engine"
    libdir = os.path.dirname(_lib.LIB_PATH)
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                        "-I", os.path.join(CUDA_HOME, "include"), str(src), "-o", str(exe),
                        "-L", libdir, "-lnwprt", "-Wl,-rpath," + libdir,
                        "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart",
                        "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe), str(model), str(env), "studio", str(gdir), str(W), str(H), str(K),
                          str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout + run.stderr
    idx = np.fromfile(tmp_path / "idx.bin", np.int32)
    st = np.fromfile(tmp_path / "strength.bin", np.float32).reshape(-1, 3)
    ridx, rst = O.haar_topk(faces_file, K)
    assert np.array_equal(idx, ridx)
    assert bits_equal(st, rst)
    ind = np.fromfile(tmp_path / "indirect.bin", np.float32).reshape(-1, 4)
    wd = np.fromfile(tmp_path / "with_direct.bin", np.float32).reshape(-1, 4)
    rind, rwd = O.relight_f32(O.Bound(desc, w, gb), ridx, rst)
    assert bits_equal(ind, rind)
    assert bits_equal(wd, rwd)

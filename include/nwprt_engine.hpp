// C++ drop-in shim over the nwprt C ABI with the reference's class shapes.
//
//   nwprt::RenderEngine   -- initTCNN / TCNNAvaliable / TCNNPass_p1 / TCNNPass_p2 / TCNNSync
//                            (Renderer/RenderEngine.h:78-83, tinycudann/tcnn.cu:49-162)
//   nwprt::Environment_Map -- faces / topWaveletCoefficients / topWaveletStrength /
//                            shCoefficients (Renderer/EnvironmentMap.h:11-40)
//   nwprt::renderConfig   -- renderConfig (Renderer/RenderEngine.h:29-42) + relight options
//
// Failures throw std::runtime_error, as the reference's CUDA_CHECK does
// (Renderer/optix7.h:27-38).  Header-only; link with -lnwprt.
#pragma once

#include <cstdint>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "nwprt.h"

namespace nwprt {

inline void check(nwprt_status s, const nwprt_ctx* ctx) {
  if (s != NWPRT_OK)
    throw std::runtime_error(std::string("nwprt: ") + nwprt_status_string(s) + ": " + nwprt_last_error(ctx));
}

struct renderConfig {
  int samplesPerPixel = 1024;
  bool waveletMode = true;
  bool finalDenoiser = false;    // denoising is outside this library
  bool indirectDenoiser = false;
  nwprt_precision precision = NWPRT_PREC_FP32;
  bool clampTerms = true;
  bool kahan = true;
  nwprt_relight_opts opts() const {
    nwprt_relight_opts o;
    o.precision = precision;
    o.clamp_terms = clampTerms ? 1 : 0;
    o.kahan = kahan ? 1 : 0;
    return o;
  }
};

// The fullFrameCUDA fields the relight reads and writes (Renderer/frames.h:143-183);
// caller-owned device memory, float4 per pixel unless noted.
struct FrameBuffers {
  int width = 0, height = 0;
  const float* fbFirstHitPos = nullptr;
  const float* fbworldNormal = nullptr;
  const float* fbFirstHitReflecDir = nullptr;
  const float* fbRoughness = nullptr;  // float per pixel
  const float* fbFirstHitKd = nullptr;
  const float* fbFirstHitKs = nullptr;
  const float* fbDirectDenoised = nullptr;
  const uint8_t* fbEnvironmentMapFlag = nullptr;  // bool per pixel
  float* fbPredictedIndirect = nullptr;
  float* fbPredictedIndirectWithDirect = nullptr;
};

class Environment_Map {
 public:
  Environment_Map() = default;
  // faces: [6][S][S][3] host floats in initCubeFaces order (EnvironmentMap.cpp:112-126)
  Environment_Map(std::vector<float> faces6, int faceSize) : faces(std::move(faces6)), face_size(faceSize) {}
  Environment_Map(std::vector<int> coefficients, std::vector<float> strength)
      : topWaveletCoefficients(std::move(coefficients)), topWaveletStrength(std::move(strength)) {}

  std::vector<float> faces;
  int face_size = 0;
  std::vector<int> topWaveletCoefficients;
  std::vector<float> topWaveletStrength;  // K x 3
  std::vector<float> shCoefficients;      // 81 x 3
};

class RenderEngine {
 public:
  explicit RenderEngine(int device = 0) : device_(device) {}
  ~RenderEngine() {
    if (ctx_) nwprt_destroy(ctx_);
  }
  RenderEngine(const RenderEngine&) = delete;
  RenderEngine& operator=(const RenderEngine&) = delete;

  // initTCNN(modelPath): reads config_comp.json and the four weight .npy files.
  void initTCNN(const std::string& modelPath) {
    std::ifstream f(modelPath + "/config_comp.json");
    if (!f) throw std::runtime_error("nwprt: cannot open " + modelPath + "/config_comp.json");
    std::stringstream ss;
    ss << f.rdbuf();
    createFromConfig(ss.str());
    check(nwprt_load_weights_dir(ctx_, modelPath.c_str()), ctx_);
    TCNNSetup = true;
  }
  void createFromConfig(const std::string& json) {
    if (ctx_) nwprt_destroy(ctx_);
    ctx_ = nullptr;
    check(nwprt_create(json.c_str(), device_, &ctx_), nullptr);
  }
  void loadWeights(const nwprt_weights& w) {
    check(nwprt_load_weights(ctx_, &w), ctx_);
    TCNNSetup = true;
  }
  bool TCNNAvaliable() const { return ctx_ && nwprt_ready(ctx_) != 0; }

  // buildLights: registers every env map; computes the wavelet table on the GPU when the
  // map carries faces and no precomputed table (K wavelets).
  void buildLights(std::vector<Environment_Map>& envs, int K = 64, void* stream = nullptr) {
    for (auto& e : envs) {
      int id = -1;
      if (e.topWaveletCoefficients.empty()) {
        check(nwprt_env_from_faces(ctx_, e.faces.data(), 0, e.face_size, K, stream, &id), ctx_);
        int k = 0;
        check(nwprt_env_get_wavelets(ctx_, id, nullptr, nullptr, 0, &k), ctx_);
        e.topWaveletCoefficients.resize(k);
        e.topWaveletStrength.resize((size_t)k * 3);
        check(nwprt_env_get_wavelets(ctx_, id, e.topWaveletCoefficients.data(), e.topWaveletStrength.data(), k, &k),
              ctx_);
      } else {
        check(nwprt_env_from_wavelets(ctx_, e.topWaveletCoefficients.data(), e.topWaveletStrength.data(),
                                      (int)e.topWaveletCoefficients.size(), 0, stream, &id),
              ctx_);
      }
      envIds_.push_back(id);
    }
    EnvmapSetup = !envIds_.empty();
  }

  void setFrameBuffers(int frameID, const FrameBuffers& fb) {
    if (frameID < 0 || frameID >= NWPRT_MAX_FRAMES) throw std::runtime_error("nwprt: frame id out of range");
    if ((int)frames_.size() <= frameID) frames_.resize(frameID + 1);
    frames_[frameID] = fb;
  }

  void TCNNPass_p1(int frameID, void* stream = nullptr) {
    const FrameBuffers& f = frame(frameID);
    nwprt_gbuffer g;
    g.width = f.width;
    g.height = f.height;
    g.first_hit_pos = f.fbFirstHitPos;
    g.world_normal = f.fbworldNormal;
    g.reflect_dir = f.fbFirstHitReflecDir;
    g.roughness = f.fbRoughness;
    g.kd = f.fbFirstHitKd;
    g.ks = f.fbFirstHitKs;
    g.direct = f.fbDirectDenoised;
    g.env_map_flag = f.fbEnvironmentMapFlag;
    check(nwprt_prepare(ctx_, frameID, &g, stream), ctx_);
  }

  void TCNNPass_p2(int envMapID, int frameID, renderConfig config, void* stream = nullptr) {
    if (envMapID < 0 || envMapID >= (int)envIds_.size()) throw std::runtime_error("nwprt: unknown envMapID");
    const FrameBuffers& f = frame(frameID);
    const nwprt_relight_opts o = config.opts();
    check(nwprt_relight(ctx_, envIds_[envMapID], frameID, &o, f.fbPredictedIndirect,
                        f.fbPredictedIndirectWithDirect, stream),
          ctx_);
  }

  void TCNNSync() { check(nwprt_sync(ctx_), ctx_); }

  nwprt_ctx* context() const { return ctx_; }
  bool TCNNSetup = false;
  bool EnvmapSetup = false;

 private:
  const FrameBuffers& frame(int frameID) const {
    if (frameID < 0 || frameID >= (int)frames_.size()) throw std::runtime_error("nwprt: frame has no buffers");
    return frames_[frameID];
  }
  int device_;
  nwprt_ctx* ctx_ = nullptr;
  std::vector<int> envIds_;
  std::vector<FrameBuffers> frames_;
};

}  // namespace nwprt

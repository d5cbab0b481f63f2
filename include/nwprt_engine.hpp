// C++ drop-in shim over the nwprt C ABI with the reference's class shapes.
//
//   nwprt::RenderEngine   -- initTCNN / TCNNAvaliable / TCNNPass_p1 / TCNNPass_p2 / TCNNSync
//                            (Renderer/RenderEngine.h:78-83, tinycudann/tcnn.cu:49-162)
//   nwprt::Environment_Map -- faces / topWaveletCoefficients / topWaveletStrength /
//                            shCoefficients, file and folder constructors
//                            (Renderer/EnvironmentMap.h:11-40, EnvironmentMap.cpp:10-126)
//   nwprt::renderConfig   -- renderConfig (Renderer/RenderEngine.h:29-42) + relight options
//
// Failures throw std::runtime_error, as the reference's CUDA_CHECK does
// (Renderer/optix7.h:27-38).  Header-only; link with -lnwprt.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "nwprt.h"

namespace nwprt {

// ---------------------------------------------------------------- file readers
// The reference reads env maps and precomputed tables from .npy files (Renderer/npy.h) and
// cross-layout cubemaps from Radiance .hdr files (Renderer/HDRloader.cpp).  These readers
// cover what Environment_Map needs from both formats; malformed files throw.
namespace io {

struct NpyArray {
  std::string descr;          // numpy type string, e.g. "<f4"
  std::vector<size_t> shape;
  std::vector<char> bytes;    // C-order element data
  size_t count() const {
    size_t n = 1;
    for (size_t d : shape) n *= d;
    return n;
  }
};

inline std::string npy_header_value(const std::string& header, const std::string& key) {
  const size_t k = header.find("'" + key + "'");
  if (k == std::string::npos) throw std::runtime_error("nwprt: .npy header lacks " + key);
  size_t v = header.find(':', k);
  if (v == std::string::npos) throw std::runtime_error("nwprt: bad .npy header");
  ++v;
  while (v < header.size() && header[v] == ' ') ++v;
  return header.substr(v);
}

// .npy versions 1-3, little-endian numeric types, C order.
inline NpyArray read_npy(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("nwprt: cannot open " + path);
  char magic[6];
  unsigned char ver[2];
  f.read(magic, 6);
  f.read(reinterpret_cast<char*>(ver), 2);
  if (!f || std::memcmp(magic, "\x93NUMPY", 6) != 0) throw std::runtime_error("nwprt: not a .npy file: " + path);
  uint32_t hlen = 0;
  unsigned char b[4] = {0, 0, 0, 0};
  if (ver[0] == 1) {
    f.read(reinterpret_cast<char*>(b), 2);
    hlen = b[0] | (b[1] << 8);
  } else if (ver[0] == 2 || ver[0] == 3) {
    f.read(reinterpret_cast<char*>(b), 4);
    hlen = b[0] | (b[1] << 8) | (b[2] << 16) | ((uint32_t)b[3] << 24);
  } else {
    throw std::runtime_error("nwprt: unsupported .npy version in " + path);
  }
  std::string header(hlen, '\0');
  f.read(&header[0], hlen);
  if (!f) throw std::runtime_error("nwprt: truncated .npy header in " + path);
  NpyArray a;
  const std::string d = npy_header_value(header, "descr");
  const size_t q0 = d.find('\''), q1 = d.find('\'', q0 + 1);
  if (q0 != 0 || q1 == std::string::npos) throw std::runtime_error("nwprt: bad .npy descr in " + path);
  a.descr = d.substr(1, q1 - 1);
  if (npy_header_value(header, "fortran_order").compare(0, 4, "True") == 0)
    throw std::runtime_error("nwprt: Fortran-order .npy files are not supported: " + path);
  const std::string sh = npy_header_value(header, "shape");
  const size_t p0 = sh.find('('), p1 = sh.find(')');
  if (p0 != 0 || p1 == std::string::npos) throw std::runtime_error("nwprt: bad .npy shape in " + path);
  std::stringstream dims(sh.substr(1, p1 - 1));
  std::string tok;
  while (std::getline(dims, tok, ','))
    if (tok.find_first_not_of(' ') != std::string::npos) a.shape.push_back(std::stoull(tok));
  if (a.descr.size() < 3 || (a.descr[0] != '<' && a.descr[0] != '|'))
    throw std::runtime_error("nwprt: only little-endian .npy data is supported: " + path);
  const size_t elem = std::stoul(a.descr.substr(2));
  a.bytes.resize(a.count() * elem);
  f.read(a.bytes.data(), (std::streamsize)a.bytes.size());
  if ((size_t)f.gcount() != a.bytes.size()) throw std::runtime_error("nwprt: truncated .npy data in " + path);
  return a;
}

inline std::vector<float> npy_as_float32(const NpyArray& a, const std::string& path) {
  if (a.descr != "<f4") throw std::runtime_error("nwprt: " + path + " must hold float32 data");
  std::vector<float> v(a.count());
  std::memcpy(v.data(), a.bytes.data(), a.bytes.size());
  return v;
}

// int32 indices; int64 files (numpy's default integer) are accepted when every value fits.
inline std::vector<int> npy_as_int32(const NpyArray& a, const std::string& path) {
  std::vector<int> v(a.count());
  if (a.descr == "<i4") {
    std::memcpy(v.data(), a.bytes.data(), a.bytes.size());
  } else if (a.descr == "<i8") {
    for (size_t i = 0; i < v.size(); ++i) {
      int64_t x;
      std::memcpy(&x, a.bytes.data() + 8 * i, 8);
      if (x < INT32_MIN || x > INT32_MAX) throw std::runtime_error("nwprt: index out of int32 range in " + path);
      v[i] = (int)x;
    }
  } else {
    throw std::runtime_error("nwprt: " + path + " must hold int32 or int64 indices");
  }
  return v;
}

// Radiance RGBE image: "#?RADIANCE" signature, header lines up to an empty line, a
// "-Y <h> +X <w>" resolution line, then h scanlines of w pixels.  A scanline is either
// run-length encoded per component (a 2, 2, w / 256, w % 256 marker, then four components
// of runs (count > 128: count - 128 copies of one byte) and dumps (count literal bytes)),
// or flat RGBE quadruples in which (1, 1, 1, n) repeats the previous pixel n << shift times.
// A channel is mantissa / 256 * 2^(E - 128), as the reference converts it
// (Renderer/HDRloader.cpp:108-125).  Returns [h][w][3] floats, rows in file order (top first).
inline std::vector<float> read_hdr(const std::string& path, int* width, int* height) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("nwprt: cannot open " + path);
  std::string line;
  std::getline(f, line);
  if (line.compare(0, 10, "#?RADIANCE") != 0) throw std::runtime_error("nwprt: not a Radiance .hdr file: " + path);
  while (std::getline(f, line) && !line.empty()) {
  }
  int w = 0, h = 0;
  if (!std::getline(f, line) || std::sscanf(line.c_str(), "-Y %d +X %d", &h, &w) != 2 || w <= 0 || h <= 0)
    throw std::runtime_error("nwprt: unsupported .hdr resolution line in " + path);
  std::vector<unsigned char> scan((size_t)w * 4);
  std::vector<float> img((size_t)w * h * 3);
  auto byte = [&]() -> unsigned char {
    const int c = f.get();
    if (c == EOF) throw std::runtime_error("nwprt: truncated .hdr data in " + path);
    return (unsigned char)c;
  };
  for (int y = 0; y < h; ++y) {
    unsigned char q[4];
    for (int c = 0; c < 4; ++c) q[c] = byte();
    if (w >= 8 && w <= 0x7fff && q[0] == 2 && q[1] == 2 && !(q[2] & 0x80)) {
      if (((int)q[2] << 8 | q[3]) != w) throw std::runtime_error("nwprt: .hdr scanline width mismatch in " + path);
      for (int c = 0; c < 4; ++c)
        for (int x = 0; x < w;) {
          int n = byte();
          if (n > 128) {
            n -= 128;
            const unsigned char v = byte();
            if (x + n > w) throw std::runtime_error("nwprt: .hdr run overflows its scanline in " + path);
            while (n--) scan[(size_t)4 * x++ + c] = v;
          } else {
            if (n == 0 || x + n > w) throw std::runtime_error("nwprt: bad .hdr dump in " + path);
            while (n--) scan[(size_t)4 * x++ + c] = byte();
          }
        }
    } else {
      int x = 0, shift = 0;
      for (bool first = true; x < w; first = false) {
        if (!first)
          for (int c = 0; c < 4; ++c) q[c] = byte();
        if (q[0] == 1 && q[1] == 1 && q[2] == 1) {
          if (x == 0) throw std::runtime_error("nwprt: .hdr repeat code without a pixel in " + path);
          const long long n = (long long)q[3] << shift;
          if (x + n > w) throw std::runtime_error("nwprt: .hdr repeat overflows its scanline in " + path);
          for (long long i = 0; i < n; ++i, ++x) std::memcpy(&scan[(size_t)4 * x], &scan[(size_t)4 * (x - 1)], 4);
          shift += 8;
        } else {
          std::memcpy(&scan[(size_t)4 * x++], q, 4);
          shift = 0;
        }
      }
    }
    for (int x = 0; x < w; ++x) {
      const float scale = (float)std::ldexp(1.0, (int)scan[(size_t)4 * x + 3] - 128);
      for (int c = 0; c < 3; ++c)
        img[((size_t)y * w + x) * 3 + c] = ((float)scan[(size_t)4 * x + c] / 256.0f) * scale;
    }
  }
  *width = w;
  *height = h;
  return img;
}

inline bool path_is_dir(const std::string& p) {
  struct stat st;
  return ::stat(p.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}
inline bool path_exists(const std::string& p) {
  struct stat st;
  return ::stat(p.c_str(), &st) == 0;
}

}  // namespace io

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

  // Environment_Map(inFileName, sh_coeff) (EnvironmentMap.cpp:10-18): a 4x3 cross cubemap
  // (.hdr or .npy) or, with sh_coeff, the env's SH coefficients (.npy [n][3]).
  explicit Environment_Map(const std::string& inFileName, bool sh_coeff = false) {
    if (sh_coeff)
      load_sh(inFileName);
    else
      loadCubeMap(inFileName);
  }

  // Environment_Map(envMapFolder, envMapName) (EnvironmentMap.cpp:20-68): cube/<name>.hdr
  // (required), then sh/<name>.npy and the waveletcoeffs/<name>.npy + waveletstrength/<name>.npy
  // pair when present.  The latlong map is read by the reference for its direct-light shader
  // only and is not part of the relight.
  Environment_Map(const std::string& envMapFolder, const std::string& envMapName) { load_folder(envMapFolder, envMapName); }
  Environment_Map(const char* envMapFolder, const char* envMapName) {
    load_folder(envMapFolder, envMapName);
  }

  // 4x3 cross [3S][4S][3] (rows in file order, top first) -> faces [6][S][S][3].  Rows are
  // flipped first: the reference stores both .npy (EnvironmentMap.cpp:96-101) and .hdr
  // (HDRLoaderResult::get, Renderer/HDRloader.h:21-25) crosses bottom row first.  The faces
  // are then the cells at (column, row) = (2,1), (0,1), (1,2), (1,0), (1,1), (3,1) of the
  // flipped image, in face units (+X, -X, +Y, -Y, -Z, +Z; EnvironmentMap.cpp:112-126).
  static std::vector<float> cross_to_faces(const std::vector<float>& cross, int width, int height, int* S) {
    const int s = height / 3;
    if (s <= 0 || height != 3 * s || width != 4 * s || cross.size() != (size_t)width * height * 3)
      throw std::runtime_error("nwprt: a cubemap cross must be 3S rows x 4S columns of RGB");
    static const int cells[6][2] = {{2, 1}, {0, 1}, {1, 2}, {1, 0}, {1, 1}, {3, 1}};
    std::vector<float> out((size_t)6 * s * s * 3);
    for (int f = 0; f < 6; ++f)
      for (int r = 0; r < s; ++r) {
        const int src_row = height - 1 - (cells[f][1] * s + r);  // row of the flipped image
        const float* src = &cross[((size_t)src_row * width + (size_t)cells[f][0] * s) * 3];
        std::memcpy(&out[((size_t)f * s + r) * s * 3], src, sizeof(float) * s * 3);
      }
    *S = s;
    return out;
  }

  std::vector<float> faces;
  int face_size = 0;
  std::vector<int> topWaveletCoefficients;
  std::vector<float> topWaveletStrength;  // K x 3
  std::vector<float> shCoefficients;      // 81 x 3

 private:
  void loadCubeMap(const std::string& path) {
    if (!io::path_exists(path)) throw std::runtime_error("Invalid Env map File Name");
    std::vector<float> img;
    int w = 0, h = 0;
    const std::string ext = path.size() >= 4 ? path.substr(path.size() - 4) : std::string();
    if (ext == ".hdr") {
      img = io::read_hdr(path, &w, &h);
    } else if (ext == ".npy") {
      const io::NpyArray a = io::read_npy(path);
      if (a.shape.size() != 3 || a.shape[2] != 3) throw std::runtime_error("nwprt: cube .npy must be [H][W][3]: " + path);
      img = io::npy_as_float32(a, path);
      h = (int)a.shape[0];
      w = (int)a.shape[1];
    } else {
      throw std::runtime_error("Unknown type " + ext);
    }
    faces = cross_to_faces(img, w, h, &face_size);
  }
  void load_sh(const std::string& path) {
    const io::NpyArray a = io::read_npy(path);
    if (a.shape.size() != 2 || a.shape[1] != 3) throw std::runtime_error("nwprt: SH .npy must be [n][3]: " + path);
    const int l = (int)std::lround(std::sqrt((double)a.shape[0])) - 1;
    if ((size_t)(l + 1) * (l + 1) != a.shape[0]) throw std::runtime_error("nwprt: SH .npy must hold (l+1)^2 rows: " + path);
    shCoefficients = io::npy_as_float32(a, path);
  }
  void load_folder(const std::string& folder, const std::string& name) {
    if (!io::path_is_dir(folder)) throw std::runtime_error("Invalid Env map Folder Name, it should not be a file");
    loadCubeMap(folder + "/cube/" + name + ".hdr");
    const std::string sh = folder + "/sh/" + name + ".npy";
    if (io::path_exists(sh)) load_sh(sh);
    const std::string wc = folder + "/waveletcoeffs/" + name + ".npy";
    const std::string ws = folder + "/waveletstrength/" + name + ".npy";
    if (io::path_exists(wc) && io::path_exists(ws)) {
      topWaveletCoefficients = io::npy_as_int32(io::read_npy(wc), wc);
      const io::NpyArray st = io::read_npy(ws);
      if (st.shape.size() != 2 || st.shape[1] != 3) throw std::runtime_error("nwprt: waveletstrength must be [K][3]: " + ws);
      topWaveletStrength = io::npy_as_float32(st, ws);
      if (topWaveletStrength.size() != topWaveletCoefficients.size() * 3)
        throw std::runtime_error("nwprt: waveletcoeffs and waveletstrength disagree on K for " + name);
    }
  }
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

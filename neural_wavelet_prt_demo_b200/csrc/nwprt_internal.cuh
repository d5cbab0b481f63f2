// Internal declarations shared by the libnwprt translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nwprt.h"

namespace nwprt {

// ------------------------------------------------------------------ errors
struct Error : std::runtime_error {
  nwprt_status status;
  Error(nwprt_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] inline void fail(nwprt_status s, const std::string& m) { throw Error(s, m); }

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    if (e == cudaErrorMemoryAllocation)
      fail(NWPRT_OOM, std::string(what) + ": " + cudaGetErrorString(e));
    fail(NWPRT_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
  }
}
#define NWPRT_CUDA(call) ::nwprt::cuda_check((call), #call)

// Device-side error codes (written to a device error word, read by the host).
enum DevError : uint32_t {
  kDevOk = 0,
  kDevWaitTimeout = 1,  // a bounded mbarrier wait ran out
  kDevBadIndex = 2,     // a gather index outside its table (input validation)
};

// ------------------------------------------------------------------ network
constexpr int kMaxLevels = 32;
constexpr int kMaxLayers = 8;

struct NetDims {
  int n_levels = 0, n_features = 0, log2_table = 0, base_resolution = 0;
  double per_level_scale = 0;
  int level_res[kMaxLevels] = {0};
  int level_size[kMaxLevels] = {0};
  int level_offset[kMaxLevels] = {0};
  int aux_width = 16;
  int op_neurons = 64, op_hidden = 0, op_out = 64;
  int cn_neurons = 64, cn_hidden = 0;
  int face_size = 64;
  int op_nl = 0, op_in[kMaxLayers] = {0}, op_outs[kMaxLayers] = {0};
  int cn_nl = 0, cn_in[kMaxLayers] = {0}, cn_outs[kMaxLayers] = {0};

  int enc_dims() const { return n_levels * n_features; }
  int n_coeffs() const { return 6 * face_size * face_size; }
  size_t n_hash_params() const {
    size_t s = 0;
    for (int l = 0; l < n_levels; ++l) s += (size_t)level_size[l];
    return s * (size_t)n_features;
  }
  size_t n_op_params() const {
    size_t s = 0;
    for (int i = 0; i < op_nl; ++i) s += (size_t)op_in[i] * op_outs[i];
    return s;
  }
  size_t n_cn_params() const {
    size_t s = 0;
    for (int i = 0; i < cn_nl; ++i) s += (size_t)cn_in[i] * cn_outs[i];
    return s;
  }
  double flops_per_eval() const;
};

NetDims parse_config(const std::string& json_text);

// Sets the calling thread's nwprt_last_error(NULL) message (api.cu).
void set_thread_error(const std::string& m);

// Hash-grid level table passed by value to kernels.
struct HashLevels {
  int n_levels, n_features;
  int res[kMaxLevels];
  uint32_t size[kMaxLevels];
  uint32_t offset[kMaxLevels];
  uint32_t dense_mask;  // bit l set: level l indexes its table densely
};

// ------------------------------------------------------------------ npy / json helpers
struct NpyArray {
  std::vector<size_t> shape;
  std::string descr;
  std::vector<char> data;
};
NpyArray read_npy(const std::string& path);

// ------------------------------------------------------------------ kernels (launchers)
// haar_topk.cu
void launch_haar_topk(const float* faces, int n_env, int S, int K, int32_t* idx, float* strength,
                      uint32_t* err, cudaStream_t st);
size_t haar_topk_smem_bytes(int S, int K);

// sh.cu
size_t sh_project_workspace_bytes(int S);
void launch_sh_project(const float* faces, int S, float* L, float* workspace, cudaStream_t st);
void launch_sh_dot(const float* T, int64_t n_px, int nc, const float* L, int abs_out, float* out,
                   uint32_t* err, cudaStream_t st);

// env_rotate.cu
void launch_env_rotate(const float* src, int S, const float* R_host, float* dst, cudaStream_t st);

// relight_common.cu
void launch_pack_gbuffer(const nwprt_gbuffer& g, float* packed, cudaStream_t st);
// out_kd: [K][D] FP32 rows; out_h (may be null): the same rows as BF16 pairs, [K][D/2]
// 32-bit words with feature 2i in the low half (D even).
void launch_gather_embedding(const float* emb, int D, int n_coeffs, const int32_t* idx, int K,
                             float* out_kd, uint32_t* out_h, uint32_t* err, cudaStream_t st);

// One relight job: a prepared frame and an env wavelet table.
struct RelightJob {
  const float* packed;    // [n_px][16]
  const uint8_t* flag;    // [n_px]
  const float* direct;    // float4 [n_px]
  const float* emb_k;     // [K][D] embedding gathered at the env's indices (FP32)
  const float* strength;  // [K][3]
  int K;
  int64_t n_px;      // end of the pixel range (exclusive)
  float* indirect;
  float* with_direct;
  int64_t px_begin;  // start of the pixel range
};

struct DeviceWeights {
  const float* hash;       // [sum T_l][F]
  const float* op_t;       // out_prd layers transposed [in][out_pad4], FP32
  const float* cn_t;       // cmp_net layers transposed
  size_t op_t_floats, cn_t_floats;
};

// relight_fp32.cu
void launch_relight_fp32(const NetDims& d, const HashLevels& hl, const DeviceWeights& w,
                         const RelightJob& job, int clamp, int kahan, cudaStream_t st);
// Host-side packing of FP32 weights into the kernel's transposed layout.
void pack_fp32_weights(const NetDims& d, const float* op, const float* cn,
                       std::vector<float>* op_t, std::vector<float>* cn_t);

// tonemap.cu
void launch_tonemap_srgb(const float* src, int64_t n, uint32_t* dst, cudaStream_t st);

// sh_vertex.cu
void launch_sh_vertex(const float* T, const float* brdf, const float* L, int64_t V, int n, float* out,
                      cudaStream_t st);
void launch_sh_interpolate(const float* vc, int64_t V, const int32_t* tri, const float* uv, int64_t P, float* out,
                           uint32_t* err, cudaStream_t st);

// relight_tc.cu (tcgen05 path: BF16 operands, or FP8 e4m3 with per-layer scales)
constexpr int kMaxTcLayers = 12;
// One tensor-core layer of the per-wavelet MLP chain (B operand offsets inside the weight blob).
struct TcLayer {
  uint32_t b_off;  // byte offset of B (N x K, canonical K-major) in the weight blob
  uint32_t b_sbo;  // B stride between 8-row groups (= K * element bytes * 8)
  int k;           // reduction length (multiple of 16 for BF16, of 32 for FP8)
  int n;           // output width: 32 or 64
  int relu;
  int aux;         // also accumulate aux (K=16, BF16) x aux block of B at aux_off
  uint32_t aux_off;
  int fin;         // the epilogue forms T_k = V_last relu(h) from this layer's output
  float scale;     // FP8: factor applied to the accumulator before the e4m3 conversion (1 = none)
};
struct TcPlan {
  TcLayer layers[kMaxTcLayers];
  int n_layers = 0;
  uint32_t blob_bytes = 0;
  float cp_scale = 1.f;     // FP8: scale of the first layer's operand hash(p) * E_k
  float vlast[3][64] = {};  // V_last, FP32 [c][j] (filled when the weights are given)
  // BF16 plans: V_last as FP16 B tile of the output layer on the tensor core (N=16: channel c
  // in row c, K = the last hidden width padded to 16), at out_b_off with 8-row stride out_sbo
  uint32_t out_b_off = 0, out_sbo = 0;
  int out_k = 0;
};
enum TcMode { kTcBf16 = 0, kTcCalibrate = 1, kTcFp8 = 2 };
bool relight_tc_supported(const NetDims& d, std::string* why);
// A bounded device wait that is made to run out (diagnostics of the timeout path).
void launch_wait_selftest(int timeout_ms, uint32_t* err, cudaStream_t st);
bool relight_tc_fp8_supported(const NetDims& d, std::string* why);
size_t tc_weight_bytes(const NetDims& d);
// Device allocation for a tensor-core weight blob of `bytes`: whole 256-byte rows, the
// 2-D view through which the relight kernel loads it with TMA (the padding is zero).
inline size_t tc_blob_alloc_bytes(size_t bytes) { return (bytes + 255) & ~size_t(255); }
// BF16 weight blob; returns its plan (with V_last), which every BF16 launch needs.
TcPlan pack_tc_weights(const NetDims& d, const float* op, const float* cn, std::vector<uint16_t>* out);
// FP8 weight blob from calibrated activation maxima amax[0..n_layers) (the input of every
// tensor-core layer); returns the plan whose scales the kernel applies.
TcPlan pack_tc_weights_fp8(const NetDims& d, const float* op, const float* cn, const float* amax,
                           std::vector<uint8_t>* out);
int tc_layer_count(const NetDims& d);
size_t relight_tc_smem_bytes(const NetDims& d);
struct TcJob {
  const float* packed;    // [n_px][16]
  const uint8_t* flag;
  const float* direct;
  const float* emb_k;     // [K][D] FP32 embedding rows of the env's wavelets
  const float* strength;  // [K][3]
  int K;
  int64_t n_px;           // end of the pixel range (exclusive)
  float* indirect;
  float* with_direct;
  long long tile_begin;   // first 128-pixel tile of this job in the launch (set by the launcher)
  int64_t px_begin;       // start of the pixel range
  const uint32_t* emb_h;  // [K][D/2] the same rows as BF16 pairs (the BF16 form's operand)
};
// mode kTcBf16 / kTcCalibrate use the BF16 blob and its plan (from pack_tc_weights);
// kTcCalibrate also records per-layer activation maxima into amax (uint bits of floats);
// kTcFp8 uses the FP8 blob and its plan.  tile_ctr: one device int, reset on `st` before
// each kernel launch; the kernel's warpgroups take 128-pixel tiles from it, so no other
// launch may use it while this one runs.
void launch_relight_tc(const NetDims& d, const HashLevels& hl, const float* hash, const void* blob_dev,
                       const TcPlan* plan, int mode, const TcJob* jobs, int n_jobs, int kahan, int clamp,
                       uint32_t* amax, uint32_t* err, int* tile_ctr, cudaStream_t st);

}  // namespace nwprt

// ------------------------------------------------------------------ device helpers
#ifdef __CUDACC__
namespace nwprt {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Bounded mbarrier wait.  Returns false (and records kDevWaitTimeout) when the
// phase did not complete within `limit` polls; callers then abandon their work.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t* err,
                                          uint32_t limit = (1u << 26)) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  if (err) atomicCAS(err, 0u, (uint32_t)kDevWaitTimeout);
  return false;
}

// ln(x) of a float by the atanh series ln m = 2 (s + s^3/3 + s^5/5 + ...), s = (m-1)/(m+1)
// (Abramowitz & Stegun 4.1.27), after x = 2^e m with m in [sqrt(1/2), sqrt(2)]; evaluated
// with IEEE double +, -, *, / and fma in a fixed order and rounded once to float, so host,
// device and the CPU oracle return the same bits (the correctly rounded logarithm except
// in rare ties).  Used for the roughness remap log(25r+1)/log(26) (utils_kernels.h:21,39).
__host__ __device__ inline float float_from_bits(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}

// ln(x) in double for a positive finite float x, by the series above; the exponent part
// is returned separately so that logf_series rounds exactly as before.
__host__ __device__ inline double log_series_mantissa(float xf, int* exponent) {
  const double x = (double)xf;
  unsigned long long b;
  memcpy(&b, &x, 8);
  int e = (int)((b >> 52) & 0x7ff) - 1023;
  b = (b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
  double m;
  memcpy(&m, &b, 8);
  if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
  const double s = (m - 1.0) / (m + 1.0);
  const double z = s * s;
  double p = 1.0 / 23.0;
  p = fma(p, z, 1.0 / 21.0);
  p = fma(p, z, 1.0 / 19.0);
  p = fma(p, z, 1.0 / 17.0);
  p = fma(p, z, 1.0 / 15.0);
  p = fma(p, z, 1.0 / 13.0);
  p = fma(p, z, 1.0 / 11.0);
  p = fma(p, z, 1.0 / 9.0);
  p = fma(p, z, 1.0 / 7.0);
  p = fma(p, z, 1.0 / 5.0);
  p = fma(p, z, 1.0 / 3.0);
  p = fma(p, z, 1.0);
  *exponent = e;
  return (2.0 * s) * p;
}

__host__ __device__ inline float logf_series(float xf) {
  if (xf != xf) return xf;
  if (xf < 0.0f) return float_from_bits(0x7fc00000u);
  if (xf == 0.0f) return float_from_bits(0xff800000u);
  if (xf > 3.4028234663852886e38f) return xf;
  int e;
  const double lm = log_series_mantissa(xf, &e);
  return (float)fma((double)e, 0.6931471805599453, lm);
}

// x^y of a float by exp(y ln x) in IEEE double, rounded once to float: ln from the series
// above, exp by reduction t = k ln2 + r (|r| <= ln2/2) and the Taylor series of e^r to r^18
// (truncation error < 1e-22).  Every step is an explicit fma or a single IEEE operation, so
// host, device and the CPU oracle return the same bits.  Negative x gives NaN, 0 gives 0
// (y > 0), +inf gives +inf -- as powf for y in (0, 1).
__host__ __device__ inline float powf_series(float xf, float yf) {
  if (xf != xf || xf < 0.0f) return float_from_bits(0x7fc00000u);
  if (xf == 0.0f) return 0.0f;
  if (xf > 3.4028234663852886e38f) return xf;
  int e;
  const double lm = log_series_mantissa(xf, &e);
  const double t = fma((double)e, 0.6931471805599453, lm) * (double)yf;
  const double kd = floor(fma(t, 1.4426950408889634, 0.5));
  const double r = fma(-kd, 0.6931471805599453, t);
  double p = 1.0 / 6402373705728000.0;  // 1/18!
  p = fma(p, r, 1.0 / 355687428096000.0);
  p = fma(p, r, 1.0 / 20922789888000.0);
  p = fma(p, r, 1.0 / 1307674368000.0);
  p = fma(p, r, 1.0 / 87178291200.0);
  p = fma(p, r, 1.0 / 6227020800.0);
  p = fma(p, r, 1.0 / 479001600.0);
  p = fma(p, r, 1.0 / 39916800.0);
  p = fma(p, r, 1.0 / 3628800.0);
  p = fma(p, r, 1.0 / 362880.0);
  p = fma(p, r, 1.0 / 40320.0);
  p = fma(p, r, 1.0 / 5040.0);
  p = fma(p, r, 1.0 / 720.0);
  p = fma(p, r, 1.0 / 120.0);
  p = fma(p, r, 1.0 / 24.0);
  p = fma(p, r, 1.0 / 6.0);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  return (float)ldexp(p, (int)kd);
}

// sRGB-style encode of one linear channel to a byte, as the reference's final-colour pass
// does it (Renderer/toneMap.cu:47-71): 1.055 (x + 1e-6)^(1/2.4) - 0.055, clamped to
// [0, 1] (NaN -> 0), times 255.9, truncated.
__host__ __device__ inline uint32_t srgb_byte(float x) {
  const float coeff = 1.055f;
  const float p = powf_series(x + 1e-6f, 1.0f / 2.4f);
  float f = fmaf(coeff, p, -(coeff - 1.0f));
  f = f > 0.0f ? f : 0.0f;  // NaN -> 0, like fmaxf(0, NaN)
  f = f < 1.0f ? f : 1.0f;
  return (uint32_t)(f * 255.9f);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 1-D bulk copy global -> this CTA's shared memory, completion on `bar` (no multicast).
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace nwprt
#endif

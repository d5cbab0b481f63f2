// Final-colour pass: linear float4 radiance -> packed RGBA8, the reference's
// computeFinalPixelColorsKernel (Renderer/toneMap.cu:47-71) applied to the relight output
// (indirect + direct, or indirect alone, Renderer/toneMap.cu:79-84).
//
// The per-channel encode srgb_byte(x) = floor(255.9 clamp(1.055 (x + 1e-6)^(1/2.4) - 0.055))
// is a non-decreasing step function of x with 255 steps.  The host finds each step's
// threshold once -- the smallest float whose byte reaches j, by bisection over the ordered
// bit patterns of non-negative floats, evaluating srgb_byte itself -- and the kernel maps a
// channel to the number of thresholds at or below it (an estimate, then one or two exact
// comparisons in shared memory).
// That equals srgb_byte wherever srgb_byte is monotonic, which the oracle checks float by
// float around every threshold.  One float4 read and one 32-bit write per pixel: HBM-bound.
#include <mutex>

#include "nwprt_internal.cuh"

namespace nwprt {
namespace {

struct SrgbTable {
  float t[256];  // t[j]: smallest float with byte >= j (j >= 1); t[0] unused
};

SrgbTable build_table() {
  SrgbTable T{};
  T.t[0] = 0.f;
  for (int j = 1; j < 256; ++j) {
    uint32_t lo = 0, hi = 0x7f800000u;  // +0 .. +inf; byte(+inf) = 255
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo) / 2;
      if (srgb_byte(float_from_bits(mid)) >= (uint32_t)j) hi = mid;
      else lo = mid + 1;
    }
    T.t[j] = float_from_bits(lo);
  }
  return T;
}

const SrgbTable& table() {
  static std::once_flag once;
  static SrgbTable T;
  std::call_once(once, [] { T = build_table(); });
  return T;
}

constexpr int kPix = 2;  // pixels per thread per iteration

// Number of thresholds at or below x.  A fast estimate (the SFU power) lands within a step or
// two of the answer; walking the exact thresholds from there makes the result independent of
// the estimate's accuracy.  NaN and negative x give 0, +inf gives 255.
__device__ __forceinline__ uint32_t lookup(const float* t, float x) {
  const float g = fmaf(1.055f, __powf(fmaxf(x, 0.f) + 1e-6f, 1.0f / 2.4f), -0.055f) * 255.9f;
  int j = g > 0.f ? (g < 255.f ? (int)g : 255) : 0;
  while (j < 255 && t[j + 1] <= x) ++j;
  while (j > 0 && !(t[j] <= x)) --j;
  return (uint32_t)j;
}

__global__ void __launch_bounds__(256) tonemap_srgb_kernel(const __grid_constant__ SrgbTable T,
                                                           const float4* __restrict__ src, int64_t n,
                                                           uint32_t* __restrict__ dst) {
  __shared__ float t[256];
  t[threadIdx.x] = T.t[threadIdx.x];
  __syncthreads();
  // a block covers kPix * 256 consecutive pixels per iteration; each thread keeps kPix
  // coalesced loads in flight before the lookups
  const int64_t span = (int64_t)kPix * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * span + threadIdx.x; base < n; base += (int64_t)gridDim.x * span) {
    float4 v[kPix];
#pragma unroll
    for (int k = 0; k < kPix; ++k) {
      const int64_t i = base + (int64_t)k * blockDim.x;
      if (i < n) v[k] = __ldg(src + i);
    }
#pragma unroll
    for (int k = 0; k < kPix; ++k) {
      const int64_t i = base + (int64_t)k * blockDim.x;
      if (i < n) dst[i] = lookup(t, v[k].x) | (lookup(t, v[k].y) << 8) | (lookup(t, v[k].z) << 16) | (255u << 24);
    }
  }
}

}  // namespace

void launch_tonemap_srgb(const float* src, int64_t n, uint32_t* dst, cudaStream_t st) {
  if (n < 0) fail(NWPRT_INVALID_ARG, "tonemap: negative pixel count");
  if (n == 0) return;
  if (!src || !dst) fail(NWPRT_INVALID_ARG, "tonemap: null pointer");
  if ((reinterpret_cast<uintptr_t>(src) & 15) || (reinterpret_cast<uintptr_t>(dst) & 3))
    fail(NWPRT_INVALID_ARG, "tonemap: src must be 16-byte aligned (float4), dst 4-byte aligned");
  int dev = 0, sms = 0;
  NWPRT_CUDA(cudaGetDevice(&dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t blocks = (n + kPix * 256 - 1) / (kPix * 256);
  const int64_t cap = (int64_t)sms * 64;  // measured: 8 -> 64 blocks per SM took 16 frames from 193 to 164 us
  tonemap_srgb_kernel<<<(int)(blocks < cap ? blocks : cap), 256, 0, st>>>(
      table(), reinterpret_cast<const float4*>(src), n, dst);
  NWPRT_CUDA(cudaGetLastError());
}

}  // namespace nwprt

// Spherical-harmonics PRT baseline kernels.
//
//  * sh_project: env-map SH coefficients L[81][3] of a cubemap, the quantity the
//    reference loads precomputed from sh/<name>.npy (Renderer/EnvironmentMap.cpp:70-77).
//    Cube projection of device_functions/sh.h:59-103 (weight (uc^2+vc^2+1)^(-3/2) * 4/S^2)
//    with texel directions from the cubemap convention of device_functions/cubeMap.cu:97-113
//    and the pbrt-v2 real SH basis of device_functions/shaderUtils.h:231-338 (order 8).
//    Deterministic: per-block partial sums in a caller-provided workspace, then one
//    fixed-order reduction.
//  * sh_dot: per-pixel out = |sum_j T[p][j] * L[j]| (RGB), the light-vector product of
//    __closesthit__SHradiance (device_functions/devicePrograms.cu:479-490).  A pure
//    streaming kernel: persistent CTAs pull 128-pixel chunks of T through a 4-stage
//    cp.async.bulk (TMA) ring into shared memory; the dot product accumulates with
//    fmaf in coefficient order (bit-identical to the oracle's orc_sh_dot_f32).
#include <cmath>

#include "nwprt_internal.cuh"

namespace nwprt {
namespace {

constexpr int kLmax = 8;
constexpr int kNc = (kLmax + 1) * (kLmax + 1);  // 81

__host__ __device__ constexpr int shi(int l, int m) { return l * l + l + m; }

// Normalisation K(l,m) = sqrt((2l+1)/(4 pi) * (l-m)!/(l+m)!) for m >= 0 at index l*l+l+m
// (the pbrt-v2 basis, device_functions/shaderUtils.h:283-285).  The table is evaluated at
// compile time (Newton's iteration for the square root, in double, then rounded once to
// float: the same bits as the correctly rounded std::sqrt for all 45 entries), so it is part
// of the module image and no call ever copies it to the device.
constexpr double sqrt_newton(double x) {
  double r = x > 1.0 ? x : 1.0;
  for (int i = 0; i < 200; ++i) r = 0.5 * (r + x / r);
  return r;
}
struct ShKTable {
  float v[kNc];
};
constexpr ShKTable make_sh_k_table() {
  ShKTable t{};
  for (int l = 0; l <= kLmax; ++l)
    for (int m = 0; m <= l; ++m) {
      double ratio = 1.0;
      for (int q = l - m + 1; q <= l + m; ++q) ratio /= (double)q;
      t.v[shi(l, m)] = (float)sqrt_newton((2.0 * l + 1.0) / (4.0 * 3.14159265358979323846) * ratio);
    }
  return t;
}
__constant__ ShKTable c_shK = make_sh_k_table();

__device__ __forceinline__ void sh_eval8(float x, float y, float z, float* Y) {
  float P[kNc];
  const float s = sqrtf(fmaxf(0.f, 1.f - z * z));
#pragma unroll
  for (int m = 0; m <= kLmax; ++m) {
    float pmm = 1.f;
#pragma unroll
    for (int i = 1; i <= m; ++i) pmm *= -(2.f * i - 1.f) * s;
    P[shi(m, m)] = pmm;
    if (m + 1 <= kLmax) P[shi(m + 1, m)] = z * (2.f * m + 1.f) * pmm;
#pragma unroll
    for (int l = m + 2; l <= kLmax; ++l)
      P[shi(l, m)] = ((2.f * l - 1.f) * z * P[shi(l - 1, m)] - (l + m - 1.f) * P[shi(l - 2, m)]) /
                     (float)(l - m);
  }
  float sn[kLmax + 1], cs[kLmax + 1];
  if (s == 0.f) {
#pragma unroll
    for (int m = 0; m <= kLmax; ++m) { sn[m] = 0.f; cs[m] = 1.f; }
  } else {
    const float sp = y / s, cp = x / s;
    sn[0] = 0.f;
    cs[0] = 1.f;
#pragma unroll
    for (int m = 0; m < kLmax; ++m) {
      sn[m + 1] = sn[m] * cp + cs[m] * sp;
      cs[m + 1] = cs[m] * cp - sn[m] * sp;
    }
  }
  const float sqrt2 = 1.41421356237309515f;
#pragma unroll
  for (int l = 0; l <= kLmax; ++l) {
    Y[shi(l, 0)] = c_shK.v[shi(l, 0)] * P[shi(l, 0)];
#pragma unroll
    for (int m = 1; m <= l; ++m) {
      const float kp = sqrt2 * c_shK.v[shi(l, m)] * P[shi(l, m)];
      Y[shi(l, m)] = kp * cs[m];
      Y[shi(l, -m)] = kp * sn[m];
    }
  }
}

constexpr int kProjThreads = 256;
constexpr int kProjPad = kProjThreads + 1;

__global__ void __launch_bounds__(kProjThreads) sh_project_partial(const float* __restrict__ faces,
                                                                   int S, float* __restrict__ part) {
  extern __shared__ float sm[];
  float* sY = sm;                         // [81][kProjPad]   Y_k * dA
  float* sF = sY + kNc * kProjPad;        // [3][kProjPad]    texel radiance
  const int tid = threadIdx.x;
  const long long SS = (long long)S * S;
  const long long t = (long long)blockIdx.x * kProjThreads + tid;
  float Y[kNc];
  if (t < 6 * SS) {
    const int f = (int)(t / SS);
    const int rem = (int)(t - (long long)f * SS);
    const int r = rem / S, c = rem - r * S;
    const float uc = 2.f * (c + 0.5f) / S - 1.f, vc = 2.f * (r + 0.5f) / S - 1.f;
    float x, y, z;
    switch (f) {
      case 0: x = 1.f; y = vc; z = uc; break;
      case 1: x = -1.f; y = vc; z = -uc; break;
      case 2: x = uc; y = 1.f; z = vc; break;
      case 3: x = uc; y = -1.f; z = -vc; break;
      case 4: x = uc; y = vc; z = -1.f; break;
      default: x = -uc; y = vc; z = 1.f; break;
    }
    const float q = uc * uc + vc * vc + 1.f;
    const float inv = rsqrtf(q);
    sh_eval8(x * inv, y * inv, z * inv, Y);
    const float dA = inv * inv * inv * (4.f / ((float)S * (float)S));
#pragma unroll
    for (int k = 0; k < kNc; ++k) sY[k * kProjPad + tid] = Y[k] * dA;
    const float* tx = faces + t * 3;
    sF[tid] = tx[0];
    sF[kProjPad + tid] = tx[1];
    sF[2 * kProjPad + tid] = tx[2];
  } else {
#pragma unroll
    for (int k = 0; k < kNc; ++k) sY[k * kProjPad + tid] = 0.f;
    sF[tid] = sF[kProjPad + tid] = sF[2 * kProjPad + tid] = 0.f;
  }
  __syncthreads();
  if (tid < kNc * 3) {
    const int k = tid / 3, ch = tid - 3 * (tid / 3);
    float acc = 0.f;
    for (int i = 0; i < kProjThreads; ++i) acc = fmaf(sY[k * kProjPad + i], sF[ch * kProjPad + i], acc);
    part[(size_t)blockIdx.x * (kNc * 3) + tid] = acc;
  }
}

__global__ void sh_project_reduce(const float* __restrict__ part, int n_blocks, float* __restrict__ L) {
  const int tid = threadIdx.x;
  if (tid < kNc * 3) {
    float acc = 0.f;
    for (int b = 0; b < n_blocks; ++b) acc += part[(size_t)b * (kNc * 3) + tid];
    L[tid] = acc;
  }
}

// ------------------------------------------------------------------ sh_dot
constexpr int kDotPx = 128;
constexpr int kDotStages = 4;
constexpr int kDotConsumers = 128;
constexpr int kDotThreads = kDotConsumers + 32;

__global__ void __launch_bounds__(kDotThreads, 1)
    sh_dot_stream(const float* __restrict__ T, long long n_chunks, int nc, const float* __restrict__ Lg,
                  int abs_out, float* __restrict__ out, uint32_t* err) {
  extern __shared__ __align__(128) char smraw[];
  const uint32_t stage_bytes = (uint32_t)(kDotPx * nc * 4);
  const uint32_t stage_stride = (stage_bytes + 127u) & ~127u;
  float* sL = (float*)(smraw + kDotStages * stage_stride);
  uint64_t* full = (uint64_t*)(smraw + kDotStages * stage_stride + ((nc * 3 * 4 + 15) & ~15));
  uint64_t* empty = full + kDotStages;
  const int tid = threadIdx.x;
  for (int i = tid; i < nc * 3; i += blockDim.x) sL[i] = Lg[i];
  if (tid == 0) {
    for (int s = 0; s < kDotStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kDotConsumers / 32);
    }
    fence_barrier_init();
  }
  __syncthreads();
  const long long my_chunks =
      blockIdx.x < n_chunks ? (n_chunks - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  if (tid >= kDotConsumers) {
    // producer warp: one elected lane streams chunks into the ring
    if (tid == kDotConsumers) {
      for (long long i = 0; i < my_chunks; ++i) {
        const int s = (int)(i % kDotStages);
        const uint32_t ph = (uint32_t)((i / kDotStages) & 1);
        if (!mbar_wait(&empty[s], ph ^ 1u, err)) break;
        const long long chunk = blockIdx.x + i * gridDim.x;
        mbar_arrive_expect_tx(&full[s], stage_bytes);
        bulk_g2s(smraw + s * stage_stride, T + chunk * (long long)kDotPx * nc, stage_bytes, &full[s]);
      }
    }
    return;
  }
  for (long long i = 0; i < my_chunks; ++i) {
    const int s = (int)(i % kDotStages);
    const uint32_t ph = (uint32_t)((i / kDotStages) & 1);
    if (!mbar_wait(&full[s], ph, err)) break;
    const float* buf = (const float*)(smraw + s * stage_stride) + tid * nc;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    for (int j = 0; j < nc; ++j) {
      const float t = buf[j];
      a0 = fmaf(t, sL[j * 3 + 0], a0);
      a1 = fmaf(t, sL[j * 3 + 1], a1);
      a2 = fmaf(t, sL[j * 3 + 2], a2);
    }
    __syncwarp();
    if ((tid & 31) == 0) mbar_arrive(&empty[s]);
    if (abs_out) { a0 = fabsf(a0); a1 = fabsf(a1); a2 = fabsf(a2); }
    const long long px = (blockIdx.x + i * gridDim.x) * (long long)kDotPx + tid;
    reinterpret_cast<float4*>(out)[px] = make_float4(a0, a1, a2, 1.f);
  }
}

__global__ void sh_dot_tail(const float* __restrict__ T, long long px0, long long n_px, int nc,
                            const float* __restrict__ L, int abs_out, float* __restrict__ out) {
  const long long px = px0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (px >= n_px) return;
  const float* t = T + px * nc;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
  for (int j = 0; j < nc; ++j) {
    a0 = fmaf(t[j], L[j * 3 + 0], a0);
    a1 = fmaf(t[j], L[j * 3 + 1], a1);
    a2 = fmaf(t[j], L[j * 3 + 2], a2);
  }
  if (abs_out) { a0 = fabsf(a0); a1 = fabsf(a1); a2 = fabsf(a2); }
  reinterpret_cast<float4*>(out)[px] = make_float4(a0, a1, a2, 1.f);
}

}  // namespace

size_t sh_project_workspace_bytes(int S) {
  const long long n = 6LL * S * S;
  const long long blocks = (n + kProjThreads - 1) / kProjThreads;
  return (size_t)blocks * kNc * 3 * sizeof(float);
}

void launch_sh_project(const float* faces, int S, float* L, float* workspace, cudaStream_t st) {
  const long long n = 6LL * S * S;
  const int blocks = (int)((n + kProjThreads - 1) / kProjThreads);
  const size_t smem = sizeof(float) * (kNc + 3) * kProjPad;
  NWPRT_CUDA(cudaFuncSetAttribute(sh_project_partial, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  sh_project_partial<<<blocks, kProjThreads, smem, st>>>(faces, S, workspace);
  NWPRT_CUDA(cudaGetLastError());
  sh_project_reduce<<<1, 256, 0, st>>>(workspace, blocks, L);
  NWPRT_CUDA(cudaGetLastError());
}

void launch_sh_dot(const float* T, int64_t n_px, int nc, const float* L, int abs_out, float* out,
                   uint32_t* err, cudaStream_t st) {
  if (n_px < 0 || nc < 1 || nc > 1024) fail(NWPRT_INVALID_ARG, "sh_dot: bad sizes");
  if (n_px == 0) return;
  if (((uintptr_t)T & 15) || ((uintptr_t)out & 15))
    fail(NWPRT_INVALID_ARG, "sh_dot: T and out must be 16-byte aligned");
  const long long n_chunks = n_px / kDotPx;
  const long long tail0 = n_chunks * kDotPx;
  const size_t stage = ((size_t)kDotPx * nc * 4 + 127) & ~size_t(127);
  const size_t smem = kDotStages * stage + ((nc * 3 * 4 + 15) & ~15) + 2 * kDotStages * 8;
  int dev = 0, sms = 0, max_smem = 0;
  NWPRT_CUDA(cudaGetDevice(&dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (n_chunks > 0 && smem <= (size_t)max_smem) {
    NWPRT_CUDA(cudaFuncSetAttribute(sh_dot_stream, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = (int)(n_chunks < sms ? n_chunks : sms);
    sh_dot_stream<<<grid, kDotThreads, smem, st>>>(T, n_chunks, nc, L, abs_out, out, err);
    NWPRT_CUDA(cudaGetLastError());
  } else {
    // coefficient counts too large for the staged ring: plain loads for everything
    const long long blocks = (n_px + 255) / 256;
    sh_dot_tail<<<(unsigned)blocks, 256, 0, st>>>(T, 0, n_px, nc, L, abs_out, out);
    NWPRT_CUDA(cudaGetLastError());
    return;
  }
  if (tail0 < n_px) {
    const long long rem = n_px - tail0;
    sh_dot_tail<<<(unsigned)((rem + 255) / 256), 256, 0, st>>>(T, tail0, n_px, nc, L, abs_out, out);
    NWPRT_CUDA(cudaGetLastError());
  }
}

}  // namespace nwprt

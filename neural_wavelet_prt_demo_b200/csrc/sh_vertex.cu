// SH radiance per mesh vertex and its barycentric interpolation: the SH path's shading
// (Renderer/device_functions/devicePrograms.cu:427-490) without the ray tracer.
//
// Per vertex v:  light[k] = sum_j T[v][k][j] L[j]        (RGB; j ascending, one fma per term)
//                c[v]     = | sum_k light[k] * brdf[v][k] |   (k ascending, one fma per term)
// with T the vertex's n x n transfer matrix (n = 81 at SH degree 8, 26 KB per vertex), L the
// env SH coefficients and brdf the vertex's BRDF projected on the SH basis (the reference
// projects it by sampling its material callables, devicePrograms.cu:448-474; here it is an
// input like T).  Per pixel: (1-u-v) c[i0] + u c[i1] + v c[i2].
//
// The vertex pass streams T once and does 2 n^2 FMAs per 4 n^2 bytes: HBM-bound.  One warp
// per vertex: the warp copies T[v] and brdf[v] into shared memory with cp.async, all copies
// in flight at once.  T[v] starts 4 (v mod 4) bytes past a 16-byte boundary (n^2 = 6561 is
// odd), so the staging base is shifted by the same amount and the body moves in 16-byte
// copies, with a head and a tail of at most three 4-byte copies.  Then lane k walks row k
// sequentially (so the sum order is the reference's).  The row stride n = 81 is odd, so the
// 32 lanes read 32 different banks.  Eight warps per SM overlap one vertex's copy with
// another's arithmetic.
#include "nwprt_internal.cuh"

namespace nwprt {
namespace {

constexpr int kMaxN = 81;
constexpr int kWarps = 8;

// Shared memory in floats: env SH, then per warp light[k] and brdf[v] ([kMaxN][3] each), then
// per warp a T staging area of n^2 floats plus up to 3 of alignment shift, rounded to 16 bytes.
__host__ __device__ constexpr int stage_offset() { return ((1 + 2 * kWarps) * kMaxN * 3 + 3) & ~3; }
__host__ __device__ constexpr int stage_stride(int n) { return (n * n + 3 + 3) & ~3; }

__global__ void __launch_bounds__(kWarps * 32) sh_vertex_kernel(const float* __restrict__ T,
                                                                const float* __restrict__ brdf,
                                                                const float* __restrict__ L, int64_t V, int n,
                                                                float* __restrict__ out) {
  extern __shared__ __align__(16) float smem[];
  const int nn = n * n;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* sL = smem;                                              // [kMaxN][3] env SH
  float* light = smem + (1 + warp) * kMaxN * 3;                  // [kMaxN][3] this warp's light[k]
  float* sb = smem + (1 + kWarps + warp) * kMaxN * 3;            // [kMaxN][3] this warp's brdf[v]
  float* stage = smem + stage_offset() + warp * stage_stride(n);  // this warp's T staging (16-byte aligned)
  for (int i = threadIdx.x; i < n * 3; i += blockDim.x) sL[i] = L[i];
  __syncthreads();
  for (int64_t v = (int64_t)blockIdx.x * kWarps + warp; v < V; v += (int64_t)gridDim.x * kWarps) {
    const float* src = T + v * nn;
    const float* bsrc = brdf + v * n * 3;
    // t[i] and src[i] share their offset modulo 16 bytes
    const int mis = (int)((reinterpret_cast<uintptr_t>(src) >> 2) & 3);
    float* t = stage + mis;
    const int head = ((4 - mis) & 3) < nn ? ((4 - mis) & 3) : nn;
    const int body = (nn - head) & ~3;
    if (lane < head)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(t + lane)), "l"(src + lane) : "memory");
    for (int i = head + 4 * lane; i < head + body; i += 128)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(t + i)), "l"(src + i) : "memory");
    for (int i = head + body + lane; i < nn; i += 32)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(t + i)), "l"(src + i) : "memory");
    for (int i = lane; i < n * 3; i += 32)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(sb + i)), "l"(bsrc + i) : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncwarp();
    // lane k owns rows k, k+32, k+64: light[k] = sum_j T[k][j] L[j], j ascending
    for (int k = lane; k < n; k += 32) {
      float l0 = 0.f, l1 = 0.f, l2 = 0.f;
      const float* row = t + k * n;
      for (int j = 0; j < n; ++j) {
        const float tj = row[j];
        l0 = fmaf(tj, sL[j * 3 + 0], l0);
        l1 = fmaf(tj, sL[j * 3 + 1], l1);
        l2 = fmaf(tj, sL[j * 3 + 2], l2);
      }
      light[k * 3] = l0;
      light[k * 3 + 1] = l1;
      light[k * 3 + 2] = l2;
    }
    __syncwarp();
    // c = | sum_k light[k] * brdf[k] |, k ascending
    if (lane == 0) {
      float s0 = 0.f, s1 = 0.f, s2 = 0.f;
      for (int k = 0; k < n; ++k) {
        s0 = fmaf(light[k * 3], sb[k * 3 + 0], s0);
        s1 = fmaf(light[k * 3 + 1], sb[k * 3 + 1], s1);
        s2 = fmaf(light[k * 3 + 2], sb[k * 3 + 2], s2);
      }
      out[v * 3 + 0] = fabsf(s0);
      out[v * 3 + 1] = fabsf(s1);
      out[v * 3 + 2] = fabsf(s2);
    }
    __syncwarp();
  }
}

__global__ void sh_interpolate_kernel(const float* __restrict__ vc, const int32_t* __restrict__ tri,
                                      const float* __restrict__ uv, int64_t P, int64_t V, float4* __restrict__ out,
                                      uint32_t* err) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += stride) {
    const int32_t i0 = __ldg(tri + p * 3), i1 = __ldg(tri + p * 3 + 1), i2 = __ldg(tri + p * 3 + 2);
    const float u = __ldg(uv + p * 2), w = __ldg(uv + p * 2 + 1);
    if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= V || i1 >= V || i2 >= V) {
      atomicCAS(err, 0u, (uint32_t)kDevBadIndex);
      out[p] = make_float4(0.f, 0.f, 0.f, 1.f);
      continue;
    }
    const float b0 = __fsub_rn(__fsub_rn(1.f, u), w);
    float r[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      r[c] = fmaf(w, __ldg(vc + i2 * 3 + c), fmaf(u, __ldg(vc + i1 * 3 + c), __fmul_rn(b0, __ldg(vc + i0 * 3 + c))));
    out[p] = make_float4(r[0], r[1], r[2], 1.f);
  }
}

}  // namespace

void launch_sh_vertex(const float* T, const float* brdf, const float* L, int64_t V, int n, float* out,
                      cudaStream_t st) {
  if (V < 0 || n < 1 || n > kMaxN) fail(NWPRT_INVALID_ARG, "sh_vertex: need V >= 0 and 1 <= n <= 81");
  if (V == 0) return;
  if (!T || !brdf || !L || !out) fail(NWPRT_INVALID_ARG, "sh_vertex: null pointer");
  int dev = 0, sms = 0;
  NWPRT_CUDA(cudaGetDevice(&dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const size_t smem = (size_t)(stage_offset() + kWarps * stage_stride(n)) * sizeof(float);
  NWPRT_CUDA(cudaFuncSetAttribute(sh_vertex_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t blocks = (V + kWarps - 1) / kWarps;
  const int64_t cap = (int64_t)sms;  // one 8-warp CTA per SM at n = 81 (227 KB of staging)
  sh_vertex_kernel<<<(int)(blocks < cap ? blocks : cap), kWarps * 32, smem, st>>>(T, brdf, L, V, n, out);
  NWPRT_CUDA(cudaGetLastError());
}

void launch_sh_interpolate(const float* vc, int64_t V, const int32_t* tri, const float* uv, int64_t P, float* out,
                           uint32_t* err, cudaStream_t st) {
  if (P < 0 || V < 0) fail(NWPRT_INVALID_ARG, "sh_interpolate: negative size");
  if (P == 0) return;
  if (!vc || !tri || !uv || !out) fail(NWPRT_INVALID_ARG, "sh_interpolate: null pointer");
  if (reinterpret_cast<uintptr_t>(out) & 15) fail(NWPRT_INVALID_ARG, "sh_interpolate: out must be 16-byte aligned");
  int dev = 0, sms = 0;
  NWPRT_CUDA(cudaGetDevice(&dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t blocks = (P + 255) / 256, cap = (int64_t)sms * 8;
  sh_interpolate_kernel<<<(int)(blocks < cap ? blocks : cap), 256, 0, st>>>(vc, tri, uv, P, V,
                                                                             reinterpret_cast<float4*>(out), err);
  NWPRT_CUDA(cudaGetLastError());
}

}  // namespace nwprt

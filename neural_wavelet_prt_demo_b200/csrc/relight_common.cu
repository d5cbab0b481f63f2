// Per-frame and per-env preparation kernels of the relight path.
//
//  * pack_gbuffer: the reference's waveletDataCopy (Renderer/tinycudann/utils_kernels.h:7-49)
//    without its K-fold replication: one 16-float input row per pixel
//    (layout prt_globals.h:4-13: pos, normal, reflect, log(25r+1)/log(26), 2kd-1, 2ks-1).
//    The reference writes 64*K bytes per pixel; this writes 64.  The roughness log uses
//    logf_series (correctly rounded, identical on host, device and oracle).
//  * gather_embedding: the per-env half of ptwise_mlt (utils_kernels.h:110-127):
//    E_k[k][d] = E[d][idx_k] for the env's K selected coefficients, so the fused
//    transport kernels read one contiguous row per wavelet instead of a strided gather
//    per (pixel, wavelet).  Indices outside [0, n_coeffs) raise kDevBadIndex and read 0.
#include <cmath>

#include "nwprt_internal.cuh"

namespace nwprt {
namespace {

__global__ void pack_gbuffer_kernel(int64_t n, const float4* __restrict__ pos,
                                    const float4* __restrict__ nrm, const float4* __restrict__ refl,
                                    const float* __restrict__ rough, const float4* __restrict__ kd,
                                    const float4* __restrict__ ks, float rgh_den,
                                    float4* __restrict__ out) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const float4 a = pos[p], b = nrm[p], c = refl[p], d = kd[p], e = ks[p];
  const float r = logf_series(fmaf(25.f, rough[p], 1.f)) * rgh_den;
  out[p * 4 + 0] = make_float4(a.x, a.y, a.z, b.x);
  out[p * 4 + 1] = make_float4(b.y, b.z, c.x, c.y);
  out[p * 4 + 2] = make_float4(c.z, r, 2.f * d.x - 1.f, 2.f * d.y - 1.f);
  out[p * 4 + 3] = make_float4(2.f * d.z - 1.f, 2.f * e.x - 1.f, 2.f * e.y - 1.f, 2.f * e.z - 1.f);
}

// One thread per feature pair (k, 2i..2i+1): both FP32 values, and (out_h) their BF16 pair.
__global__ void gather_embedding_kernel(const float* __restrict__ emb, int D, int n_coeffs,
                                        const int32_t* __restrict__ idx, int K,
                                        float* __restrict__ out, uint32_t* __restrict__ out_h, uint32_t* err) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int H = D / 2;
  if (t >= (int64_t)K * H) return;
  const int k = (int)(t / H), d = 2 * (int)(t - (int64_t)k * H);
  const int32_t j = idx[k];
  float v0 = 0.f, v1 = 0.f;
  if (j >= 0 && j < n_coeffs) {
    v0 = emb[(int64_t)d * n_coeffs + j];
    v1 = emb[(int64_t)(d + 1) * n_coeffs + j];
  } else if (err) {
    atomicCAS(err, 0u, (uint32_t)kDevBadIndex);
  }
  out[(int64_t)k * D + d] = v0;
  out[(int64_t)k * D + d + 1] = v1;
  if (out_h) {
    uint32_t h;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(h) : "f"(v1), "f"(v0));
    out_h[t] = h;
  }
}

}  // namespace

void launch_pack_gbuffer(const nwprt_gbuffer& g, float* packed, cudaStream_t st) {
  const int64_t n = (int64_t)g.width * g.height;
  if (n == 0) return;
  // the reference's constant 1/log(26) (utils_kernels.h:21), evaluated once on the host
  const float rgh_den = 1.f / logf_series(25.f + 1.f);
  const int bs = 256;
  pack_gbuffer_kernel<<<(unsigned)((n + bs - 1) / bs), bs, 0, st>>>(
      n, (const float4*)g.first_hit_pos, (const float4*)g.world_normal, (const float4*)g.reflect_dir,
      g.roughness, (const float4*)g.kd, (const float4*)g.ks, rgh_den, (float4*)packed);
  NWPRT_CUDA(cudaGetLastError());
}

void launch_gather_embedding(const float* emb, int D, int n_coeffs, const int32_t* idx, int K,
                             float* out_kd, uint32_t* out_h, uint32_t* err, cudaStream_t st) {
  if (D % 2) fail(NWPRT_UNSUPPORTED, "embedding gather needs an even feature count");
  const int64_t n = (int64_t)K * (D / 2);
  if (n == 0) return;
  gather_embedding_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(emb, D, n_coeffs, idx, K,
                                                                        out_kd, out_h, err);
  NWPRT_CUDA(cudaGetLastError());
}

}  // namespace nwprt

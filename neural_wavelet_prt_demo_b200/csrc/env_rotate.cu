// Env-map rotation: resamples a cubemap under a rotation R, L_R(d) = L(R^T d).
//
// The serving stream relights with rotated copies of resident env maps; the rotated faces
// then go through the Haar + top-K kernel like any new map.  Sampling follows the
// reference's cubemap lookup exactly: texel centre -> direction by EnvUVToDirec
// (device_functions/cubeMap.cu:97-113, left unnormalised: the face choice and (u,v) only
// depend on the direction), direction -> face and (u,v) by EnvDirecToUV (cubeMap.cu:23-96,
// the six tests applied in order, a later match overriding an earlier one), and a
// point-sampled, wrap-addressed texel fetch as the faces are bound in buildLights
// (Renderer/textures.h:64-68, textures.cpp:32-36).  Every operation is an IEEE FP32 op
// without contraction, so the CPU oracle selects the same source texel bit for bit.
#include "nwprt_internal.cuh"

namespace nwprt {
namespace {

struct Rot {
  float m[9];  // row-major R
};

__device__ __forceinline__ void uv_to_dir(int f, float uc, float vc, float& x, float& y, float& z) {
  switch (f) {
    case 0: x = 1.f; y = vc; z = uc; break;
    case 1: x = -1.f; y = vc; z = -uc; break;
    case 2: x = uc; y = 1.f; z = vc; break;
    case 3: x = uc; y = -1.f; z = -vc; break;
    case 4: x = uc; y = vc; z = -1.f; break;
    default: x = -uc; y = vc; z = 1.f; break;
  }
}

__global__ void env_rotate_kernel(const float* __restrict__ src, int S, Rot R, float* __restrict__ dst) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long SS = (long long)S * S;
  if (t >= 6 * SS) return;
  const int f = (int)(t / SS);
  const int rem = (int)(t - (long long)f * SS);
  const int r = rem / S, c = rem - r * S;
  const float fs = (float)S;
  // texel centre (u, v) -> [-1, 1]
  const float uc = __fsub_rn(__fmul_rn(2.f, __fdiv_rn(__fadd_rn((float)c, 0.5f), fs)), 1.f);
  const float vc = __fsub_rn(__fmul_rn(2.f, __fdiv_rn(__fadd_rn((float)r, 0.5f), fs)), 1.f);
  float x, y, z;
  uv_to_dir(f, uc, vc, x, y, z);
  // source direction R^T d
  const float sx = __fadd_rn(__fadd_rn(__fmul_rn(R.m[0], x), __fmul_rn(R.m[3], y)), __fmul_rn(R.m[6], z));
  const float sy = __fadd_rn(__fadd_rn(__fmul_rn(R.m[1], x), __fmul_rn(R.m[4], y)), __fmul_rn(R.m[7], z));
  const float sz = __fadd_rn(__fadd_rn(__fmul_rn(R.m[2], x), __fmul_rn(R.m[5], y)), __fmul_rn(R.m[8], z));
  const float ax = fabsf(sx), ay = fabsf(sy), az = fabsf(sz);
  float maxa = 1.f, su = 0.f, sv = 0.f;
  int sf = 0;
  if (sx > 0.f && ax >= ay && ax >= az) { maxa = ax; su = sz; sv = sy; sf = 0; }
  if (!(sx > 0.f) && ax >= ay && ax >= az) { maxa = ax; su = -sz; sv = sy; sf = 1; }
  if (sy > 0.f && ay >= ax && ay >= az) { maxa = ay; su = sx; sv = sz; sf = 2; }
  if (!(sy > 0.f) && ay >= ax && ay >= az) { maxa = ay; su = sx; sv = -sz; sf = 3; }
  if (!(sz > 0.f) && az >= ax && az >= ay) { maxa = az; su = sx; sv = sy; sf = 4; }
  if (sz > 0.f && az >= ax && az >= ay) { maxa = az; su = -sx; sv = sy; sf = 5; }
  if (!(maxa > 0.f)) { maxa = 1.f; su = -1.f; sv = -1.f; sf = 0; }  // singular R: texel (0, 0)
  const float u = __fmul_rn(0.5f, __fadd_rn(__fdiv_rn(su, maxa), 1.f));
  const float v = __fmul_rn(0.5f, __fadd_rn(__fdiv_rn(sv, maxa), 1.f));
  int col = (int)floorf(__fmul_rn(u, fs));
  int row = (int)floorf(__fmul_rn(v, fs));
  col %= S;
  row %= S;
  if (col < 0) col += S;
  if (row < 0) row += S;
  const float* s = src + (((long long)sf * S + row) * S + col) * 3;
  float* d = dst + t * 3;
  d[0] = s[0];
  d[1] = s[1];
  d[2] = s[2];
}

}  // namespace

void launch_env_rotate(const float* src, int S, const float* R_host, float* dst, cudaStream_t st) {
  if (!src || !dst || !R_host) fail(NWPRT_INVALID_ARG, "env_rotate: null pointer");
  if (S < 1 || S > 4096) fail(NWPRT_INVALID_ARG, "env_rotate: face size out of range");
  if (src == dst) fail(NWPRT_INVALID_ARG, "env_rotate: source and destination must differ");
  Rot R;
  for (int i = 0; i < 9; ++i) {
    if (!(R_host[i] == R_host[i]) || R_host[i] > 2.f || R_host[i] < -2.f)
      fail(NWPRT_INVALID_ARG, "env_rotate: rotation entries must be finite and in [-2, 2]");
    R.m[i] = R_host[i];
  }
  const long long n = 6LL * S * S;
  env_rotate_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src, S, R, dst);
  NWPRT_CUDA(cudaGetLastError());
}

}  // namespace nwprt

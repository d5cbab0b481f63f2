// Host build of the reference's own relight kernels -- TEST INFRASTRUCTURE ONLY.
//
// Compiles Renderer/tinycudann/utils_kernels.h from the reference tree, unmodified,
// for the CPU: __global__ functions become plain functions and the CUDA thread
// indices become thread-local variables that the drivers below set for every
// "thread" of the launch grid.  The result (oracle/_ref/libref_utils.so) pins the
// oracle's G-buffer remap, embedding gather and clamped radiance sum against the
// reference's code.  Built by oracle/Makefile only where the reference tree exists.
#include <cstdint>
#include <cmath>

struct nwprt_ref_dim3 { unsigned x, y, z; };
struct int2 { int x, y; };
static thread_local nwprt_ref_dim3 threadIdx, blockIdx, blockDim;
#define __global__ static
#include "tinycudann/utils_kernels.h"
#undef __global__

static void grid2d(int w, int h, int x, int y) {
  blockDim = {1, 1, 1};
  threadIdx = {0, 0, 0};
  blockIdx = {(unsigned)x, (unsigned)y, 0};
  (void)w; (void)h;
}

extern "C" {

int ref_wavelet_num(void) { return WAVELETNUM; }

// prt::waveletDataCopy<float> over a W x H grid; out: [W*H*WAVELETNUM][16]
void ref_wavelet_data_copy(int w, int h, const float* pos, const float* normal,
                           const float* reflect, const float* rough, const float* kd,
                           const float* ks, float* out) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      grid2d(w, h, x, y);
      prt::waveletDataCopy<float>(int2{w, h}, pos, normal, reflect, rough, kd, ks, out);
    }
}

// prt::computeResponse over a W x H grid; response: [W*H*WAVELETNUM][3]
void ref_compute_response(int w, int h, const float* response, const float* direct,
                          const float* light, const uint8_t* flag, float* indirect,
                          float* with_direct) {
  static_assert(sizeof(bool) == 1, "bool flag buffer");
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      grid2d(w, h, x, y);
      prt::computeResponse(int2{w, h}, response, direct, light,
                           reinterpret_cast<const bool*>(flag), indirect, with_direct);
    }
}

// prt::ptwise_mlt<float> as launched by linear_kernel (1-D over n_elements)
void ref_ptwise_mlt(uint32_t n_elements, uint32_t batch, const float* inp, const float* emb,
                    const int* coefs, float* out) {
  blockDim = {1, 1, 1};
  threadIdx = {0, 0, 0};
  for (uint32_t i = 0; i < n_elements; ++i) {
    blockIdx = {i, 0, 0};
    prt::ptwise_mlt<float>(n_elements, batch, inp, emb, coefs, out);
  }
}

}  // extern "C"

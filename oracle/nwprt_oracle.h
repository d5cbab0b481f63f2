/* CPU oracle for the neural wavelet PRT relight path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker for the CUDA path: only tests/, the smoke check
 * and bench.py's CPU-baseline leg load it.  The product path never calls it.
 *
 * Parity status: PARTLY PINNED.
 *  - G-buffer remap, wavelet-embedding gather and the clamped radiance sum are
 *    pinned against the reference's own kernels (Renderer/tinycudann/
 *    utils_kernels.h) compiled for the host by oracle/Makefile into oracle/_ref.
 *  - Hash grid and MLPs: parity unpinned.  They live in tiny-cuda-nn, which is an
 *    empty submodule in the reference (.gitmodules:1-3); this file restates the
 *    published Instant-NGP hash encoding (Mueller et al. 2022) and a bias-free
 *    ReLU MLP.
 *  - Haar transform + top-K: the reference only loads precomputed results
 *    (EnvironmentMap.cpp:97-108); the order defined here IS the reference order.
 *  - SH basis / projection: restated from the pbrt-v2 method the reference uses
 *    (device_functions/shaderUtils.h:231-338, device_functions/sh.h:59-103);
 *    unpinned (the reference's SH code needs OptiX headers).
 *
 * FP32 functions mirror the GPU kernels' operation order (fmaf where the GPU
 * fuses, plain ops elsewhere; built with -ffp-contract=off).  FP64 functions are
 * the accuracy reference for error / PSNR reports.
 */
#ifndef NWPRT_ORACLE_H
#define NWPRT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_LEVELS 32
#define ORC_MAX_LAYERS 16
#define ORC_MAX_WIDTH 256

typedef struct {
  int n_levels, n_features;
  int level_res[ORC_MAX_LEVELS];
  int level_size[ORC_MAX_LEVELS];
  int level_offset[ORC_MAX_LEVELS];
  int aux_width;
  int op_nl, op_in[ORC_MAX_LAYERS], op_out[ORC_MAX_LAYERS];
  int cn_nl, cn_in[ORC_MAX_LAYERS], cn_out[ORC_MAX_LAYERS];
  int n_coeffs;
} orc_net;

typedef struct {
  const float* hash;  /* [sum T_l][F] */
  const float* op;    /* out_prd layers, row-major [out][in], concatenated */
  const float* cn;    /* cmp_net layers */
  const float* emb;   /* [D][n_coeffs] */
} orc_weights;

typedef struct {
  int width, height;
  const float *pos, *normal, *reflect; /* float4 per pixel */
  const float* roughness;              /* float per pixel */
  const float *kd, *ks, *direct;       /* float4 per pixel */
  const uint8_t* flag;                 /* bool per pixel */
} orc_gbuf;

/* ---- env map: Haar + top-K (FP32, bit-exact definition) ---- */
float orc_wavelet_key(float r, float g, float b);
void orc_haar_face(float* face, int S);                      /* in place, [S][S][3] */
void orc_haar_inverse_face_f64(double* face, int S);
int orc_haar_topk(const float* faces, int S, int K, int32_t* idx, float* strength);
int orc_haar_topk_batch(const float* faces, int n_env, int S, int K, int32_t* idx,
                        float* strength, int n_threads);

/* ---- env-map rotation (point-sampled, as the reference's cubemap lookup) ---- */
void orc_env_rotate(const float* src, int S, const float R[9], float* dst);

/* ---- SH baseline ---- */
void orc_sh_eval_f64(double x, double y, double z, int lmax, double* out);
void orc_sh_project_f64(const float* faces, int S, int lmax, double* L, double* L_abs);
void orc_sh_dot_f32(const float* T, int64_t N, int nc, const float* L, int abs_out,
                    float* out4, int n_threads);
void orc_sh_dot_f64(const float* T, int64_t N, int nc, const double* L, int abs_out, double* out3);

/* ---- relight pieces ---- */
float orc_logf_series(float x);
float orc_powf_series(float x, float y);
void orc_tonemap_srgb(const float* src, int64_t n, uint32_t* dst);
void orc_srgb_thresholds(float* t256);
void orc_sh_vertex_radiance(const float* T, const float* brdf, const float* L, int64_t V, int n, float* out);
int64_t orc_sh_interpolate(const float* vc, int64_t V, const int32_t* tri, const float* uv, int64_t P, float* out);
int64_t orc_srgb_threshold_mismatches(const float* t256, int radius);
void orc_remap_f32(const orc_gbuf* g, int64_t px, float row[16]);
void orc_hash_encode_f32(const orc_net* net, const float* hash, const float pos[3], float* out);
void orc_hash_encode_f64(const orc_net* net, const float* hash, const float pos[3], double* out);
/* transport T_k for one pixel and all K wavelets: out[K][3] */
int orc_transport_f32(const orc_net* net, const orc_weights* w, const orc_gbuf* g, int64_t px,
                      const int32_t* idx, int K, float* out);
int orc_transport_f64(const orc_net* net, const orc_weights* w, const orc_gbuf* g, int64_t px,
                      const int32_t* idx, int K, double* out);

/* Full relight over pixels [px_begin, px_end).
 * f32: writes indirect4 / with_direct4 (float4 per pixel, indexed by absolute px).
 * f64: writes rgb3 (double3 per pixel, indexed by px - px_begin).
 * clamp: reference's max(L*T, 0) per term (utils_kernels.h:87-89); kahan: compensated sum. */
int orc_relight_f32(const orc_net* net, const orc_weights* w, const orc_gbuf* g,
                    const int32_t* idx, const float* strength, int K, int clamp, int kahan,
                    int64_t px_begin, int64_t px_end, int n_threads,
                    float* indirect4, float* with_direct4);
/* orc_relight_f32 with the per-pixel input rows given instead of remapped from the G-buffer:
 * rows[(px - px_begin) * 16 + c] in the layout of prt_globals.h:4-13 (the flag and the direct
 * light still come from g).  Feeds the reference's own waveletDataCopy rows
 * (utils_kernels.h:7-49, built from oracle/_ref) through the same network. */
int orc_relight_rows_f32(const orc_net* net, const orc_weights* w, const orc_gbuf* g,
                         const float* rows, const int32_t* idx, const float* strength, int K,
                         int clamp, int kahan, int64_t px_begin, int64_t px_end, int n_threads,
                         float* indirect4, float* with_direct4);
int orc_relight_f64(const orc_net* net, const orc_weights* w, const orc_gbuf* g,
                    const int32_t* idx, const float* strength, int K, int clamp,
                    int64_t px_begin, int64_t px_end, int n_threads, double* rgb3);

int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif

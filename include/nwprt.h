/* nwprt -- B200-native neural wavelet PRT relighting, C ABI (libnwprt.so).
 *
 * This is the drop-in boundary for the reference's neural relight path.  Every
 * entry point names the reference interface it replaces (paths inside the
 * AlstonXiao/neural_wavelet_prt_demo tree).  Plain C: pointers, sizes and status
 * codes only; no exception ever crosses this boundary.
 *
 * Conventions
 *  - Device pointers are borrowed (caller-owned CUDA device memory) unless a
 *    parameter says "host".
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *    All work is stream-ordered on the caller's stream.  Calls that block the host:
 *    nwprt_load_weights / _dir, nwprt_env_get_wavelets, nwprt_calibrate_fp8 and nwprt_sync;
 *    nwprt_env_from_faces / nwprt_env_from_wavelets when their arrays are host memory
 *    (they synchronise `stream` after the upload); nwprt_prepare when a frame grows beyond
 *    the buffers it had (it synchronises the device before it frees them).
 *  - A context is bound to one device and is externally synchronised: one host
 *    thread at a time per context.
 *  - float4 buffers are 16-byte aligned arrays of 4 floats per pixel, row-major
 *    pixel index x + width*y, as the reference's fullFrameCUDA buffers
 *    (Renderer/frames.h:143-183).
 */
#ifndef NWPRT_H
#define NWPRT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NWPRT_ABI_VERSION 1
#if defined(__GNUC__)
#define NWPRT_API __attribute__((visibility("default")))
#else
#define NWPRT_API
#endif
#define NWPRT_MAX_FRAMES 16

/* Error model of the reference: CUDA_CHECK throws std::runtime_error
 * (Renderer/optix7.h:27-38), asserts (tinycudann/tcnn.cu:126).  Here: codes. */
typedef enum {
  NWPRT_OK = 0,
  NWPRT_INVALID_ARG = 1,
  NWPRT_OOM = 2,
  NWPRT_CUDA_ERROR = 3,
  NWPRT_TIMEOUT = 4,
  NWPRT_NOT_READY = 5,
  NWPRT_IO_ERROR = 6,
  NWPRT_UNSUPPORTED = 7
} nwprt_status;

/* Transport MLP arithmetic. */
typedef enum {
  NWPRT_PREC_FP32 = 0, /* plain FP32 SIMT path: the drop-in, <= 1e-5 rel vs the FP32 reference math */
  NWPRT_PREC_BF16 = 1, /* tcgen05 tensor cores, BF16 operands, FP32 accumulate */
  NWPRT_PREC_FP8 = 2   /* tcgen05 tensor cores, E4M3 operands with per-layer scales, FP32 accumulate;
                          needs nwprt_calibrate_fp8 after the weights are loaded */
} nwprt_precision;

typedef struct nwprt_ctx nwprt_ctx;

/* G-buffer of one frame: the fields of fullFrameCUDA the relight reads
 * (Renderer/frames.h:143-183), encoded as the camera program writes them
 * (device_functions/camera.cu:248-270).  All device pointers. */
typedef struct {
  int width, height;
  const float* first_hit_pos; /* float4: (p - bbox.lower) / bbox.size  (fbFirstHitPos) */
  const float* world_normal;  /* float4: n/2 + 0.5                      (fbworldNormal) */
  const float* reflect_dir;   /* float4: r/2 + 0.5                      (fbFirstHitReflecDir) */
  const float* roughness;     /* float                                   (fbRoughness) */
  const float* kd;            /* float4                                  (fbFirstHitKd) */
  const float* ks;            /* float4                                  (fbFirstHitKs) */
  const float* direct;        /* float4: direct light added to the indirect (fbDirectDenoised) */
  const uint8_t* env_map_flag; /* bool: pixel hit geometry              (fbEnvironmentMapFlag) */
} nwprt_gbuffer;

typedef struct {
  int precision;   /* nwprt_precision */
  int clamp_terms; /* 1: sum_k max(L_k * T_k, 0) as utils_kernels.h:87-89 (default); 0: plain product */
  int kahan;       /* 1: Kahan-compensated FP32 sum over k (default); 0: plain FP32 sum */
} nwprt_relight_opts;

/* Host copies of the four weight files of initTCNN (tinycudann/tcnn.cu:58-65),
 * in the layout the config JSON documents (row-major [out][in] dense layers). */
typedef struct {
  const float* hash_params; size_t n_hash_params; /* vtx_enc.npy */
  const float* out_prd;     size_t n_out_prd;     /* out_prd.npy */
  const float* cmp_net;     size_t n_cmp_net;     /* cmp_net.npy */
  const float* wve_enc;     size_t n_wve_enc;     /* wve_enc.npy, [D][6*S*S] */
} nwprt_weights;

/* Sizes derived from the config (for callers sizing their buffers). */
typedef struct {
  int enc_dims;          /* hash-grid output width D = levels * features */
  int n_coeffs;          /* wavelet index space 6*S*S */
  int face_size;         /* S */
  int aux_width;
  size_t n_hash_params, n_out_prd, n_cmp_net, n_wve_enc;
  double flops_per_eval; /* MLP FLOPs per (pixel, wavelet) evaluation, aux product hoisted */
} nwprt_network_info;

/* One relight of a batch (serving): env `env_id` applied to prepared frame `frame_id`. */
typedef struct {
  int env_id;
  int frame_id;
  float* indirect;    /* float4 per pixel (fbPredictedIndirect) */
  float* with_direct; /* float4 per pixel (fbPredictedIndirectWithDirect) */
} nwprt_request;

/* A relight of the pixel range [px_begin, px_end) of a prepared frame (pixel index
 * x + width*y).  Lets a scheduler split large requests into chunks and pack chunks of
 * many requests into one device pass.  px_end <= 0 means "to the end of the frame". */
typedef struct {
  int env_id;
  int frame_id;
  float* indirect;    /* float4 per pixel of the whole frame; only the range is written */
  float* with_direct;
  int64_t px_begin;
  int64_t px_end;
} nwprt_range_request;

/* ---------------------------------------------------------------- library */
NWPRT_API int nwprt_abi_version(void);
NWPRT_API const char* nwprt_status_string(nwprt_status s);
/* Last error message of `ctx`, or of the calling thread when ctx is NULL. */
NWPRT_API const char* nwprt_last_error(const nwprt_ctx* ctx);

/* ---------------------------------------------------------------- engine */
/* Parses the network JSON (keys vtx_enc / cmp_enc / out_prd / cmp_net / wve_enc) and
 * binds a context to `device`.  Replaces the config part of RenderEngine::initTCNN
 * (tinycudann/tcnn.cu:49-56) and PRT_Network's constructor (prt_network.h:38-61). */
NWPRT_API nwprt_status nwprt_create(const char* config_json, int device, nwprt_ctx** out);
NWPRT_API void nwprt_destroy(nwprt_ctx* ctx);
NWPRT_API nwprt_status nwprt_get_network_info(const nwprt_ctx* ctx, nwprt_network_info* info);

/* Uploads weights from host memory (synchronous).  Replaces the weight loading of
 * RenderEngine::initTCNN (tinycudann/tcnn.cu:58-74). */
NWPRT_API nwprt_status nwprt_load_weights(nwprt_ctx* ctx, const nwprt_weights* host);
/* Same from a model directory holding vtx_enc.npy, out_prd.npy, cmp_net.npy,
 * wve_enc.npy (float32 .npy files) -- RenderEngine::initTCNN(modelPath). */
NWPRT_API nwprt_status nwprt_load_weights_dir(nwprt_ctx* ctx, const char* model_dir);
/* 1 when weights and at least one env map are loaded -- RenderEngine::TCNNAvaliable
 * (tinycudann/tcnn.cu:160-162). */
NWPRT_API int nwprt_ready(const nwprt_ctx* ctx);

/* ---------------------------------------------------------------- env maps */
/* Cubemap faces [6][S][S][3] float32 (order +X,-X,+Y,-Y,-Z,+Z; Environment_Map::
 * initCubeFaces, EnvironmentMap.cpp:112-126) -> Haar transform + top-K selection on
 * the device; registers the resulting wavelet table.  `faces_on_device` = 0 reads
 * host memory (copied on `stream`).  Replaces loading waveletcoeffs/<name>.npy and
 * waveletstrength/<name>.npy (EnvironmentMap.cpp:97-108) + buildLights' upload
 * (RenderEngine.cpp:162-175). */
NWPRT_API nwprt_status nwprt_env_from_faces(nwprt_ctx* ctx, const float* faces, int faces_on_device, int S,
                                  int K, void* stream, int* env_id);
/* Registers a precomputed wavelet table: idx int32[K], strength float[K][3]
 * (the npy pair of EnvironmentMap.cpp:97-108). */
NWPRT_API nwprt_status nwprt_env_from_wavelets(nwprt_ctx* ctx, const int32_t* idx, const float* strength,
                                     int K, int on_device, void* stream, int* env_id);
/* Copies an env's table to host (synchronous) -- Environment_Map::topWaveletCoefficients /
 * topWaveletStrength (EnvironmentMap.h:24-25).  `capacity` = entries available. */
NWPRT_API nwprt_status nwprt_env_get_wavelets(nwprt_ctx* ctx, int env_id, int32_t* idx_host,
                                    float* strength_host, int capacity, int* K);
/* Frees the env id.  Its device buffers stay with the context and are reused, in stream
 * order, by a later registration of K or fewer wavelets -- work already queued that still
 * reads the env must be on the same stream as that later registration. */
NWPRT_API nwprt_status nwprt_env_release(nwprt_ctx* ctx, int env_id);

/* ---------------------------------------------------------------- frames */
/* Pass 1: registers the frame's G-buffer and packs the per-pixel 16-float input row
 * (no K-fold replication).  Replaces RenderEngine::TCNNPass_p1 (tinycudann/tcnn.cu:83-108)
 * and prt::waveletDataCopy (utils_kernels.h:7-49).  Asynchronous on `stream`.  The
 * G-buffer memory must stay valid until the frame's relights have run. */
NWPRT_API nwprt_status nwprt_prepare(nwprt_ctx* ctx, int frame_id, const nwprt_gbuffer* gbuffer,
                           void* stream);
/* Pass 2: evaluates the transport of every pixel for the env's K wavelets and reduces
 * sum_k T_k * L_k straight into `indirect` and `with_direct` (float4 per pixel; the
 * N x K transport never reaches memory).  Replaces RenderEngine::TCNNPass_p2
 * (tinycudann/tcnn.cu:111-152), PRT_Network::inference (prt_network.h:73-154) and
 * prt::computeResponse (utils_kernels.h:52-91).  Asynchronous: unlike the reference it
 * does not block the host.  `opts` NULL = {FP32, clamp, kahan}.  BF16/FP8 relights may be
 * captured into a CUDA graph: each captured launch keeps one of the context's 64 tile
 * counters for good (a further capture fails with NWPRT_UNSUPPORTED). */
NWPRT_API nwprt_status nwprt_relight(nwprt_ctx* ctx, int env_id, int frame_id,
                           const nwprt_relight_opts* opts, float* indirect, float* with_direct,
                           void* stream);
/* Many relights in one device pass (cross-request batching for serving). */
NWPRT_API nwprt_status nwprt_relight_batch(nwprt_ctx* ctx, const nwprt_request* reqs, int n_reqs,
                                 const nwprt_relight_opts* opts, void* stream);
/* Pixel-range relights, all in one device pass for NWPRT_PREC_BF16 / NWPRT_PREC_FP8 (one
 * launch per range for NWPRT_PREC_FP32).  Ranges of one frame/output may not overlap
 * within a call. */
NWPRT_API nwprt_status nwprt_relight_ranges(nwprt_ctx* ctx, const nwprt_range_request* reqs, int n_reqs,
                                            const nwprt_relight_opts* opts, void* stream);
/* FP8 calibration (no reference counterpart: the reference runs tcnn's FP16 network,
 * prt_network.h:53-60).  Relights pixels [px_begin, px_end) of a prepared frame (px_end
 * <= 0: to the end of the frame) with env `env_id` in BF16, records the maximum activation
 * entering every tensor-core layer, and builds the FP8 weights and per-layer scales from
 * them.  The scales then stay fixed for every NWPRT_PREC_FP8 relight until the next
 * calibration or weight load, so a result does not depend on what it is batched with.
 * Blocks on `stream`, then on the device before it replaces a previous FP8 blob. */
NWPRT_API nwprt_status nwprt_calibrate_fp8(nwprt_ctx* ctx, int env_id, int frame_id, int64_t px_begin,
                                           int64_t px_end, void* stream);
/* The calibrated maxima: one per tensor-core layer input, then the input of the 3-wide
 * output layer.  Writes min(capacity, n) values and sets *n_values = n. */
NWPRT_API nwprt_status nwprt_get_fp8_calibration(const nwprt_ctx* ctx, float* amax, int capacity,
                                                 int* n_values);
/* Diagnostics (no counterpart in the reference): launches one warp that waits, through the
 * bounded wait every persistent kernel of this library uses, on a barrier that nothing ever
 * signals.  The wait gives up after timeout_ms (1..2000) and records a timeout, so the next
 * nwprt_sync returns NWPRT_TIMEOUT and clears it; the context stays usable.  It shows that a
 * device wait that cannot finish surfaces as a status instead of a hang. */
NWPRT_API nwprt_status nwprt_selftest_device_wait(nwprt_ctx* ctx, int timeout_ms, void* stream);
/* Blocks until all work the context issued has finished -- RenderEngine::TCNNSync
 * (tinycudann/tcnn.cu:154-158). */
NWPRT_API nwprt_status nwprt_sync(nwprt_ctx* ctx);

/* ---------------------------------------------------------------- kernels without a context */
/* Haar + top-K of `n_env` cubemaps [n_env][6][S][S][3] -> idx[n_env][K], strength[n_env][K][3].
 * S a power of two <= 64 (larger faces: NWPRT_UNSUPPORTED), 1 <= K <= min(6*S*S, 1024).  Order: |luminance| descending,
 * flat index face*S*S + row*S + col ascending. */
NWPRT_API nwprt_status nwprt_haar_topk(const float* faces, int n_env, int S, int K, int32_t* idx,
                             float* strength, void* stream);
/* Rotated copy of a cubemap: dst(d) = src(R^T d) for every texel direction d, sampled as
 * the reference samples its env cubemaps (point filtering, wrap addressing;
 * device_functions/cubeMap.cu:23-113, Renderer/textures.h:64-68).  R: 9 floats, row-major,
 * host memory.  src and dst are device buffers of [6][S][S][3] floats and must differ.
 * Feeds rotated env maps to nwprt_env_from_faces (the reference precomputes such
 * rotations offline, README "EnvmapRotation" sets). */
NWPRT_API nwprt_status nwprt_env_rotate(const float* src, int S, const float* R, float* dst, void* stream);
/* Final colour of a relit frame -- RenderEngine::computeFinalPixelColors
 * (Renderer/toneMap.cu:47-98) on fbPredictedIndirectWithDirect or fbPredictedIndirect:
 * per channel 1.055 (x + 1e-6)^(1/2.4) - 0.055, clamped to [0, 1], times 255.9, truncated;
 * packed r | g << 8 | b << 16 | 255 << 24.  src: n_px float4 (16-byte aligned), dst: n_px
 * uint32, both device memory. */
NWPRT_API nwprt_status nwprt_tonemap_srgb(const float* src, int64_t n_px, uint32_t* dst, void* stream);
/* SH shading of mesh vertices -- the SH path's closest-hit program without the ray tracer
 * (Renderer/device_functions/devicePrograms.cu:427-486): for every vertex v,
 *   light[k] = sum_j T[v][k][j] L[j]  (j ascending),  out[v] = | sum_k light[k] * brdf[v][k] |
 * per RGB channel (k ascending).  T: [V][n][n] transfer matrices (the reference's T_matrix,
 * RenderEngine.cpp:410-448), brdf_sh: [V][n][3] the BRDF projected on the SH basis (sampled
 * from the material in the reference, devicePrograms.cu:448-474), L: [n][3] env SH,
 * out: [V][3]; n = (degree + 1)^2 <= 81.  All device memory. */
NWPRT_API nwprt_status nwprt_sh_vertex_radiance(const float* T, const float* brdf_sh, const float* L,
                                                int64_t n_vertices, int n_coeffs, float* out, void* stream);
/* Pixel colours from their triangle's vertex colours (devicePrograms.cu:488-490):
 * out[p] = ((1 - u - v) c[i0] + u c[i1] + v c[i2], 1), evaluated as
 * fma(v, c2, fma(u, c1, (1 - u - v) c0)).  tri: [P][3] int32 vertex indices, uv: [P][2]
 * barycentrics, out: [P] float4 (16-byte aligned).  An index outside [0, n_vertices) yields
 * (0, 0, 0, 1) and is reported by nwprt_sync. */
NWPRT_API nwprt_status nwprt_sh_interpolate(nwprt_ctx* ctx, const float* vertex_rgb, int64_t n_vertices,
                                            const int32_t* tri, const float* uv, int64_t n_px, float* out,
                                            void* stream);
/* SH projection (order 8, 81 coefficients) of a cubemap [6][S][S][3] -> L[81][3]
 * (the env SH the reference loads from sh/<name>.npy, EnvironmentMap.cpp:70-77).
 * `workspace` must hold nwprt_sh_project_workspace_size(S) bytes of device memory. */
NWPRT_API size_t nwprt_sh_project_workspace_size(int S);
NWPRT_API nwprt_status nwprt_sh_project(const float* faces, int S, float* L, void* workspace,
                              size_t workspace_bytes, void* stream);
/* nwprt_sh_project without a workspace, for callers that cannot allocate device memory
 * (a frame loop that must never reach cudaMalloc/cudaFree, which can synchronise the device,
 * or a host that reserves all device memory up front).  No counterpart in the reference.
 * The partial sums live in a fixed static device array (373,248 bytes, held by every GPU
 * that loads the library until exit), so S must be <= 128.  The first call on a device
 * looks up that array's address with the device current; make it before any stream
 * capture, and do not call cudaDeviceReset afterwards in the same process (the cached
 * address would be stale).  Each device has its own array: calls that overlap on the same
 * device (e.g. on two streams) race and must be serialised by the caller; calls on
 * different devices do not race. */
NWPRT_API nwprt_status nwprt_sh_project_static(const float* faces, int S, float* L, void* stream);
/* Per-pixel SH dot product out[p] = (|sum_j T[p][j] L[j]|, 1) (float4 per pixel) -- the
 * light-vector product of __closesthit__SHradiance (device_functions/devicePrograms.cu:479-490)
 * for per-pixel transport vectors.  abs_out = 0 drops the abs of :490. */
NWPRT_API nwprt_status nwprt_sh_dot(const float* T, int64_t n_px, int n_coeffs, const float* L,
                          int abs_out, float* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* NWPRT_H */

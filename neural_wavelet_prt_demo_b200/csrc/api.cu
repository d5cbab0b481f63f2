// libnwprt C ABI: context, weights, env-map registry, frames and dispatch.
//
// Mirrors the reference's engine entry points (Renderer/RenderEngine.h:78-83,
// Renderer/tinycudann/tcnn.cu:49-162) behind status codes: nothing throws across the
// boundary, every failure leaves a message in nwprt_last_error().
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>

#include "nwprt_internal.cuh"

#include <nvtx3/nvToolsExt.h>

using namespace nwprt;

namespace {

thread_local std::string g_last_error;

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (dev < 0) return;
    NWPRT_CUDA(cudaGetDevice(&prev));
    if (prev != dev) NWPRT_CUDA(cudaSetDevice(dev));
    else prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

template <class T>
T* dev_alloc(size_t n) {
  if (n == 0) n = 1;
  void* p = nullptr;
  NWPRT_CUDA(cudaMalloc(&p, n * sizeof(T)));
  return static_cast<T*>(p);
}

void dev_free(void* p) {
  if (p) cudaFree(p);
}

struct EnvEntry {
  bool live = false;
  int K = 0;
  int cap = 0;                // wavelets the buffers below can hold (kept across reuse)
  int32_t* idx = nullptr;
  float* strength = nullptr;
  float* emb_k = nullptr;     // [K][D], valid when emb_ready; then [cap][D/2] BF16 pairs
  bool emb_ready = false;
  bool owned = false;         // buffers of its own (else carved from a chunk of slots)
};

// The BF16 pairs of an env's embedding rows, stored after the FP32 rows.
const uint32_t* emb_pairs(const EnvEntry& e, int D) {
  return reinterpret_cast<const uint32_t*>(e.emb_k + (size_t)e.cap * D);
}

void free_env_buffers(EnvEntry& e) {
  if (e.owned) {
    dev_free(e.idx);
    dev_free(e.strength);
    dev_free(e.emb_k);
  }
  e = EnvEntry{};
}

struct Frame {
  bool prepared = false;
  int width = 0, height = 0;
  float* packed = nullptr;
  size_t cap_px = 0;
  const uint8_t* flag = nullptr;
  const float* direct = nullptr;
};

}  // namespace

struct nwprt_ctx {
  int device = 0;
  NetDims dims;
  HashLevels hl{};
  std::string last_error;
  bool weights_loaded = false;
  float* d_hash = nullptr;
  float* d_emb = nullptr;
  float* d_w32 = nullptr;
  size_t op_t_floats = 0, cn_t_floats = 0;
  uint16_t* d_tc_w = nullptr;
  bool tc_supported = false;
  std::string tc_why;
  // FP8: host copies of the MLP weights (the blob is rebuilt at every calibration), the
  // calibrated per-layer activation maxima and the plan/blob built from them
  std::vector<float> h_op, h_cn;
  uint8_t* d_tc_w8 = nullptr;
  TcPlan fp8_plan{};
  TcPlan bf16_plan{};
  bool fp8_ready = false;
  std::vector<float> fp8_amax;
  std::vector<EnvEntry> envs;
  std::vector<void*> env_chunks;  // device memory the pooled env slots are carved from
  Frame frames[NWPRT_MAX_FRAMES];
  uint32_t* d_err = nullptr;
  // Tile counters of the tensor-core relight (its warpgroups take tiles from one counter per
  // launch): a ring for eager launches, so that launches in flight on different streams use
  // different counters, and one counter of its own for each launch captured into a CUDA graph
  // (a graph replays its counter, so no later launch may be handed it).
  static constexpr int kTileCounters = 64, kCapturedCounters = 64;
  int* d_tile_ctr = nullptr;
  int tile_ctr_next = 0, captured_next = 0;
  float* d_stage = nullptr;
  size_t stage_cap = 0;

  ~nwprt_ctx() {
    DeviceGuard g(device);
    cudaDeviceSynchronize();
    dev_free(d_hash);
    dev_free(d_emb);
    dev_free(d_w32);
    dev_free(d_tc_w);
    dev_free(d_tc_w8);
    dev_free(d_err);
    dev_free(d_tile_ctr);
    dev_free(d_stage);
    for (auto& e : envs) free_env_buffers(e);
    for (void* c : env_chunks) dev_free(c);
    for (auto& f : frames) dev_free(f.packed);
  }
};

namespace {

void set_error(const nwprt_ctx* ctx, const std::string& m) {
  g_last_error = m;
  if (ctx) const_cast<nwprt_ctx*>(ctx)->last_error = m;
}

// NVTX range around an entry point (header-only NVTX3: a no-op unless a profiler is attached).
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

template <class F>
nwprt_status guarded(const nwprt_ctx* ctx, F&& f) {
  try {
    DeviceGuard g(ctx ? ctx->device : -1);
    f();
    return NWPRT_OK;
  } catch (const Error& e) {
    set_error(ctx, e.what());
    return e.status;
  } catch (const std::bad_alloc&) {
    set_error(ctx, "host out of memory");
    return NWPRT_OOM;
  } catch (const std::exception& e) {
    set_error(ctx, e.what());
    return NWPRT_CUDA_ERROR;
  }
}

void need(bool cond, nwprt_status s, const char* msg) {
  if (!cond) fail(s, msg);
}

HashLevels make_levels(const NetDims& d) {
  HashLevels h{};
  h.n_levels = d.n_levels;
  h.n_features = d.n_features;
  h.dense_mask = 0;
  for (int l = 0; l < d.n_levels; ++l) {
    h.res[l] = d.level_res[l];
    h.size[l] = (uint32_t)d.level_size[l];
    h.offset[l] = (uint32_t)d.level_offset[l];
    const uint64_t n1 = (uint64_t)d.level_res[l] + 1;
    if (n1 * n1 * n1 <= (uint64_t)d.level_size[l]) h.dense_mask |= 1u << l;
  }
  return h;
}

EnvEntry& env_at(nwprt_ctx* ctx, int id) {
  need(id >= 0 && id < (int)ctx->envs.size() && ctx->envs[id].live, NWPRT_INVALID_ARG,
       "unknown env id");
  return ctx->envs[id];
}

void ensure_emb(nwprt_ctx* ctx, EnvEntry& e, cudaStream_t st) {
  if (e.emb_ready) return;
  need(ctx->weights_loaded, NWPRT_NOT_READY, "weights are not loaded");
  const int D = ctx->dims.enc_dims();
  launch_gather_embedding(ctx->d_emb, D, ctx->dims.n_coeffs(), e.idx, e.K, e.emb_k,
                          const_cast<uint32_t*>(emb_pairs(e, D)), ctx->d_err, st);
  e.emb_ready = true;
}

// Registers an env slot for K wavelets.  Released slots are reused in stream order without
// any allocation or synchronisation: a pooled slot holds kEnvSlotWavelets wavelets (~200 KB at
// 32 hash features), so any released slot fits any K the Haar path produces.  Pooled slots come
// kEnvChunkSlots at a time from one allocation, since a serving loop's live set can grow to
// hundreds of env maps and each cudaMalloc costs milliseconds of host time.  A larger K gets a
// slot with buffers of its own.  Slots are freed with the context.  (Replacing a smaller slot
// would need a device-wide synchronisation before its buffers could be freed, which drains a
// serving loop's queue of launches.)
constexpr int kEnvSlotWavelets = 1024;
constexpr int kEnvChunkSlots = 64;

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int new_env(nwprt_ctx* ctx, int K, int D) {
  int id = -1;
  for (size_t i = 0; i < ctx->envs.size(); ++i) {
    const EnvEntry& e = ctx->envs[i];
    if (e.live || e.cap < K) continue;
    if (id < 0 || e.cap < ctx->envs[id].cap) id = (int)i;
  }
  if (id < 0 && K <= kEnvSlotWavelets) {
    const size_t cap = kEnvSlotWavelets;
    const size_t b_idx = align256(cap * 4), b_st = align256(cap * 12), b_emb = align256(cap * (D + D / 2) * 4);
    const size_t per = b_idx + b_st + b_emb;
    uint8_t* base = dev_alloc<uint8_t>(per * kEnvChunkSlots);
    ctx->env_chunks.push_back(base);
    id = (int)ctx->envs.size();
    for (int j = 0; j < kEnvChunkSlots; ++j) {
      EnvEntry e;
      uint8_t* p = base + per * j;
      e.idx = reinterpret_cast<int32_t*>(p);
      e.strength = reinterpret_cast<float*>(p + b_idx);
      e.emb_k = reinterpret_cast<float*>(p + b_idx + b_st);
      e.cap = (int)cap;
      ctx->envs.push_back(e);
    }
  } else if (id < 0) {
    EnvEntry e;
    e.owned = true;
    try {
      e.idx = dev_alloc<int32_t>(K);
      e.strength = dev_alloc<float>((size_t)K * 3);
      e.emb_k = dev_alloc<float>((size_t)K * D + (size_t)K * (D / 2));
    } catch (...) {
      free_env_buffers(e);
      throw;
    }
    e.cap = K;
    ctx->envs.push_back(e);
    id = (int)ctx->envs.size() - 1;
  }
  EnvEntry& e = ctx->envs[id];
  e.K = K;
  e.emb_ready = false;
  e.live = true;
  return id;
}

void release_env(EnvEntry& e) {
  e.live = false;
  e.emb_ready = false;
}

nwprt_relight_opts default_opts() {
  nwprt_relight_opts o;
  o.precision = NWPRT_PREC_FP32;
  o.clamp_terms = 1;
  o.kahan = 1;
  return o;
}

void check_out(const float* p, const char* what) {
  need(p != nullptr, NWPRT_INVALID_ARG, what);
  need(((uintptr_t)p & 15) == 0, NWPRT_INVALID_ARG, "output buffers must be 16-byte aligned (float4)");
}

}  // namespace

namespace nwprt {
// Records a message for nwprt_last_error(NULL) from entry points defined in other files.
void set_thread_error(const std::string& m) { g_last_error = m; }
}  // namespace nwprt

extern "C" {

int nwprt_abi_version(void) { return NWPRT_ABI_VERSION; }

const char* nwprt_status_string(nwprt_status s) {
  switch (s) {
    case NWPRT_OK: return "ok";
    case NWPRT_INVALID_ARG: return "invalid argument";
    case NWPRT_OOM: return "out of memory";
    case NWPRT_CUDA_ERROR: return "CUDA error";
    case NWPRT_TIMEOUT: return "device wait timed out";
    case NWPRT_NOT_READY: return "not ready";
    case NWPRT_IO_ERROR: return "I/O error";
    case NWPRT_UNSUPPORTED: return "unsupported";
  }
  return "unknown status";
}

const char* nwprt_last_error(const nwprt_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : g_last_error.c_str();
}

nwprt_status nwprt_create(const char* config_json, int device, nwprt_ctx** out) {
  if (out) *out = nullptr;
  return guarded(nullptr, [&] {
    need(config_json && out, NWPRT_INVALID_ARG, "nwprt_create: null argument");
    NetDims d = parse_config(config_json);
    int n_dev = 0;
    NWPRT_CUDA(cudaGetDeviceCount(&n_dev));
    need(device >= 0 && device < n_dev, NWPRT_INVALID_ARG, "nwprt_create: no such device");
    DeviceGuard g(device);
    std::unique_ptr<nwprt_ctx> c(new nwprt_ctx());
    c->device = device;
    c->dims = d;
    c->hl = make_levels(d);
    c->tc_supported = relight_tc_supported(d, &c->tc_why);
    c->d_err = dev_alloc<uint32_t>(1);
    NWPRT_CUDA(cudaMemset(c->d_err, 0, sizeof(uint32_t)));
    c->d_tile_ctr = dev_alloc<int>(nwprt_ctx::kTileCounters + nwprt_ctx::kCapturedCounters);
    *out = c.release();
  });
}

void nwprt_destroy(nwprt_ctx* ctx) {
  try {
    delete ctx;
  } catch (...) {
  }
}

nwprt_status nwprt_get_network_info(const nwprt_ctx* ctx, nwprt_network_info* info) {
  return guarded(ctx, [&] {
    need(ctx && info, NWPRT_INVALID_ARG, "null argument");
    const NetDims& d = ctx->dims;
    info->enc_dims = d.enc_dims();
    info->n_coeffs = d.n_coeffs();
    info->face_size = d.face_size;
    info->aux_width = d.aux_width;
    info->n_hash_params = d.n_hash_params();
    info->n_out_prd = d.n_op_params();
    info->n_cmp_net = d.n_cn_params();
    info->n_wve_enc = (size_t)d.enc_dims() * d.n_coeffs();
    info->flops_per_eval = d.flops_per_eval();
  });
}

nwprt_status nwprt_load_weights(nwprt_ctx* ctx, const nwprt_weights* w) {
  return guarded(ctx, [&] {
    TraceRange trace("nwprt_load_weights");
    need(ctx && w, NWPRT_INVALID_ARG, "null argument");
    const NetDims& d = ctx->dims;
    need(w->hash_params && w->out_prd && w->cmp_net && w->wve_enc, NWPRT_INVALID_ARG,
         "null weight pointer");
    if (w->n_hash_params != d.n_hash_params() || w->n_out_prd != d.n_op_params() ||
        w->n_cmp_net != d.n_cn_params() || w->n_wve_enc != (size_t)d.enc_dims() * d.n_coeffs()) {
      std::ostringstream m;
      m << "weight sizes do not match the config: expected hash " << d.n_hash_params() << ", out_prd "
        << d.n_op_params() << ", cmp_net " << d.n_cn_params() << ", wve_enc "
        << (size_t)d.enc_dims() * d.n_coeffs() << "; got " << w->n_hash_params << ", " << w->n_out_prd
        << ", " << w->n_cmp_net << ", " << w->n_wve_enc;
      fail(NWPRT_INVALID_ARG, m.str());
    }
    NWPRT_CUDA(cudaDeviceSynchronize());
    dev_free(ctx->d_hash);
    dev_free(ctx->d_emb);
    dev_free(ctx->d_w32);
    dev_free(ctx->d_tc_w);
    dev_free(ctx->d_tc_w8);
    ctx->d_hash = ctx->d_emb = ctx->d_w32 = nullptr;
    ctx->d_tc_w = nullptr;
    ctx->d_tc_w8 = nullptr;
    ctx->fp8_ready = false;
    ctx->fp8_amax.clear();
    ctx->weights_loaded = false;
    ctx->d_hash = dev_alloc<float>(w->n_hash_params);
    NWPRT_CUDA(cudaMemcpy(ctx->d_hash, w->hash_params, w->n_hash_params * 4, cudaMemcpyHostToDevice));
    ctx->d_emb = dev_alloc<float>(w->n_wve_enc);
    NWPRT_CUDA(cudaMemcpy(ctx->d_emb, w->wve_enc, w->n_wve_enc * 4, cudaMemcpyHostToDevice));
    std::vector<float> op_t, cn_t;
    pack_fp32_weights(d, w->out_prd, w->cmp_net, &op_t, &cn_t);
    ctx->op_t_floats = op_t.size();
    ctx->cn_t_floats = cn_t.size();
    ctx->d_w32 = dev_alloc<float>(op_t.size() + cn_t.size());
    NWPRT_CUDA(cudaMemcpy(ctx->d_w32, op_t.data(), op_t.size() * 4, cudaMemcpyHostToDevice));
    NWPRT_CUDA(cudaMemcpy(ctx->d_w32 + op_t.size(), cn_t.data(), cn_t.size() * 4, cudaMemcpyHostToDevice));
    ctx->h_op.assign(w->out_prd, w->out_prd + w->n_out_prd);
    ctx->h_cn.assign(w->cmp_net, w->cmp_net + w->n_cmp_net);
    if (ctx->tc_supported) {
      std::vector<uint16_t> tw;
      ctx->bf16_plan = pack_tc_weights(d, w->out_prd, w->cmp_net, &tw);
      tw.resize(tc_blob_alloc_bytes(tw.size() * 2) / 2, 0);  // whole rows of the kernel's TMA view
      ctx->d_tc_w = dev_alloc<uint16_t>(tw.size());
      NWPRT_CUDA(cudaMemcpy(ctx->d_tc_w, tw.data(), tw.size() * 2, cudaMemcpyHostToDevice));
    }
    for (auto& e : ctx->envs) e.emb_ready = false;
    ctx->weights_loaded = true;
  });
}

nwprt_status nwprt_load_weights_dir(nwprt_ctx* ctx, const char* dir) {
  return guarded(ctx, [&] {
    need(ctx && dir, NWPRT_INVALID_ARG, "null argument");
    std::string base(dir);
    if (!base.empty() && base.back() != '/') base += '/';
    NpyArray hp = read_npy(base + "vtx_enc.npy");
    NpyArray op = read_npy(base + "out_prd.npy");
    NpyArray cn = read_npy(base + "cmp_net.npy");
    NpyArray we = read_npy(base + "wve_enc.npy");
    for (NpyArray* a : {&hp, &op, &cn, &we})
      need(a->descr == "<f4", NWPRT_IO_ERROR, "weight files must be float32 (<f4)");
    nwprt_weights w;
    w.hash_params = (const float*)hp.data.data();
    w.n_hash_params = hp.data.size() / 4;
    w.out_prd = (const float*)op.data.data();
    w.n_out_prd = op.data.size() / 4;
    w.cmp_net = (const float*)cn.data.data();
    w.n_cmp_net = cn.data.size() / 4;
    w.wve_enc = (const float*)we.data.data();
    w.n_wve_enc = we.data.size() / 4;
    nwprt_status s = nwprt_load_weights(ctx, &w);
    if (s != NWPRT_OK) fail(s, ctx->last_error);
  });
}

int nwprt_ready(const nwprt_ctx* ctx) {
  if (!ctx || !ctx->weights_loaded) return 0;
  for (const auto& e : ctx->envs)
    if (e.live) return 1;
  return 0;
}

nwprt_status nwprt_env_from_faces(nwprt_ctx* ctx, const float* faces, int on_device, int S, int K,
                                  void* stream, int* env_id) {
  return guarded(ctx, [&] {
    TraceRange trace("nwprt_env_from_faces");
    need(ctx && faces && env_id, NWPRT_INVALID_ARG, "null argument");
    need(S == ctx->dims.face_size, NWPRT_INVALID_ARG,
         "cubemap face size must equal the network's wve_enc.face_size");
    need(K >= 1 && K <= 6 * S * S && K <= 1024, NWPRT_INVALID_ARG, "K must be in [1, min(6*S*S, 1024)]");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)6 * S * S * 3;
    const float* src = faces;
    if (!on_device) {
      if (ctx->stage_cap < n) {
        NWPRT_CUDA(cudaStreamSynchronize(st));
        dev_free(ctx->d_stage);
        ctx->d_stage = nullptr;
        ctx->d_stage = dev_alloc<float>(n);
        ctx->stage_cap = n;
      }
      NWPRT_CUDA(cudaMemcpyAsync(ctx->d_stage, faces, n * 4, cudaMemcpyHostToDevice, st));
      src = ctx->d_stage;
    }
    const int id = new_env(ctx, K, ctx->dims.enc_dims());
    EnvEntry& e = ctx->envs[id];
    try {
      launch_haar_topk(src, 1, S, K, e.idx, e.strength, ctx->d_err, st);
      if (ctx->weights_loaded) ensure_emb(ctx, e, st);
    } catch (...) {
      release_env(e);
      throw;
    }
    if (!on_device) NWPRT_CUDA(cudaStreamSynchronize(st));  // staging buffer reuse
    *env_id = id;
  });
}

nwprt_status nwprt_env_from_wavelets(nwprt_ctx* ctx, const int32_t* idx, const float* strength,
                                     int K, int on_device, void* stream, int* env_id) {
  return guarded(ctx, [&] {
    TraceRange trace("nwprt_env_from_wavelets");
    need(ctx && idx && strength && env_id, NWPRT_INVALID_ARG, "null argument");
    need(K >= 1 && K <= (1 << 20), NWPRT_INVALID_ARG, "K out of range");
    cudaStream_t st = (cudaStream_t)stream;
    const int nc = ctx->dims.n_coeffs();
    if (!on_device)
      for (int k = 0; k < K; ++k)
        need(idx[k] >= 0 && idx[k] < nc, NWPRT_INVALID_ARG, "wavelet index outside [0, 6*S*S)");
    const int id = new_env(ctx, K, ctx->dims.enc_dims());
    EnvEntry& e = ctx->envs[id];
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    NWPRT_CUDA(cudaMemcpyAsync(e.idx, idx, (size_t)K * 4, kind, st));
    NWPRT_CUDA(cudaMemcpyAsync(e.strength, strength, (size_t)K * 12, kind, st));
    if (ctx->weights_loaded) ensure_emb(ctx, e, st);
    if (!on_device) NWPRT_CUDA(cudaStreamSynchronize(st));
    *env_id = id;
  });
}

nwprt_status nwprt_env_get_wavelets(nwprt_ctx* ctx, int env_id, int32_t* idx_host,
                                    float* strength_host, int capacity, int* K) {
  return guarded(ctx, [&] {
    need(ctx && K, NWPRT_INVALID_ARG, "null argument");
    EnvEntry& e = env_at(ctx, env_id);
    *K = e.K;
    if (!idx_host && !strength_host) return;
    need(capacity >= e.K, NWPRT_INVALID_ARG, "capacity smaller than K");
    NWPRT_CUDA(cudaDeviceSynchronize());
    if (idx_host) NWPRT_CUDA(cudaMemcpy(idx_host, e.idx, (size_t)e.K * 4, cudaMemcpyDeviceToHost));
    if (strength_host)
      NWPRT_CUDA(cudaMemcpy(strength_host, e.strength, (size_t)e.K * 12, cudaMemcpyDeviceToHost));
  });
}

nwprt_status nwprt_env_release(nwprt_ctx* ctx, int env_id) {
  return guarded(ctx, [&] {
    need(ctx != nullptr, NWPRT_INVALID_ARG, "null argument");
    EnvEntry& e = env_at(ctx, env_id);
    release_env(e);
  });
}

nwprt_status nwprt_prepare(nwprt_ctx* ctx, int frame_id, const nwprt_gbuffer* g, void* stream) {
  return guarded(ctx, [&] {
    TraceRange trace("nwprt_prepare");
    need(ctx && g, NWPRT_INVALID_ARG, "null argument");
    need(frame_id >= 0 && frame_id < NWPRT_MAX_FRAMES, NWPRT_INVALID_ARG, "frame id out of range");
    need(g->width >= 0 && g->height >= 0 && (int64_t)g->width * g->height <= (1LL << 31),
         NWPRT_INVALID_ARG, "frame size out of range");
    const size_t n = (size_t)g->width * g->height;
    if (n > 0) {
      need(g->first_hit_pos && g->world_normal && g->reflect_dir && g->roughness && g->kd && g->ks &&
               g->direct && g->env_map_flag,
           NWPRT_INVALID_ARG, "null G-buffer pointer");
      for (const float* p : {g->first_hit_pos, g->world_normal, g->reflect_dir, g->kd, g->ks, g->direct})
        need(((uintptr_t)p & 15) == 0, NWPRT_INVALID_ARG, "float4 G-buffers must be 16-byte aligned");
    }
    Frame& f = ctx->frames[frame_id];
    if (f.cap_px < n) {
      // resize like TCNNPass_p1's GPUMatrix reallocation (tcnn.cu:88-97)
      NWPRT_CUDA(cudaDeviceSynchronize());
      dev_free(f.packed);
      f.packed = nullptr;
      f.packed = dev_alloc<float>(n * 16);
      f.cap_px = n;
    }
    f.width = g->width;
    f.height = g->height;
    f.flag = g->env_map_flag;
    f.direct = g->direct;
    launch_pack_gbuffer(*g, f.packed, (cudaStream_t)stream);
    f.prepared = true;
  });
}

// A relight of pixels [px_begin, px_end) of a prepared frame (px_end <= 0: whole frame).
struct RangeReq {
  int env_id, frame_id;
  float* indirect;
  float* with_direct;
  int64_t px_begin, px_end;
};

static int64_t resolve_range(nwprt_ctx* ctx, RangeReq& r) {
  need(r.frame_id >= 0 && r.frame_id < NWPRT_MAX_FRAMES, NWPRT_INVALID_ARG, "frame id out of range");
  Frame& f = ctx->frames[r.frame_id];
  need(f.prepared, NWPRT_NOT_READY, "frame was not prepared (call nwprt_prepare first)");
  const int64_t n = (int64_t)f.width * f.height;
  if (r.px_end <= 0) r.px_end = n;
  need(r.px_begin >= 0 && r.px_begin <= r.px_end && r.px_end <= n, NWPRT_INVALID_ARG,
       "pixel range outside the frame");
  check_out(r.indirect, "null indirect output");
  check_out(r.with_direct, "null with_direct output");
  return n;
}

static void relight_one(nwprt_ctx* ctx, RangeReq r, const nwprt_relight_opts& o, cudaStream_t st) {
  need(ctx->weights_loaded, NWPRT_NOT_READY, "weights are not loaded");
  EnvEntry& e = env_at(ctx, r.env_id);
  resolve_range(ctx, r);
  Frame& f = ctx->frames[r.frame_id];
  ensure_emb(ctx, e, st);
  if (o.precision == NWPRT_PREC_FP32) {
    RelightJob j{f.packed, f.flag, f.direct, e.emb_k, e.strength, e.K, r.px_end, r.indirect, r.with_direct,
                 r.px_begin};
    DeviceWeights w{ctx->d_hash, ctx->d_w32, ctx->d_w32 + ctx->op_t_floats, ctx->op_t_floats, ctx->cn_t_floats};
    launch_relight_fp32(ctx->dims, ctx->hl, w, j, o.clamp_terms, o.kahan, st);
  } else {
    fail(NWPRT_INVALID_ARG, "unknown precision");
  }
}

static void relight_many_tc(nwprt_ctx* ctx, const RangeReq* reqs, int n_reqs, const nwprt_relight_opts& o,
                            int mode, uint32_t* amax, cudaStream_t st) {
  need(ctx->weights_loaded, NWPRT_NOT_READY, "weights are not loaded");
  need(ctx->tc_supported, NWPRT_UNSUPPORTED, ctx->tc_why.c_str());
  if (mode == kTcFp8)
    need(ctx->fp8_ready, NWPRT_NOT_READY, "FP8 scales are not calibrated (call nwprt_calibrate_fp8 first)");
  std::vector<TcJob> jobs;
  jobs.reserve(n_reqs);
  for (int i = 0; i < n_reqs; ++i) {
    RangeReq r = reqs[i];
    EnvEntry& e = env_at(ctx, r.env_id);
    resolve_range(ctx, r);
    Frame& f = ctx->frames[r.frame_id];
    ensure_emb(ctx, e, st);
    if (r.px_end == r.px_begin) continue;
    jobs.push_back(TcJob{f.packed, f.flag, f.direct, e.emb_k, e.strength, e.K, r.px_end, r.indirect, r.with_direct,
                         0, r.px_begin, emb_pairs(e, ctx->dims.enc_dims())});
  }
  if (jobs.empty()) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  NWPRT_CUDA(cudaStreamIsCapturing(st, &cs));
  int* ctr;
  if (cs == cudaStreamCaptureStatusActive) {
    need(ctx->captured_next < nwprt_ctx::kCapturedCounters, NWPRT_UNSUPPORTED,
         "too many tensor-core relights captured into CUDA graphs for one context (64)");
    ctr = ctx->d_tile_ctr + nwprt_ctx::kTileCounters + ctx->captured_next++;
  } else {
    ctr = ctx->d_tile_ctr + ctx->tile_ctr_next;
    ctx->tile_ctr_next = (ctx->tile_ctr_next + 1) % nwprt_ctx::kTileCounters;
  }
  if (mode == kTcFp8)
    launch_relight_tc(ctx->dims, ctx->hl, ctx->d_hash, ctx->d_tc_w8, &ctx->fp8_plan, mode, jobs.data(),
                      (int)jobs.size(), o.kahan, o.clamp_terms, nullptr, ctx->d_err, ctr, st);
  else
    launch_relight_tc(ctx->dims, ctx->hl, ctx->d_hash, ctx->d_tc_w, &ctx->bf16_plan, mode, jobs.data(),
                      (int)jobs.size(), o.kahan, o.clamp_terms, amax, ctx->d_err, ctr, st);
}

static void relight_ranges(nwprt_ctx* ctx, const std::vector<RangeReq>& reqs, const nwprt_relight_opts& o,
                           cudaStream_t st) {
  if (o.precision == NWPRT_PREC_BF16) {
    relight_many_tc(ctx, reqs.data(), (int)reqs.size(), o, kTcBf16, nullptr, st);
  } else if (o.precision == NWPRT_PREC_FP8) {
    relight_many_tc(ctx, reqs.data(), (int)reqs.size(), o, kTcFp8, nullptr, st);
  } else {
    for (const RangeReq& r : reqs) relight_one(ctx, r, o, st);
  }
}

nwprt_status nwprt_relight(nwprt_ctx* ctx, int env_id, int frame_id, const nwprt_relight_opts* opts,
                           float* indirect, float* with_direct, void* stream) {
  return guarded(ctx, [&] {
    TraceRange trace("nwprt_relight");
    need(ctx != nullptr, NWPRT_INVALID_ARG, "null context");
    const nwprt_relight_opts o = opts ? *opts : default_opts();
    relight_ranges(ctx, {RangeReq{env_id, frame_id, indirect, with_direct, 0, 0}}, o, (cudaStream_t)stream);
  });
}

nwprt_status nwprt_relight_batch(nwprt_ctx* ctx, const nwprt_request* reqs, int n_reqs,
                                 const nwprt_relight_opts* opts, void* stream) {
  return guarded(ctx, [&] {
    TraceRange trace("nwprt_relight_batch");
    need(ctx && (reqs || n_reqs == 0) && n_reqs >= 0, NWPRT_INVALID_ARG, "bad request list");
    const nwprt_relight_opts o = opts ? *opts : default_opts();
    std::vector<RangeReq> v;
    v.reserve(n_reqs);
    for (int i = 0; i < n_reqs; ++i)
      v.push_back(RangeReq{reqs[i].env_id, reqs[i].frame_id, reqs[i].indirect, reqs[i].with_direct, 0, 0});
    relight_ranges(ctx, v, o, (cudaStream_t)stream);
  });
}

nwprt_status nwprt_relight_ranges(nwprt_ctx* ctx, const nwprt_range_request* reqs, int n_reqs,
                                  const nwprt_relight_opts* opts, void* stream) {
  return guarded(ctx, [&] {
    TraceRange trace("nwprt_relight_ranges");
    need(ctx && (reqs || n_reqs == 0) && n_reqs >= 0, NWPRT_INVALID_ARG, "bad request list");
    const nwprt_relight_opts o = opts ? *opts : default_opts();
    std::vector<RangeReq> v;
    v.reserve(n_reqs);
    for (int i = 0; i < n_reqs; ++i)
      v.push_back(RangeReq{reqs[i].env_id, reqs[i].frame_id, reqs[i].indirect, reqs[i].with_direct,
                           reqs[i].px_begin, reqs[i].px_end});
    relight_ranges(ctx, v, o, (cudaStream_t)stream);
  });
}

nwprt_status nwprt_calibrate_fp8(nwprt_ctx* ctx, int env_id, int frame_id, int64_t px_begin, int64_t px_end,
                                void* stream) {
  return guarded(ctx, [&] {
    TraceRange trace("nwprt_calibrate_fp8");
    need(ctx != nullptr, NWPRT_INVALID_ARG, "null context");
    need(ctx->weights_loaded, NWPRT_NOT_READY, "weights are not loaded");
    std::string why;
    need(relight_tc_fp8_supported(ctx->dims, &why), NWPRT_UNSUPPORTED, why.c_str());
    cudaStream_t st = (cudaStream_t)stream;
    RangeReq r{env_id, frame_id, nullptr, nullptr, px_begin, px_end};
    {
      // the range is checked before anything is allocated
      need(frame_id >= 0 && frame_id < NWPRT_MAX_FRAMES, NWPRT_INVALID_ARG, "frame id out of range");
      Frame& f = ctx->frames[frame_id];
      need(f.prepared, NWPRT_NOT_READY, "frame was not prepared (call nwprt_prepare first)");
      const int64_t n = (int64_t)f.width * f.height;
      if (r.px_end <= 0) r.px_end = n;
      need(r.px_begin >= 0 && r.px_begin < r.px_end && r.px_end <= n, NWPRT_INVALID_ARG,
           "calibration range must be a non-empty pixel range inside the frame");
    }
    const int n_layers = tc_layer_count(ctx->dims);
    const int64_t n_px = r.px_end - r.px_begin;
    // scratch outputs: the calibration pass is a full BF16 relight of the range
    float* out = dev_alloc<float>((size_t)n_px * 8);
    uint32_t* amax = nullptr;
    try {
      amax = dev_alloc<uint32_t>(n_layers + 1);
      NWPRT_CUDA(cudaMemsetAsync(amax, 0, (n_layers + 1) * 4, st));
      // outputs are indexed by absolute pixel: offset the scratch so the range lands in it
      r.indirect = out - r.px_begin * 4;
      r.with_direct = out + n_px * 4 - r.px_begin * 4;
      relight_many_tc(ctx, &r, 1, default_opts(), kTcCalibrate, amax, st);
      std::vector<uint32_t> bits(n_layers + 1);
      NWPRT_CUDA(cudaMemcpyAsync(bits.data(), amax, bits.size() * 4, cudaMemcpyDeviceToHost, st));
      NWPRT_CUDA(cudaStreamSynchronize(st));
      uint32_t err = 0;
      NWPRT_CUDA(cudaMemcpy(&err, ctx->d_err, 4, cudaMemcpyDeviceToHost));
      need(err == kDevOk, NWPRT_TIMEOUT, "the calibration pass reported a device error");
      std::vector<float> am(n_layers + 1);
      std::memcpy(am.data(), bits.data(), am.size() * 4);
      std::vector<uint8_t> blob;
      TcPlan plan = pack_tc_weights_fp8(ctx->dims, ctx->h_op.data(), ctx->h_cn.data(), am.data(), &blob);
      blob.resize(tc_blob_alloc_bytes(blob.size()), 0);  // whole rows of the kernel's TMA view
      // no launch may still read the previous blob
      NWPRT_CUDA(cudaDeviceSynchronize());
      dev_free(ctx->d_tc_w8);
      ctx->d_tc_w8 = nullptr;
      ctx->fp8_ready = false;
      ctx->d_tc_w8 = dev_alloc<uint8_t>(blob.size());
      NWPRT_CUDA(cudaMemcpy(ctx->d_tc_w8, blob.data(), blob.size(), cudaMemcpyHostToDevice));
      ctx->fp8_plan = plan;
      ctx->fp8_amax = am;
      ctx->fp8_ready = true;
    } catch (...) {
      cudaStreamSynchronize(st);
      dev_free(out);
      dev_free(amax);
      throw;
    }
    dev_free(out);
    dev_free(amax);
  });
}

nwprt_status nwprt_get_fp8_calibration(const nwprt_ctx* ctx, float* amax, int capacity, int* n_values) {
  return guarded(ctx, [&] {
    need(ctx && n_values && (amax || capacity == 0) && capacity >= 0, NWPRT_INVALID_ARG, "bad argument");
    need(ctx->fp8_ready, NWPRT_NOT_READY, "FP8 scales are not calibrated");
    *n_values = (int)ctx->fp8_amax.size();
    for (int i = 0; i < capacity && i < *n_values; ++i) amax[i] = ctx->fp8_amax[i];
  });
}

nwprt_status nwprt_tonemap_srgb(const float* src, int64_t n_px, uint32_t* dst, void* stream) {
  return guarded(nullptr, [&] { launch_tonemap_srgb(src, n_px, dst, (cudaStream_t)stream); });
}

nwprt_status nwprt_sh_vertex_radiance(const float* T, const float* brdf_sh, const float* L, int64_t n_vertices,
                                      int n_coeffs, float* out, void* stream) {
  return guarded(nullptr, [&] { launch_sh_vertex(T, brdf_sh, L, n_vertices, n_coeffs, out, (cudaStream_t)stream); });
}

nwprt_status nwprt_sh_interpolate(nwprt_ctx* ctx, const float* vertex_rgb, int64_t n_vertices, const int32_t* tri,
                                  const float* uv, int64_t n_px, float* out, void* stream) {
  return guarded(ctx, [&] {
    TraceRange trace("nwprt_sh_interpolate");
    need(ctx != nullptr, NWPRT_INVALID_ARG, "null context");
    launch_sh_interpolate(vertex_rgb, n_vertices, tri, uv, n_px, out, ctx->d_err, (cudaStream_t)stream);
  });
}

nwprt_status nwprt_selftest_device_wait(nwprt_ctx* ctx, int timeout_ms, void* stream) {
  return guarded(ctx, [&] {
    need(ctx != nullptr, NWPRT_INVALID_ARG, "null context");
    launch_wait_selftest(timeout_ms, ctx->d_err, (cudaStream_t)stream);
  });
}

nwprt_status nwprt_sync(nwprt_ctx* ctx) {
  return guarded(ctx, [&] {
    need(ctx != nullptr, NWPRT_INVALID_ARG, "null context");
    NWPRT_CUDA(cudaDeviceSynchronize());
    uint32_t err = 0;
    NWPRT_CUDA(cudaMemcpy(&err, ctx->d_err, 4, cudaMemcpyDeviceToHost));
    if (err != kDevOk) {
      NWPRT_CUDA(cudaMemset(ctx->d_err, 0, 4));
      if (err == kDevWaitTimeout) fail(NWPRT_TIMEOUT, "a device-side wait timed out; results are invalid");
      fail(NWPRT_INVALID_ARG, "a wavelet index was outside the embedding table; it read as 0");
    }
  });
}

nwprt_status nwprt_haar_topk(const float* faces, int n_env, int S, int K, int32_t* idx, float* strength,
                             void* stream) {
  return guarded(nullptr, [&] { launch_haar_topk(faces, n_env, S, K, idx, strength, nullptr, (cudaStream_t)stream); });
}

nwprt_status nwprt_env_rotate(const float* src, int S, const float* R, float* dst, void* stream) {
  return guarded(nullptr, [&] { launch_env_rotate(src, S, R, dst, (cudaStream_t)stream); });
}

size_t nwprt_sh_project_workspace_size(int S) { return S > 0 ? sh_project_workspace_bytes(S) : 0; }

nwprt_status nwprt_sh_project(const float* faces, int S, float* L, void* workspace, size_t workspace_bytes,
                              void* stream) {
  return guarded(nullptr, [&] {
    need(faces && L && workspace, NWPRT_INVALID_ARG, "null argument");
    need(S >= 1 && S <= 4096, NWPRT_INVALID_ARG, "face size out of range");
    need(workspace_bytes >= sh_project_workspace_bytes(S), NWPRT_INVALID_ARG,
         "workspace smaller than nwprt_sh_project_workspace_size(S)");
    launch_sh_project(faces, S, L, (float*)workspace, (cudaStream_t)stream);
  });
}

nwprt_status nwprt_sh_dot(const float* T, int64_t n_px, int n_coeffs, const float* L, int abs_out, float* out,
                          void* stream) {
  return guarded(nullptr, [&] {
    need((T && L && out) || n_px == 0, NWPRT_INVALID_ARG, "null argument");
    launch_sh_dot(T, n_px, n_coeffs, L, abs_out, out, nullptr, (cudaStream_t)stream);
  });
}

}  // extern "C"

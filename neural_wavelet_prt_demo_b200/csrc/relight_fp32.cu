// Fused plain-FP32 relight kernel: the drop-in path.
//
// One thread owns one pixel for the whole pass.  It encodes the pixel's position with
// the multiresolution hash grid once, then for each of the env's K wavelets runs
//   cp = enc * E_k                         (ptwise_mlt, utils_kernels.h:110-127)
//   out_prd MLP -> [out_prd || aux] -> cmp_net MLP -> T_k (RGB)  (prt_network.h:73-154)
//   sum += max(L_k * T_k, 0)               (computeResponse, utils_kernels.h:84-91)
// keeping T_k in registers: the N x K transport matrix and the K-fold replicated input
// of the reference never exist.  Every dot product accumulates fmaf(W[j][i], x_i, .) from
// 0 in ascending i -- the order of the FP32 oracle (oracle/nwprt_oracle.c: dense_f32) --
// and the K-sum is Kahan-compensated by default.
//
// Layout: all layer weights live in shared memory transposed to [in][out4] so that each
// input element meets a warp-uniform float4 row (broadcast reads); each thread keeps its
// activation vector in a private shared-memory column (conflict-free, stride = block size).
#include <cmath>

#include "nwprt_internal.cuh"

namespace nwprt {
namespace {

constexpr int r4(int x) { return (x + 3) & ~3; }
constexpr int kMaxKChunk = 16;

struct Fp32Params {
  HashLevels hl;
  const float* hash;
  const float* w;        // op_t || cn_t, transposed and padded
  int w_floats;          // multiple of 4
  const float* packed;
  const uint8_t* flag;
  const float* direct;
  const float* emb_k;
  const float* strength;
  int K;
  int64_t px_begin, n_px;  // pixel range [px_begin, n_px)
  float* indirect;
  float* with_direct;
  int clamp, kahan;
};

// Hash-grid encoding of one position (oracle/nwprt_oracle.c: orc_hash_encode_f32).
__device__ __forceinline__ void hash_encode(const HashLevels& hl, const float* __restrict__ table,
                                            float px, float py, float pz, float* act, int stride,
                                            int row0) {
  const float p[3] = {fminf(fmaxf(px, 0.f), 1.f), fminf(fmaxf(py, 0.f), 1.f),
                      fminf(fmaxf(pz, 0.f), 1.f)};
  const int F = hl.n_features;
  for (int l = 0; l < hl.n_levels; ++l) {
    const int N = hl.res[l];
    uint32_t i0[3];
    float w[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float xl = __fmul_rn(p[d], (float)N);
      int i = (int)floorf(xl);
      if (i > N - 1) i = N - 1;
      i0[d] = (uint32_t)i;
      w[d] = __fsub_rn(xl, (float)i);
    }
    const uint32_t N1 = (uint32_t)N + 1u;
    const bool dense = (hl.dense_mask >> l) & 1u;
    const uint32_t T = hl.size[l];
    const float* lvl = table + (size_t)hl.offset[l] * F;
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const uint32_t bx = c & 1, by = (c >> 1) & 1, bz = (c >> 2) & 1;
      const float wx = bx ? w[0] : __fsub_rn(1.f, w[0]);
      const float wy = by ? w[1] : __fsub_rn(1.f, w[1]);
      const float wz = bz ? w[2] : __fsub_rn(1.f, w[2]);
      const float wc = __fmul_rn(__fmul_rn(wx, wy), wz);
      const uint32_t x = i0[0] + bx, y = i0[1] + by, z = i0[2] + bz;
      const uint32_t e = dense ? x + y * N1 + z * N1 * N1
                               : ((x ^ (y * 2654435761u) ^ (z * 805459861u)) & (T - 1u));
      const float* th = lvl + (size_t)e * F;
      if (F == 2) {
        const float2 v = __ldg(reinterpret_cast<const float2*>(th));
        acc[0] = fmaf(wc, v.x, acc[0]);
        acc[1] = fmaf(wc, v.y, acc[1]);
      } else {
        for (int f = 0; f < F; ++f) acc[f] = fmaf(wc, __ldg(th + f), acc[f]);
      }
    }
    for (int f = 0; f < F; ++f) act[(row0 + l * F + f) * stride] = acc[f];
  }
}

// Two FP32 values in one 64-bit register, and the packed FMA of sm_100 on such pairs:
// fma.rn.f32x2 rounds each lane once, exactly as fmaf does, so a pair of output neurons
// accumulated side by side keeps the oracle's bits with half the FMA instructions.
__device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ void f2_fma(unsigned long long& acc, unsigned long long a, unsigned long long b) {
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(a), "l"(b));
}

// y = act(W x) over one thread's activation column.
// MODE 0: x_i = act row i.  MODE 1: x_i = act row (ENC + i) * e[i] (the CP product).
// MODE 2: x_i = act row i for i < OPO, else act row (AUX + i - OPO) (the [out_prd || aux] concat).
template <int IN, int OUT, bool RELU, int MODE, int NT, int ENC, int AUX, int OPO>
__device__ __forceinline__ void dense(const float* __restrict__ Wt, float* act,
                                      const float* __restrict__ e, float* outv) {
  constexpr int O4 = r4(OUT) / 4;
  unsigned long long acc2[O4 * 2];  // output pairs (2j, 2j + 1)
#pragma unroll
  for (int j = 0; j < O4 * 2; ++j) acc2[j] = 0ull;
#pragma unroll 4
  for (int i = 0; i < IN; ++i) {
    float xi;
    if (MODE == 0) xi = act[i * NT];
    else if (MODE == 1) xi = __fmul_rn(act[(ENC + i) * NT], e[i]);
    else xi = (i < OPO) ? act[i * NT] : act[(AUX + i - OPO) * NT];
    const unsigned long long x2 = f2_pack(xi, xi);
    const float4* w4 = reinterpret_cast<const float4*>(Wt + i * O4 * 4);
#pragma unroll
    for (int j = 0; j < O4; ++j) {
      const float4 w = w4[j];
      f2_fma(acc2[2 * j], f2_pack(w.x, w.y), x2);
      f2_fma(acc2[2 * j + 1], f2_pack(w.z, w.w), x2);
    }
  }
  float acc[O4 * 4];
#pragma unroll
  for (int j = 0; j < O4 * 2; ++j) f2_unpack(acc2[j], acc[2 * j], acc[2 * j + 1]);
#pragma unroll
  for (int j = 0; j < OUT; ++j) {
    const float v = RELU ? fmaxf(acc[j], 0.f) : acc[j];
    if (outv) outv[j] = v;
    else act[j * NT] = v;
  }
}

// Compile-time network shape: D hash features, out_prd with OPH hidden layers of width W and
// OPO outputs, cmp_net with CNH hidden layers of width W, AUXW aux inputs, NT threads.
template <int D, int OPH, int OPO, int CNH, int W, int AUXW, int NT>
struct Net {
  static constexpr int kActRows = (W > OPO ? W : OPO);
  static constexpr int kEnc = kActRows;
  static constexpr int kAux = kActRows + D;
  static constexpr int kRows = kAux + AUXW;
  static constexpr int kCnIn = OPO + AUXW;

  static constexpr int weight_floats() {
    int f = 0;
    if (OPH == 0) f += D * r4(OPO);
    else f += D * r4(W) + (OPH - 1) * W * r4(W) + W * r4(OPO);
    if (CNH == 0) f += kCnIn * r4(3);
    else f += kCnIn * r4(W) + (CNH - 1) * W * r4(W) + W * r4(3);
    return f;
  }

  __device__ static void eval(const float* sW, float* act, const float* e, float* T) {
    const float* w = sW;
    if constexpr (OPH == 0) {
      dense<D, OPO, false, 1, NT, kEnc, kAux, OPO>(w, act, e, nullptr);
      w += D * r4(OPO);
    } else {
      dense<D, W, true, 1, NT, kEnc, kAux, OPO>(w, act, e, nullptr);
      w += D * r4(W);
#pragma unroll 1
      for (int l = 1; l < OPH; ++l) {
        dense<W, W, true, 0, NT, kEnc, kAux, OPO>(w, act, nullptr, nullptr);
        w += W * r4(W);
      }
      dense<W, OPO, false, 0, NT, kEnc, kAux, OPO>(w, act, nullptr, nullptr);
      w += W * r4(OPO);
    }
    if constexpr (CNH == 0) {
      dense<kCnIn, 3, false, 2, NT, kEnc, kAux, OPO>(w, act, nullptr, T);
    } else {
      dense<kCnIn, W, true, 2, NT, kEnc, kAux, OPO>(w, act, nullptr, nullptr);
      w += kCnIn * r4(W);
#pragma unroll 1
      for (int l = 1; l < CNH; ++l) {
        dense<W, W, true, 0, NT, kEnc, kAux, OPO>(w, act, nullptr, nullptr);
        w += W * r4(W);
      }
      dense<W, 3, false, 0, NT, kEnc, kAux, OPO>(w, act, nullptr, T);
    }
  }

  static size_t smem_bytes(int w_floats) {
    return sizeof(float) * ((size_t)w_floats + kMaxKChunk * D + kMaxKChunk * 4 + (size_t)kRows * NT);
  }
};

template <class NET, int D, int AUXW, int NT>
__global__ void __launch_bounds__(NT, 1) relight_fp32_kernel(Fp32Params p) {
  extern __shared__ __align__(16) float sm[];
  float* sW = sm;
  float* sE = sW + p.w_floats;
  float* sL = sE + kMaxKChunk * D;
  float* sAct = sL + kMaxKChunk * 4;
  const int tid = threadIdx.x;
  for (int i = tid * 4; i < p.w_floats; i += NT * 4)
    *reinterpret_cast<float4*>(sW + i) = __ldg(reinterpret_cast<const float4*>(p.w + i));
  const int64_t px = p.px_begin + (int64_t)blockIdx.x * NT + tid;
  const bool valid = px < p.n_px;
  const bool active = valid && p.flag[px] != 0;
  float* act = sAct + tid;
  if (valid) {
    const float4* row = reinterpret_cast<const float4*>(p.packed) + px * 4;
    const float4 r0 = row[0], r1 = row[1], r2 = row[2], r3 = row[3];
    if (active) hash_encode(p.hl, p.hash, r0.x, r0.y, r0.z, act, NT, NET::kEnc);
    const float aux13[13] = {r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w, r3.x, r3.y, r3.z, r3.w};
#pragma unroll
    for (int i = 0; i < AUXW; ++i) act[(NET::kAux + i) * NT] = i < 13 ? aux13[i] : 1.0f;
  }
  float s[3] = {0.f, 0.f, 0.f}, comp[3] = {0.f, 0.f, 0.f};
  for (int k0 = 0; k0 < p.K; k0 += kMaxKChunk) {
    const int kc = min(kMaxKChunk, p.K - k0);
    __syncthreads();
    for (int i = tid; i < kc * D; i += NT) sE[i] = p.emb_k[(size_t)k0 * D + i];
    for (int i = tid; i < kc * 3; i += NT) sL[(i / 3) * 4 + i % 3] = p.strength[(size_t)k0 * 3 + i];
    __syncthreads();
    if (!active) continue;
    for (int kk = 0; kk < kc; ++kk) {
      float T[3];
      NET::eval(sW, act, sE + kk * D, T);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float term = __fmul_rn(sL[kk * 4 + c], T[c]);
        if (p.clamp) term = fmaxf(term, 0.0f);
        if (p.kahan) {
          const float y = __fsub_rn(term, comp[c]);
          const float t = __fadd_rn(s[c], y);
          comp[c] = __fsub_rn(__fsub_rn(t, s[c]), y);
          s[c] = t;
        } else {
          s[c] = __fadd_rn(s[c], term);
        }
      }
    }
  }
  if (valid) {
    const float4 dl = reinterpret_cast<const float4*>(p.direct)[px];
    reinterpret_cast<float4*>(p.indirect)[px] = make_float4(s[0], s[1], s[2], 1.f);
    reinterpret_cast<float4*>(p.with_direct)[px] =
        make_float4(__fadd_rn(s[0], dl.x), __fadd_rn(s[1], dl.y), __fadd_rn(s[2], dl.z), 1.f);
  }
}

// ---- any other supported network: the same arithmetic with the layer sequence read at run
// time.  Every dot product still accumulates fmaf(W[j][i], x_i, .) from 0 in ascending i, so
// results are the same bits as the oracle's.  Output widths up to kGenMaxOut.
constexpr int kGenMaxOut = 64;
constexpr int kGenMaxLayers = 2 * kMaxLayers;
struct GenLayer {
  int in, out, relu, mode;  // mode as in dense(): 0 plain, 1 CP product, 2 [out_prd || aux]
  int w_off;                // float offset of the [in][round4(out)] block
};
struct GenNet {
  GenLayer l[kGenMaxLayers];
  int n = 0;
  int enc = 0, aux = 0, rows = 0, opo = 0, d = 0, auxw = 0;
};

template <int NT>
__device__ __forceinline__ void dense_rt(const GenLayer& L, const GenNet& g, const float* __restrict__ Wt,
                                         float* act, const float* __restrict__ e, float* outv) {
  unsigned long long acc2[kGenMaxOut / 2];  // output pairs (2j, 2j + 1)
#pragma unroll
  for (int j = 0; j < kGenMaxOut / 2; ++j) acc2[j] = 0ull;
  const int o4 = (L.out + 3) / 4;
  for (int i = 0; i < L.in; ++i) {
    float xi;
    if (L.mode == 0) xi = act[i * NT];
    else if (L.mode == 1) xi = __fmul_rn(act[(g.enc + i) * NT], e[i]);
    else xi = (i < g.opo) ? act[i * NT] : act[(g.aux + i - g.opo) * NT];
    const unsigned long long x2 = f2_pack(xi, xi);
    const float4* w4 = reinterpret_cast<const float4*>(Wt + (size_t)i * o4 * 4);
#pragma unroll
    for (int j = 0; j < kGenMaxOut / 4; ++j) {
      if (j < o4) {
        const float4 w = w4[j];
        f2_fma(acc2[2 * j], f2_pack(w.x, w.y), x2);
        f2_fma(acc2[2 * j + 1], f2_pack(w.z, w.w), x2);
      }
    }
  }
  float acc[kGenMaxOut];
#pragma unroll
  for (int j = 0; j < kGenMaxOut / 2; ++j) f2_unpack(acc2[j], acc[2 * j], acc[2 * j + 1]);
#pragma unroll
  for (int j = 0; j < kGenMaxOut; ++j) {
    if (j < L.out) {
      const float v = L.relu ? fmaxf(acc[j], 0.f) : acc[j];
      if (outv) outv[j] = v;
      else act[j * NT] = v;
    }
  }
}

template <int NT>
__global__ void __launch_bounds__(NT, 1) relight_fp32_generic_kernel(Fp32Params p, const __grid_constant__ GenNet g) {
  extern __shared__ __align__(16) float sm[];
  float* sW = sm;
  float* sE = sW + p.w_floats;
  float* sL = sE + kMaxKChunk * g.d;
  float* sAct = sL + kMaxKChunk * 4;
  const int tid = threadIdx.x;
  for (int i = tid * 4; i < p.w_floats; i += NT * 4)
    *reinterpret_cast<float4*>(sW + i) = __ldg(reinterpret_cast<const float4*>(p.w + i));
  const int64_t px = p.px_begin + (int64_t)blockIdx.x * NT + tid;
  const bool valid = px < p.n_px;
  const bool active = valid && p.flag[px] != 0;
  float* act = sAct + tid;
  if (valid) {
    const float4* row = reinterpret_cast<const float4*>(p.packed) + px * 4;
    const float4 r0 = row[0], r1 = row[1], r2 = row[2], r3 = row[3];
    if (active) hash_encode(p.hl, p.hash, r0.x, r0.y, r0.z, act, NT, g.enc);
    const float aux13[13] = {r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w, r3.x, r3.y, r3.z, r3.w};
    for (int i = 0; i < g.auxw; ++i) act[(g.aux + i) * NT] = i < 13 ? aux13[i] : 1.0f;
  }
  float s[3] = {0.f, 0.f, 0.f}, comp[3] = {0.f, 0.f, 0.f};
  for (int k0 = 0; k0 < p.K; k0 += kMaxKChunk) {
    const int kc = min(kMaxKChunk, p.K - k0);
    __syncthreads();
    for (int i = tid; i < kc * g.d; i += NT) sE[i] = p.emb_k[(size_t)k0 * g.d + i];
    for (int i = tid; i < kc * 3; i += NT) sL[(i / 3) * 4 + i % 3] = p.strength[(size_t)k0 * 3 + i];
    __syncthreads();
    if (!active) continue;
    for (int kk = 0; kk < kc; ++kk) {
      float T[3];
      for (int li = 0; li < g.n; ++li)
        dense_rt<NT>(g.l[li], g, sW + g.l[li].w_off, act, sE + kk * g.d, li + 1 == g.n ? T : nullptr);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float term = __fmul_rn(sL[kk * 4 + c], T[c]);
        if (p.clamp) term = fmaxf(term, 0.0f);
        if (p.kahan) {
          const float y = __fsub_rn(term, comp[c]);
          const float t = __fadd_rn(s[c], y);
          comp[c] = __fsub_rn(__fsub_rn(t, s[c]), y);
          s[c] = t;
        } else {
          s[c] = __fadd_rn(s[c], term);
        }
      }
    }
  }
  if (valid) {
    const float4 dl = reinterpret_cast<const float4*>(p.direct)[px];
    reinterpret_cast<float4*>(p.indirect)[px] = make_float4(s[0], s[1], s[2], 1.f);
    reinterpret_cast<float4*>(p.with_direct)[px] =
        make_float4(__fadd_rn(s[0], dl.x), __fadd_rn(s[1], dl.y), __fadd_rn(s[2], dl.z), 1.f);
  }
}

// The run-time layer sequence of d: out_prd's layers (the first takes the CP product), then
// cmp_net's (the first takes [out_prd || aux]); the last layer writes T.
bool gen_net(const NetDims& d, GenNet* g, std::string* why) {
  auto no = [&](const char* m) { if (why) *why = m; return false; };
  if (d.op_nl + d.cn_nl > kGenMaxLayers) return no("fp32 relight: too many layers");
  int off = 0, widest = d.op_out;
  for (int i = 0; i < d.op_nl; ++i) {
    if (d.op_outs[i] > kGenMaxOut) return no("fp32 relight: layer widths above 64 are not supported");
    g->l[g->n++] = GenLayer{d.op_in[i], d.op_outs[i], i + 1 < d.op_nl ? 1 : 0, i == 0 ? 1 : 0, off};
    off += d.op_in[i] * r4(d.op_outs[i]);
    widest = d.op_outs[i] > widest ? d.op_outs[i] : widest;
  }
  for (int i = 0; i < d.cn_nl; ++i) {
    if (d.cn_outs[i] > kGenMaxOut) return no("fp32 relight: layer widths above 64 are not supported");
    g->l[g->n++] = GenLayer{d.cn_in[i], d.cn_outs[i], i + 1 < d.cn_nl ? 1 : 0, i == 0 ? 2 : 0, off};
    off += d.cn_in[i] * r4(d.cn_outs[i]);
    if (i + 1 < d.cn_nl) widest = d.cn_outs[i] > widest ? d.cn_outs[i] : widest;
  }
  if (d.cn_outs[d.cn_nl - 1] != 3) return no("fp32 relight: cmp_net must end in 3 outputs");
  g->d = d.enc_dims();
  g->opo = d.op_out;
  g->auxw = d.aux_width;
  g->enc = widest;
  g->aux = widest + g->d;
  g->rows = g->aux + g->auxw;
  return true;
}

size_t gen_smem_bytes(const GenNet& g, int w_floats, int nt) {
  return sizeof(float) * ((size_t)w_floats + kMaxKChunk * g.d + kMaxKChunk * 4 + (size_t)g.rows * nt);
}

template <int D, int OPH, int OPO, int CNH, int W, int AUXW>
bool try_launch(const NetDims& d, const Fp32Params& p, cudaStream_t st) {
  if (d.enc_dims() != D || d.op_hidden != OPH || d.op_out != OPO || d.cn_hidden != CNH ||
      d.aux_width != AUXW || (OPH > 0 && d.op_neurons != W) || (CNH > 0 && d.cn_neurons != W))
    return false;
  int dev = 0, max_smem = 0;
  NWPRT_CUDA(cudaGetDevice(&dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  using N256 = Net<D, OPH, OPO, CNH, W, AUXW, 256>;
  using N128 = Net<D, OPH, OPO, CNH, W, AUXW, 128>;
  if (N256::weight_floats() != p.w_floats) fail(NWPRT_INVALID_ARG, "fp32 weight layout mismatch");
  const int64_t n = p.n_px - p.px_begin;
  if (N256::smem_bytes(p.w_floats) <= (size_t)max_smem && n >= 256 * 148) {
    auto k = relight_fp32_kernel<N256, D, AUXW, 256>;
    const size_t smem = N256::smem_bytes(p.w_floats);
    NWPRT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<(unsigned)((n + 255) / 256), 256, smem, st>>>(p);
  } else {
    auto k = relight_fp32_kernel<N128, D, AUXW, 128>;
    const size_t smem = N128::smem_bytes(p.w_floats);
    if (smem > (size_t)max_smem) fail(NWPRT_UNSUPPORTED, "fp32 relight: network too large for shared memory");
    NWPRT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<(unsigned)((n + 127) / 128), 128, smem, st>>>(p);
  }
  NWPRT_CUDA(cudaGetLastError());
  return true;
}

}  // namespace

// Transposes each row-major [out][in] layer to [in][round4(out)] (zero padded).
void pack_fp32_weights(const NetDims& d, const float* op, const float* cn, std::vector<float>* op_t,
                       std::vector<float>* cn_t) {
  auto pack = [](int nl, const int* in, const int* out, const float* src, std::vector<float>* dst) {
    dst->clear();
    for (int l = 0; l < nl; ++l) {
      const int o4 = r4(out[l]);
      size_t base = dst->size();
      dst->resize(base + (size_t)in[l] * o4, 0.f);
      for (int j = 0; j < out[l]; ++j)
        for (int i = 0; i < in[l]; ++i) (*dst)[base + (size_t)i * o4 + j] = src[(size_t)j * in[l] + i];
      src += (size_t)in[l] * out[l];
    }
  };
  pack(d.op_nl, d.op_in, d.op_outs, op, op_t);
  pack(d.cn_nl, d.cn_in, d.cn_outs, cn, cn_t);
}

// The two standard shapes run compile-time kernels; every other network whose layers are at
// most 64 wide (and whose weights fit in shared memory) runs the generic kernel.
void launch_relight_fp32(const NetDims& d, const HashLevels& hl, const DeviceWeights& w,
                         const RelightJob& job, int clamp, int kahan, cudaStream_t st) {
  if (job.n_px <= job.px_begin) return;
  Fp32Params p;
  p.hl = hl;
  p.hash = w.hash;
  p.w = w.op_t;  // op_t and cn_t are stored back to back
  p.w_floats = (int)(w.op_t_floats + w.cn_t_floats);
  p.packed = job.packed;
  p.flag = job.flag;
  p.direct = job.direct;
  p.emb_k = job.emb_k;
  p.strength = job.strength;
  p.K = job.K;
  p.px_begin = job.px_begin;
  p.n_px = job.n_px;
  p.indirect = job.indirect;
  p.with_direct = job.with_direct;
  p.clamp = clamp;
  p.kahan = kahan;
  if (try_launch<16, 0, 26, 2, 64, 16>(d, p, st)) return;
  if (try_launch<32, 3, 64, 3, 64, 16>(d, p, st)) return;
  GenNet g;
  std::string why;
  if (!gen_net(d, &g, &why)) fail(NWPRT_UNSUPPORTED, why);
  const GenLayer& last = g.l[g.n - 1];
  if (last.w_off + last.in * r4(last.out) != p.w_floats) fail(NWPRT_INVALID_ARG, "fp32 weight layout mismatch");
  int dev = 0, max_smem = 0;
  NWPRT_CUDA(cudaGetDevice(&dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const size_t smem = gen_smem_bytes(g, p.w_floats, 128);
  if (smem > (size_t)max_smem) fail(NWPRT_UNSUPPORTED, "fp32 relight: network too large for shared memory");
  auto k = relight_fp32_generic_kernel<128>;
  NWPRT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t n = p.n_px - p.px_begin;
  k<<<(unsigned)((n + 127) / 128), 128, smem, st>>>(p, g);
  NWPRT_CUDA(cudaGetLastError());
}

}  // namespace nwprt

// Cubemap Haar transform + top-K wavelet selection, one thread-block cluster per env map.
//
// The reference only loads precomputed results (waveletcoeffs/<name>.npy and
// waveletstrength/<name>.npy, Renderer/EnvironmentMap.cpp:97-108); the transform and
// the selection order are defined by the oracle (oracle/nwprt_oracle.c:
// orc_haar_face / orc_haar_topk) and reproduced here bit for bit:
//  * per face, non-standard 2-D Haar with orthonormal 1/2 factors, Mallat layout,
//    evaluated with the same FP32 adds/multiplies (no contraction: __fadd_rn etc.);
//  * key = |0.212671 r + 0.715160 g + 0.072169 b| (EnvironmentMap.cpp:149-151), NaN -> 0;
//  * order = key descending, flat index face*S*S + row*S + col ascending.
//
// Design: a cluster of 6 CTAs (one per face) keeps every face in its own shared
// memory.  The top-K threshold is found by a 4-pass 8-bit radix select whose
// per-face histograms are summed through distributed shared memory; ties at the
// threshold are taken in flat-index order by an ordered block compaction; the K
// winners are gathered into CTA 0's shared memory and ranked there.  Nothing but
// the inputs and outputs touches global memory.
#include <cooperative_groups.h>

#include "nwprt_internal.cuh"

namespace cg = cooperative_groups;

namespace nwprt {
namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxS = 64;
constexpr int kMaxK = 1024;

struct Gathered {
  float r, g, b;
  int32_t idx;
};

struct HaarSmem {
  float* C;        // [S][S][3] coefficients
  float* Tm;       // [(S/2)^2][3] level scratch
  uint32_t* keys;  // [S*S]
  uint32_t* hist;  // [2][256]
  uint32_t* all_h; // [6][256] local copy of the cluster's histograms
  uint64_t* gkey;  // [K] composite keys (CTA 0)
  Gathered* gval;  // [K]
  int* warp_tot;   // [kWarps]
  int* scal;       // scalars
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline size_t smem_layout(int S, int K, char* base, HaarSmem* L) {
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o = align16(o + bytes); return at; };
  size_t oC = take(sizeof(float) * S * S * 3);
  size_t oT = take(sizeof(float) * (S / 2 > 0 ? (S / 2) * (S / 2) : 1) * 3);
  size_t oK = take(sizeof(uint32_t) * S * S);
  size_t oH = take(sizeof(uint32_t) * 512);
  size_t oA = take(sizeof(uint32_t) * 6 * 256);
  size_t oG = take(sizeof(uint64_t) * K);
  size_t oV = take(sizeof(Gathered) * K);
  size_t oW = take(sizeof(int) * kWarps);
  size_t oS = take(sizeof(int) * 32);
  if (L) {
    L->C = (float*)(base + oC);
    L->Tm = (float*)(base + oT);
    L->keys = (uint32_t*)(base + oK);
    L->hist = (uint32_t*)(base + oH);
    L->all_h = (uint32_t*)(base + oA);
    L->gkey = (uint64_t*)(base + oG);
    L->gval = (Gathered*)(base + oV);
    L->warp_tot = (int*)(base + oW);
    L->scal = (int*)(base + oS);
  }
  return o;
}

__device__ __forceinline__ void haar4(float a, float b, float c, float d, float& ll, float& hl,
                                      float& lh, float& hh) {
  const float s0 = __fadd_rn(a, b), d0 = __fsub_rn(a, b);
  const float s1 = __fadd_rn(c, d), d1 = __fsub_rn(c, d);
  ll = __fmul_rn(__fadd_rn(s0, s1), 0.5f);
  hl = __fmul_rn(__fadd_rn(d0, d1), 0.5f);
  lh = __fmul_rn(__fsub_rn(s0, s1), 0.5f);
  hh = __fmul_rn(__fsub_rn(d0, d1), 0.5f);
}

__device__ __forceinline__ uint32_t wavelet_key_bits(float r, float g, float b) {
  float t = __fmul_rn(0.212671f, r);
  t = __fadd_rn(t, __fmul_rn(0.715160f, g));
  t = __fadd_rn(t, __fmul_rn(0.072169f, b));
  t = fabsf(t);
  if (t != t) t = 0.0f;
  return __float_as_uint(t);
}

// Exclusive rank of `pred` among the block's threads in thread order, plus the
// block total.  Two __syncthreads.
__device__ __forceinline__ int block_rank(bool pred, int* warp_tot, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned m = __ballot_sync(0xffffffffu, pred);
  const int in_warp = __popc(m & ((1u << lane) - 1u));
  if (lane == 0) warp_tot[warp] = __popc(m);
  __syncthreads();
  int before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    const int t = warp_tot[w];
    before += (w < warp) ? t : 0;
    all += t;
  }
  __syncthreads();
  *total = all;
  return before + in_warp;
}

__global__ void __cluster_dims__(6, 1, 1) __launch_bounds__(kThreads)
    haar_topk_kernel(const float* __restrict__ faces, int S, int K, int32_t* __restrict__ idx_out,
                     float* __restrict__ st_out) {
  extern __shared__ __align__(16) char smem_raw[];
  HaarSmem sm;
  smem_layout(S, K, smem_raw, &sm);
  cg::cluster_group cluster = cg::this_cluster();
  const int face = (int)cluster.block_rank();
  const int env = blockIdx.x / 6;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int SS = S * S;
  const float* src = faces + ((size_t)env * 6 + face) * (size_t)SS * 3;

  // ---- level n = S, straight from global memory into C
  if (S >= 2) {
    const int h = S >> 1;
    for (int b = tid; b < h * h; b += nt) {
      const int i = b / h, j = b - i * h;
      const float* r0 = src + ((size_t)(2 * i) * S + 2 * j) * 3;
      const float* r1 = r0 + (size_t)S * 3;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float ll, hl, lh, hh;
        haar4(__ldg(r0 + c), __ldg(r0 + 3 + c), __ldg(r1 + c), __ldg(r1 + 3 + c), ll, hl, lh, hh);
        sm.C[(i * S + j) * 3 + c] = ll;
        sm.C[(i * S + j + h) * 3 + c] = hl;
        sm.C[((i + h) * S + j) * 3 + c] = lh;
        sm.C[((i + h) * S + j + h) * 3 + c] = hh;
      }
    }
  } else {
    if (tid < 3) sm.C[tid] = src[tid];
  }
  __syncthreads();
  // ---- remaining levels inside shared memory
  for (int n = S >> 1; n >= 2; n >>= 1) {
    const int h = n >> 1;
    for (int b = tid; b < h * h; b += nt) {
      const int i = b / h, j = b - i * h;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float ll, hl, lh, hh;
        haar4(sm.C[((2 * i) * S + 2 * j) * 3 + c], sm.C[((2 * i) * S + 2 * j + 1) * 3 + c],
              sm.C[((2 * i + 1) * S + 2 * j) * 3 + c], sm.C[((2 * i + 1) * S + 2 * j + 1) * 3 + c],
              ll, hl, lh, hh);
        sm.Tm[(i * n + j) * 3 + c] = ll;
        sm.Tm[(i * n + j + h) * 3 + c] = hl;
        sm.Tm[((i + h) * n + j) * 3 + c] = lh;
        sm.Tm[((i + h) * n + j + h) * 3 + c] = hh;
      }
    }
    __syncthreads();
    for (int e = tid; e < n * n * 3; e += nt) {
      const int r = e / (n * 3), rem = e - r * (n * 3);
      sm.C[r * S * 3 + rem] = sm.Tm[e];
    }
    __syncthreads();
  }
  // ---- keys
  for (int p = tid; p < SS; p += nt) sm.keys[p] = wavelet_key_bits(sm.C[p * 3], sm.C[p * 3 + 1], sm.C[p * 3 + 2]);
  // ---- 4-pass radix select of the K-th largest key over the whole cluster
  uint32_t prefix = 0, mask = 0;
  int remaining = K;
  int* gt = sm.scal + 8;   // [6] keys above the threshold, per face
  int* eq = sm.scal + 16;  // [6] keys equal to the threshold, per face
  if (tid < 6) { gt[tid] = 0; eq[tid] = 0; }
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = 24 - 8 * pass;
    uint32_t* h = sm.hist + (pass & 1) * 256;
    for (int d = tid; d < 256; d += nt) h[d] = 0;
    __syncthreads();
    for (int p = tid; p < SS; p += nt) {
      const uint32_t k = sm.keys[p];
      if ((k & mask) == prefix) atomicAdd(&h[(k >> shift) & 255u], 1u);
    }
    cluster.sync();
    if (tid < 256) {
#pragma unroll
      for (int g = 0; g < 6; ++g) sm.all_h[g * 256 + tid] = cluster.map_shared_rank(h, g)[tid];
    }
    __syncthreads();
    if (tid < 32) {
      // lane l covers digits 255-8l .. 248-8l (highest digits first)
      const int lane = tid;
      const int d_hi = 255 - 8 * lane;
      uint32_t tot8[8];
      uint32_t local = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        uint32_t t = 0;
#pragma unroll
        for (int g = 0; g < 6; ++g) t += sm.all_h[g * 256 + d_hi - q];
        tot8[q] = t;
        local += t;
      }
      uint32_t incl = local;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const uint32_t excl = incl - local;
      const unsigned hit = __ballot_sync(0xffffffffu, incl >= (uint32_t)remaining);
      const int cl = __ffs(hit) - 1;  // the total count >= remaining, so hit != 0
      int dsel = 0;
      uint32_t above = 0;
      if (lane == cl) {
        uint32_t cum = excl;
        for (int q = 0; q < 8; ++q) {
          if (cum + tot8[q] >= (uint32_t)remaining) { dsel = d_hi - q; break; }
          cum += tot8[q];
        }
        above = cum;
      }
      dsel = __shfl_sync(0xffffffffu, dsel, cl);
      above = __shfl_sync(0xffffffffu, above, cl);
      // per-face counts of keys whose digit is above dsel
#pragma unroll
      for (int g = 0; g < 6; ++g) {
        uint32_t s = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int d = d_hi - q;
          s += d > dsel ? sm.all_h[g * 256 + d] : 0u;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
          gt[g] += (int)s;
          if (pass == 3) eq[g] = (int)sm.all_h[g * 256 + dsel];
        }
      }
      if (lane == 0) {
        sm.scal[0] = (int)(prefix | ((uint32_t)dsel << shift));
        sm.scal[1] = (int)(mask | (255u << shift));
        sm.scal[2] = remaining - (int)above;
      }
    }
    __syncthreads();
    prefix = (uint32_t)sm.scal[0];
    mask = (uint32_t)sm.scal[1];
    remaining = sm.scal[2];
  }
  // ---- this face's share of the winners
  const uint32_t thr = prefix;
  int eq_before = 0, n_before = 0;
  for (int g = 0; g < face; ++g) {
    int take_g = remaining - eq_before;
    take_g = take_g < 0 ? 0 : (take_g > eq[g] ? eq[g] : take_g);
    n_before += gt[g] + take_g;
    eq_before += eq[g];
  }
  int take = remaining - eq_before;
  take = take < 0 ? 0 : (take > eq[face] ? eq[face] : take);
  uint64_t* dkey = cluster.map_shared_rank(sm.gkey, 0);
  Gathered* dval = cluster.map_shared_rank(sm.gval, 0);
  int base_tie = 0, base_sel = 0;
  for (int p0 = 0; p0 < SS; p0 += nt) {
    const int p = p0 + tid;
    const uint32_t k = p < SS ? sm.keys[p] : 0u;
    const bool is_tie = p < SS && k == thr;
    const bool is_gt = p < SS && k > thr;
    int n_tie;
    const int tie_rank = base_tie + block_rank(is_tie, sm.warp_tot, &n_tie);
    const bool sel = is_gt || (is_tie && tie_rank < take);
    int n_sel;
    const int sel_rank = base_sel + block_rank(sel, sm.warp_tot, &n_sel);
    if (sel) {
      const int slot = n_before + sel_rank;
      const int32_t flat = face * SS + p;
      // composite key: larger key first, then smaller index first
      dkey[slot] = ((uint64_t)k << 32) | (uint64_t)(0xFFFFFFFFu - (uint32_t)flat);
      dval[slot] = Gathered{sm.C[p * 3], sm.C[p * 3 + 1], sm.C[p * 3 + 2], flat};
    }
    base_tie += n_tie;
    base_sel += n_sel;
  }
  cluster.sync();
  // ---- rank the K winners (CTA 0)
  if (face == 0) {
    for (int e = tid; e < K; e += nt) {
      const uint64_t me = sm.gkey[e];
      int rank = 0;
      for (int o = 0; o < K; ++o) rank += sm.gkey[o] > me;
      const Gathered v = sm.gval[e];
      const size_t out = (size_t)env * K + rank;
      idx_out[out] = v.idx;
      st_out[out * 3 + 0] = v.r;
      st_out[out * 3 + 1] = v.g;
      st_out[out * 3 + 2] = v.b;
    }
  }
}

}  // namespace

size_t haar_topk_smem_bytes(int S, int K) { return smem_layout(S, K, nullptr, nullptr); }

void launch_haar_topk(const float* faces, int n_env, int S, int K, int32_t* idx, float* strength,
                      uint32_t* err, cudaStream_t st) {
  (void)err;
  if (n_env < 1 || n_env > (1 << 28)) fail(NWPRT_INVALID_ARG, "haar_topk: n_env out of range");
  if (S < 1 || S > kMaxS || (S & (S - 1)))
    fail(S > kMaxS ? NWPRT_UNSUPPORTED : NWPRT_INVALID_ARG,
         "haar_topk: face size must be a power of two <= 64");
  if (K < 1 || K > 6 * S * S || K > kMaxK)
    fail(NWPRT_INVALID_ARG, "haar_topk: K must be in [1, min(6*S*S, 1024)]");
  if (!faces || !idx || !strength) fail(NWPRT_INVALID_ARG, "haar_topk: null pointer");
  const size_t smem = haar_topk_smem_bytes(S, K);
  NWPRT_CUDA(cudaFuncSetAttribute(haar_topk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  haar_topk_kernel<<<6 * n_env, kThreads, smem, st>>>(faces, S, K, idx, strength);
  NWPRT_CUDA(cudaGetLastError());
}

}  // namespace nwprt

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
// memory: one bulk copy brings the face in, and every Haar level runs in place (operands
// to registers, barrier, results back).  The top-K threshold is found by a 4-pass 8-bit
// radix select: each CTA histograms its face, the cluster totals are summed through
// distributed shared memory (the six remote loads issued together), and every CTA scans
// the totals redundantly, so a pass costs one cluster barrier.  Ties at the threshold are
// taken in flat-index order (one ordered block scan over the tie flags); the winners are
// written into CTA 0's shared memory and ranked there.  Nothing but the inputs and
// outputs touches global memory.
#include <cooperative_groups.h>

#include "nwprt_internal.cuh"

namespace cg = cooperative_groups;

namespace nwprt {
namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxS = 64;
constexpr int kMaxK = 1024;
constexpr int kMaxPerThread = kMaxS * kMaxS / kThreads;            // keys per thread in the compaction
constexpr int kMaxLevelQuads = (kMaxS / 2) * (kMaxS / 2) / kThreads;  // 2x2 Haar blocks per thread

struct Gathered {
  float r, g, b;
  int32_t idx;
};

struct HaarSmem {
  float* C;         // [S][S][3] the face, then its coefficients (in place)
  uint32_t* keys;   // [S*S]
  uint32_t* hist;   // [2][256] this face's histogram of the pass (double buffered)
  uint32_t* all_h;  // [6][256] the cluster's histograms of the pass
  uint32_t* tot;    // [256] their sum
  uint64_t* gkey;   // [K] composite keys (CTA 0)
  Gathered* gval;   // [K]
  int* warp_tot;    // [kWarps]
  int* scal;        // scalars
  uint64_t* bar;    // bulk-copy completion
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline size_t smem_layout(int S, int K, char* base, HaarSmem* L) {
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o = align16(o + bytes); return at; };
  size_t oC = take(sizeof(float) * S * S * 3);
  size_t oK = take(sizeof(uint32_t) * S * S);
  size_t oH = take(sizeof(uint32_t) * 512);
  size_t oA = take(sizeof(uint32_t) * 6 * 256);
  size_t oT = take(sizeof(uint32_t) * 256);
  size_t oG = take(sizeof(uint64_t) * K);
  size_t oV = take(sizeof(Gathered) * K);
  size_t oW = take(sizeof(int) * kWarps);
  size_t oS = take(sizeof(int) * 32);
  size_t oB = take(sizeof(uint64_t));
  if (L) {
    L->C = (float*)(base + oC);
    L->keys = (uint32_t*)(base + oK);
    L->hist = (uint32_t*)(base + oH);
    L->all_h = (uint32_t*)(base + oA);
    L->tot = (uint32_t*)(base + oT);
    L->gkey = (uint64_t*)(base + oG);
    L->gval = (Gathered*)(base + oV);
    L->warp_tot = (int*)(base + oW);
    L->scal = (int*)(base + oS);
    L->bar = (uint64_t*)(base + oB);
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

// Exclusive prefix of `v` over the block's threads in thread order, plus the block total.
__device__ __forceinline__ int block_exclusive_sum(int v, int* warp_tot, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[warp] = incl;
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
  return before + incl - v;
}

__global__ void __cluster_dims__(6, 1, 1) __launch_bounds__(kThreads)
    haar_topk_kernel(const float* __restrict__ faces, int S, int K, int32_t* __restrict__ idx_out,
                     float* __restrict__ st_out, uint32_t* err) {
  extern __shared__ __align__(16) char smem_raw[];
  HaarSmem sm;
  smem_layout(S, K, smem_raw, &sm);
  cg::cluster_group cluster = cg::this_cluster();
  const int face = (int)cluster.block_rank();
  const int env = blockIdx.x / 6;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int SS = S * S;
  const float* src = faces + ((size_t)env * 6 + face) * (size_t)SS * 3;

  // ---- the face into shared memory: one bulk copy when the source allows it
  const uint32_t face_bytes = (uint32_t)SS * 12u;
  const bool bulk = ((reinterpret_cast<uintptr_t>(src) & 15) == 0) && (face_bytes % 16 == 0);
  if (bulk) {
    if (tid == 0) {
      mbar_init(sm.bar, 1);
      fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0) {
      mbar_arrive_expect_tx(sm.bar, face_bytes);
      bulk_g2s(sm.C, src, face_bytes, sm.bar);
    }
    // on a timeout the face reads as whatever is in shared memory; the error is reported
    // and every CTA still reaches the cluster barriers below
    mbar_wait(sm.bar, 0, err);
  } else {
    for (int e = tid; e < SS * 3; e += nt) sm.C[e] = __ldg(src + e);
    __syncthreads();
  }
  // ---- Haar levels n = S, S/2, ..., 2 in place on the top-left n x n block: each thread
  // reads its 2x2 blocks (3 channels, two 8-byte-aligned runs of 6 floats), then after a
  // barrier writes their LL, HL, LH, HH
  for (int n = S, lg = 0; n >= 2; n >>= 1) {
    const int h = n >> 1;
    while ((1 << lg) < h) ++lg;
    while ((1 << lg) > h) --lg;
    float in[kMaxLevelQuads][12];
#pragma unroll
    for (int u = 0; u < kMaxLevelQuads; ++u) {
      const int b = tid + u * nt;
      if (b < h * h) {
        const int i = b >> lg, j = b & (h - 1);
        const float2* r0 = reinterpret_cast<const float2*>(sm.C + ((2 * i) * S + 2 * j) * 3);
        const float2* r1 = reinterpret_cast<const float2*>(sm.C + ((2 * i + 1) * S + 2 * j) * 3);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const float2 x = r0[q], y = r1[q];
          in[u][2 * q] = x.x;
          in[u][2 * q + 1] = x.y;
          in[u][6 + 2 * q] = y.x;
          in[u][6 + 2 * q + 1] = y.y;
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kMaxLevelQuads; ++u) {
      const int b = tid + u * nt;
      if (b < h * h) {
        const int i = b >> lg, j = b & (h - 1);
        // in[]: row 2i = (px 2j: r g b, px 2j+1: r g b), then row 2i+1 likewise
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float ll, hl, lh, hh;
          haar4(in[u][c], in[u][3 + c], in[u][6 + c], in[u][9 + c], ll, hl, lh, hh);
          sm.C[(i * S + j) * 3 + c] = ll;
          sm.C[(i * S + j + h) * 3 + c] = hl;
          sm.C[((i + h) * S + j) * 3 + c] = lh;
          sm.C[((i + h) * S + j + h) * 3 + c] = hh;
        }
      }
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
    // buffer (pass & 1) was last read remotely in pass - 2, before the previous cluster barrier
    for (int d = tid; d < 256; d += nt) h[d] = 0;
    __syncthreads();
    for (int p = tid; p < SS; p += nt) {
      const uint32_t k = sm.keys[p];
      if ((k & mask) == prefix) atomicAdd(&h[(k >> shift) & 255u], 1u);
    }
    cluster.sync();
    if (tid < 256) {
      uint32_t v[6];
#pragma unroll
      for (int g = 0; g < 6; ++g) v[g] = cluster.map_shared_rank(h, g)[tid];
      uint32_t t = 0;
#pragma unroll
      for (int g = 0; g < 6; ++g) {
        sm.all_h[g * 256 + tid] = v[g];
        t += v[g];
      }
      sm.tot[tid] = t;
    }
    __syncthreads();
    if (warp == 0) {
      // lane l covers digits 255-8l .. 248-8l (highest digits first)
      const int d_hi = 255 - 8 * lane;
      uint32_t tot8[8];
      uint32_t local = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        tot8[q] = sm.tot[d_hi - q];
        local += tot8[q];
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
      if (lane == 0) {
        sm.scal[0] = (int)(prefix | ((uint32_t)dsel << shift));
        sm.scal[1] = (int)(mask | (255u << shift));
        sm.scal[2] = remaining - (int)above;
        sm.scal[3] = dsel;
      }
    }
    __syncthreads();
    prefix = (uint32_t)sm.scal[0];
    mask = (uint32_t)sm.scal[1];
    remaining = sm.scal[2];
    // per-face counts of keys whose digit is above the selected one (warp g: face g)
    if (warp < 6) {
      const int dsel = sm.scal[3];
      const int d_hi = 255 - 8 * lane;
      uint32_t s = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int d = d_hi - q;
        s += d > dsel ? sm.all_h[warp * 256 + d] : 0u;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) {
        gt[warp] += (int)s;
        if (pass == 3) eq[warp] = (int)sm.all_h[warp * 256 + dsel];
      }
    }
    // the next pass starts with a barrier; the loop's last one follows below
  }
  __syncthreads();
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
  // thread t owns keys [t*per, t*per + per): ties get their flat-index rank from one
  // ordered scan; the winners' slots in CTA 0 only need to be distinct (the final rank
  // orders them), so they come from a shared counter
  const int per = (SS + nt - 1) / nt;
  const int p0 = tid * per;
  int n_tie_mine = 0;
#pragma unroll
  for (int u = 0; u < kMaxPerThread; ++u) {
    const int p = p0 + u;
    if (u < per && p < SS && sm.keys[p] == thr) ++n_tie_mine;
  }
  int *counter = sm.scal + 24;
  if (tid == 0) *counter = 0;
  int n_tie_all;
  int tie_rank = block_exclusive_sum(n_tie_mine, sm.warp_tot, &n_tie_all);
#pragma unroll
  for (int u = 0; u < kMaxPerThread; ++u) {
    const int p = p0 + u;
    if (u >= per || p >= SS) continue;
    const uint32_t k = sm.keys[p];
    bool sel = k > thr;
    if (k == thr) sel = tie_rank++ < take;
    if (sel) {
      const int slot = n_before + atomicAdd(counter, 1);
      const int32_t flat = face * SS + p;
      // composite key: larger key first, then smaller index first
      dkey[slot] = ((uint64_t)k << 32) | (uint64_t)(0xFFFFFFFFu - (uint32_t)flat);
      dval[slot] = Gathered{sm.C[p * 3], sm.C[p * 3 + 1], sm.C[p * 3 + 2], flat};
    }
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
  if (n_env < 1 || n_env > (1 << 28)) fail(NWPRT_INVALID_ARG, "haar_topk: n_env out of range");
  if (S < 1 || S > kMaxS || (S & (S - 1)))
    fail(S > kMaxS ? NWPRT_UNSUPPORTED : NWPRT_INVALID_ARG,
         "haar_topk: face size must be a power of two <= 64");
  if (K < 1 || K > 6 * S * S || K > kMaxK)
    fail(NWPRT_INVALID_ARG, "haar_topk: K must be in [1, min(6*S*S, 1024)]");
  if (!faces || !idx || !strength) fail(NWPRT_INVALID_ARG, "haar_topk: null pointer");
  const size_t smem = haar_topk_smem_bytes(S, K);
  NWPRT_CUDA(cudaFuncSetAttribute(haar_topk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  haar_topk_kernel<<<6 * n_env, kThreads, smem, st>>>(faces, S, K, idx, strength, err);
  NWPRT_CUDA(cudaGetLastError());
}

}  // namespace nwprt

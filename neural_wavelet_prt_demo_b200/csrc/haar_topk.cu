// Cubemap Haar transform + top-K wavelet selection: one thread-block cluster per env map for
// single maps and small batches, one persistent CTA per map for batches of 32 maps or more
// (haar_topk_batch_kernel, described where it is defined).
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
// Cluster form: 6 CTAs (one per face) of 256 threads.  Nothing but the inputs and outputs
// touches global memory, and the face never goes through shared memory:
//  * Haar in registers.  Thread t owns the 4x4 texel block at block coordinates
//    (bi, bj) = Morton(t) (bj on the even bits) and evaluates the first two levels on it
//    alone: 15 detail coefficients stay in its registers, one LL value moves on.  Because
//    the LL grid is held in Morton order, every 2x2 block of the next level sits in 4
//    consecutive lanes and the next 16 in one warp, so two more levels are warp shuffles.
//    The (at most 16) LL values left go through shared memory to warp 0, which finishes
//    the last levels the same way: one block barrier for the whole transform.  The
//    coefficients of those upper levels fill exactly the top-left (S/4)^2 block of the
//    face, one per thread, so each thread owns 16 coefficients.
//  * 4-pass 8-bit radix select of the K-th largest key over the cluster: each CTA
//    histograms its keys (registers -> shared atomics), the six histograms are summed
//    through distributed shared memory after one cluster barrier, and one block scan over
//    the totals (thread t = digit 255 - t) finds the digit.
//  * Ties at the threshold are ranked by flat index with a per-face bitmap and popcount
//    prefixes; the per-face tie counts come from the last pass's histograms.
//  * Winners get slots from one counter in CTA 0 (one atomic per warp) and are written to
//    all six CTAs, so each CTA ranks a sixth of them (one warp per winner) and writes
//    their outputs.
#include <cooperative_groups.h>

#include <mutex>

#include "nwprt_internal.cuh"

namespace cg = cooperative_groups;

namespace nwprt {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxS = 64;
constexpr int kMaxK = 1024;

struct Winner {
  float r, g, b;
  int32_t idx;
};

struct HaarSmem {
  uint32_t* hist;    // [2][256] this face's histogram of the pass (double buffered)
  float* upper;      // [(S/4)^2][3] coefficients of the top-left (S/4)^2 block
  float* llg;        // [16][3] LL values handed to warp 0 for the last levels
  uint32_t* bits;    // [S*S/32] ties at the threshold, by flat index within the face
  uint32_t* wpre;    // [S*S/32] exclusive popcount prefix of `bits`
  uint64_t* gkey;    // [K] composite keys of the winners (every CTA holds all of them)
  Winner* gval;      // [K]
  int* warp_tot;     // [kWarps]
  int* scal;         // scalars
};

// scal[] slots
constexpr int kScPrefix = 0, kScMask = 1, kScRemaining = 2, kScCounter = 3, kScEq = 8;  // eq: [6]
constexpr int kScNAbove = 16, kScNCand = 17;  // batched kernel: winners above the window bin, candidates in it
// Candidates (keys in the window's selected bin) the batched kernel ranks directly; they share
// the histogram region: composite keys (8 B) + ids (4 B).
constexpr int kCandCap = 680;

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline size_t smem_layout(int S, int K, char* base, HaarSmem* L) {
  const int G = S < 4 ? 1 : S / 4;
  const int nw = (S * S + 31) / 32;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o = align16(o + bytes); return at; };
  size_t oH = take(sizeof(uint32_t) * 512);
  size_t oU = take(sizeof(float) * 3 * G * G);
  size_t oL = take(sizeof(float) * 3 * 16);
  size_t oB = take(sizeof(uint32_t) * nw);
  size_t oP = take(sizeof(uint32_t) * nw);
  size_t oG = take(sizeof(uint64_t) * K);
  size_t oV = take(sizeof(Winner) * K);
  size_t oW = take(sizeof(int) * kWarps);
  size_t oS = take(sizeof(int) * 32);
  if (L) {
    L->hist = (uint32_t*)(base + oH);
    L->upper = (float*)(base + oU);
    L->llg = (float*)(base + oL);
    L->bits = (uint32_t*)(base + oB);
    L->wpre = (uint32_t*)(base + oP);
    L->gkey = (uint64_t*)(base + oG);
    L->gval = (Winner*)(base + oV);
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

// Bits 0, 2, 4, 6 of x packed into bits 0..3 (Morton decode of one coordinate).
__device__ __forceinline__ int morton_even(int x) {
  x &= 0x55;
  x = (x | (x >> 1)) & 0x33;
  x = (x | (x >> 2)) & 0x0f;
  return x;
}

// Inclusive prefix of `v` over the block's threads in thread order (a block of NWARPS warps);
// `total` = block sum.
template <int NWARPS = kWarps>
__device__ __forceinline__ uint32_t block_inclusive_sum(uint32_t v, int* warp_tot, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[warp] = (int)incl;
  __syncthreads();
  uint32_t before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < NWARPS; ++w) {
    const uint32_t t = (uint32_t)warp_tot[w];
    before += (w < warp) ? t : 0u;
    all += t;
  }
  __syncthreads();
  *total = all;
  return before + incl;
}

// One level of the transform over LL values held in Morton order by the lanes of a warp:
// the 2x2 block of LL grid positions (2i..2i+1, 2j..2j+1) is held by lanes
// base, base + s, base + 2s, base + 3s (a = (2i,2j), b = (2i,2j+1), c = (2i+1,2j),
// d = (2i+1,2j+1)).  The leader lane (base) keeps LL; the three details go to `upper` at
// (i, j+h), (i+h, j), (i+h, j+h) of the G x G upper block, h = the new LL side.
__device__ __forceinline__ void shuffle_level(float ll[3], int lane, int s, int m, int h, bool live,
                                              float* upper, int G) {
  float v[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    v[0][c] = __shfl_down_sync(0xffffffffu, ll[c], s);
    v[1][c] = __shfl_down_sync(0xffffffffu, ll[c], 2 * s);
    v[2][c] = __shfl_down_sync(0xffffffffu, ll[c], 3 * s);
  }
  if (live && (lane & (4 * s - 1)) == 0) {
    const int j = morton_even(m), i = morton_even(m >> 1);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float a, hl, lh, hh;
      haar4(ll[c], v[0][c], v[1][c], v[2][c], a, hl, lh, hh);
      ll[c] = a;
      upper[(i * G + j + h) * 3 + c] = hl;
      upper[((i + h) * G + j) * 3 + c] = lh;
      upper[((i + h) * G + j + h) * 3 + c] = hh;
    }
  }
}

// shuffle_level with the details stored to a face's scratch slice, laid out [channel][thread]
// (thread i * G + j owns upper-block entry (i, j)).
__device__ __forceinline__ void shuffle_level_scratch(float ll[3], int lane, int s, int m, int h, bool live,
                                                      float* upf, int G) {
  float v[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    v[0][c] = __shfl_down_sync(0xffffffffu, ll[c], s);
    v[1][c] = __shfl_down_sync(0xffffffffu, ll[c], 2 * s);
    v[2][c] = __shfl_down_sync(0xffffffffu, ll[c], 3 * s);
  }
  if (live && (lane & (4 * s - 1)) == 0) {
    const int j = morton_even(m), i = morton_even(m >> 1);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float a, hl, lh, hh;
      haar4(ll[c], v[0][c], v[1][c], v[2][c], a, hl, lh, hh);
      ll[c] = a;
      upf[c * 256 + i * G + j + h] = hl;
      upf[c * 256 + (i + h) * G + j] = lh;
      upf[c * 256 + (i + h) * G + j + h] = hh;
    }
  }
}

// Geometry of one face's transform: thread t < T owns the B x B texel block at Morton(t).
template <int S>
struct FaceGeom {
  static constexpr int B = S < 4 ? S : 4;   // texel block per thread: B x B
  static constexpr int G = S / B;           // thread blocks per face side; the upper block is G x G
  static constexpr int T = G * G;           // threads holding coefficients
  static constexpr int SS = S * S;
  static constexpr int NR = B == 4 ? 15 : (B == 2 ? 3 : 0);  // coefficients held in registers
  static constexpr int NK = NR + 1;                         // plus one entry of the upper block
};

// Index within the face of thread tid's coefficient u (u == NR: its upper-block entry).
template <int S>
__device__ __forceinline__ int flat_in_face(int tid, int u) {
  using F = FaceGeom<S>;
  if (u == F::NR) return (tid / F::G) * S + (tid % F::G);
  int i = 0, j = 0, h = 1;
  if constexpr (F::B == 4) {
    const int bj = morton_even(tid), bi = morton_even(tid >> 1);
    const int q = u / 3;
    i = q < 4 ? 2 * bi + (q >> 1) : bi;
    j = q < 4 ? 2 * bj + (q & 1) : bj;
    h = q < 4 ? S / 2 : S / 4;
  }
  const int band = u % 3;
  return band == 0 ? i * S + j + h : (band == 1 ? (i + h) * S + j : (i + h) * S + j + h);
}

// Coefficient u < NR of thread tid's texel block (all three channels), recomputed from the
// face at `src` with the same FP32 operations, in the same order, as the transform below:
// a level-1 detail from its 2x2 quad, a level-2 detail from the four quads' LL values.  The
// batched kernel keeps no copy of these coefficients; it recomputes the K winners' instead.
template <int S>
__device__ __forceinline__ void block_coef(const float* __restrict__ src, int tid, int u, float (&out)[3]) {
  using F = FaceGeom<S>;
  const int bj = morton_even(tid), bi = morton_even(tid >> 1);
  const float* blk = src + ((size_t)(F::B * bi) * S + F::B * bj) * 3;
  const int q = u / 3, band = u % 3;
  auto quad = [&](int qi, int qj, int c, float& a, float& hl, float& lh, float& hh) {
    const float* p0 = blk + ((size_t)(2 * qi) * S + 2 * qj) * 3 + c;
    haar4(__ldg(p0), __ldg(p0 + 3), __ldg(p0 + S * 3), __ldg(p0 + S * 3 + 3), a, hl, lh, hh);
  };
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float a, hl, lh, hh;
    if (q < 4) {
      quad(q >> 1, q & 1, c, a, hl, lh, hh);
    } else {
      float l1[4], x, y, z;
#pragma unroll
      for (int k = 0; k < 4; ++k) quad(k >> 1, k & 1, c, l1[k], x, y, z);
      haar4(l1[0], l1[1], l1[2], l1[3], a, hl, lh, hh);
    }
    out[c] = band == 0 ? hl : (band == 1 ? lh : hh);
  }
}

// The first part of the transform below, split out for the batched form: block_load loads
// thread t's B x B texel block (t < T), block_levels runs levels 1-2 on it in registers (co:
// its NR detail coefficients, ll: the block's LL value), with the same operations in the same
// order as haar_face_in_registers.
template <int S>
__device__ __forceinline__ void block_load(const float* __restrict__ src, int tid,
                                           float (&px)[FaceGeom<S>::B][FaceGeom<S>::B][3]) {
  using F = FaceGeom<S>;
  constexpr int B = F::B;
  if (tid >= F::T) return;
  const int bj = morton_even(tid), bi = morton_even(tid >> 1);
  const float* blk = src + ((size_t)(B * bi) * S + B * bj) * 3;
  if constexpr (B == 4) {
    if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const float4* row = reinterpret_cast<const float4*>(blk + (size_t)r * S * 3);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const float4 v = __ldg(row + q);
          const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
          for (int k = 0; k < 4; ++k) px[r][(4 * q + k) / 3][(4 * q + k) % 3] = e[k];
        }
      }
    } else {
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 12; ++q) px[r][q / 3][q % 3] = __ldg(blk + (size_t)r * S * 3 + q);
    }
  } else {
#pragma unroll
    for (int r = 0; r < B; ++r)
#pragma unroll
      for (int q = 0; q < 3 * B; ++q) px[r][q / 3][q % 3] = __ldg(blk + (size_t)r * S * 3 + q);
  }
}

template <int S>
__device__ __forceinline__ void block_levels(const float (&px)[FaceGeom<S>::B][FaceGeom<S>::B][3], int tid,
                                             float (&co)[FaceGeom<S>::NR > 0 ? FaceGeom<S>::NR : 1][3],
                                             float (&ll)[3]) {
  using F = FaceGeom<S>;
  constexpr int B = F::B, NR = F::NR;
#pragma unroll
  for (int u = 0; u < (NR > 0 ? NR : 1); ++u) co[u][0] = co[u][1] = co[u][2] = 0.f;
  ll[0] = ll[1] = ll[2] = 0.f;
  if (tid >= F::T) return;
  if constexpr (B == 4) {
    float l1[2][2][3];
#pragma unroll
    for (int qi = 0; qi < 2; ++qi)
#pragma unroll
      for (int qj = 0; qj < 2; ++qj)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float a, hl, lh, hh;
          haar4(px[2 * qi][2 * qj][c], px[2 * qi][2 * qj + 1][c], px[2 * qi + 1][2 * qj][c],
                px[2 * qi + 1][2 * qj + 1][c], a, hl, lh, hh);
          l1[qi][qj][c] = a;
          const int u = (qi * 2 + qj) * 3;
          co[u][c] = hl;
          co[u + 1][c] = lh;
          co[u + 2][c] = hh;
        }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float a, hl, lh, hh;
      haar4(l1[0][0][c], l1[0][1][c], l1[1][0][c], l1[1][1][c], a, hl, lh, hh);
      ll[c] = a;
      co[12][c] = hl;
      co[13][c] = lh;
      co[14][c] = hh;
    }
  } else if constexpr (B == 2) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float a, hl, lh, hh;
      haar4(px[0][0][c], px[0][1][c], px[1][0][c], px[1][1][c], a, hl, lh, hh);
      ll[c] = a;
      co[0][c] = hl;
      co[1][c] = lh;
      co[2][c] = hh;
    }
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) ll[c] = px[0][0][c];
  }
}

// The full Haar transform of one face [S][S][3] at `src` by the block's kThreads threads:
// levels 1-2 on each thread's B x B block in registers (co: its NR detail coefficients),
// the next levels by warp shuffles, the last ones in warp 0.  The G x G upper block of the
// result (levels >= 3 and the DC term) lands in `upper` [G*G][3]; `llg` is [16][3] staging.
// Ends with a block barrier, after which `upper` is complete.
template <int S>
__device__ __forceinline__ void haar_face_in_registers(const float* __restrict__ src, int tid,
                                                       float (&co)[FaceGeom<S>::NR > 0 ? FaceGeom<S>::NR : 1][3],
                                                       float* upper, float* llg) {
  using F = FaceGeom<S>;
  constexpr int G = F::G;
  const int lane = tid & 31, warp = tid >> 5;
  const bool owner = tid < F::T;
  float ll[3];
  {
    float px[F::B][F::B][3];
    block_load<S>(src, tid, px);
    block_levels<S>(px, tid, co, ll);
  }
  // ---- the remaining levels over the G x G LL grid, held in Morton order by threads 0..T-1
  {
    int n = G, s = 1;  // LL grid side; lane stride between the values of one 2x2 block
#pragma unroll
    for (int lev = 0; lev < 2; ++lev)
      if (n >= 2) {
        shuffle_level(ll, lane, s, tid / (4 * s), n / 2, owner, upper, G);
        n /= 2;
        s *= 4;
      }
    if (n >= 2) {
      // at most 4 x 4 values left: leaders hand them to warp 0
      if (owner && (tid & (s - 1)) == 0)
#pragma unroll
        for (int c = 0; c < 3; ++c) llg[(tid / s) * 3 + c] = ll[c];
      __syncthreads();
      if (warp == 0) {
        const bool live = lane < n * n;
#pragma unroll
        for (int c = 0; c < 3; ++c) ll[c] = live ? llg[lane * 3 + c] : 0.f;
        int s2 = 1;
#pragma unroll
        for (int lev = 0; lev < 2; ++lev)
          if (n >= 2) {
            shuffle_level(ll, lane, s2, lane / (4 * s2), n / 2, live, upper, G);
            n /= 2;
            s2 *= 4;
          }
        if (lane == 0)
#pragma unroll
          for (int c = 0; c < 3; ++c) upper[c] = ll[c];
      }
    } else if (tid == 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) upper[c] = ll[c];
    }
  }
  __syncthreads();
}

template <int S>
// Two CTAs per SM at most: this form serves batches under kBatchMinMaps (at most 186 CTAs
// on 148 SMs), and the bound leaves the transform its registers (three per SM spilled).
__global__ void __cluster_dims__(6, 1, 1) __launch_bounds__(kThreads, 2)
    haar_topk_kernel(const float* __restrict__ faces, int K, int32_t* __restrict__ idx_out,
                     float* __restrict__ st_out) {
  using F = FaceGeom<S>;
  constexpr int T = F::T, SS = F::SS, NR = F::NR;
  constexpr int NW = (SS + 31) / 32;
  static_assert(T <= kThreads, "one 4x4 block per thread");

  extern __shared__ __align__(16) char smem_raw[];
  HaarSmem sm;
  smem_layout(S, K, smem_raw, &sm);
  cg::cluster_group cluster = cg::this_cluster();
  const int face = (int)cluster.block_rank();
  const int env = blockIdx.x / 6;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const float* src = faces + ((size_t)env * 6 + face) * (size_t)SS * 3;
  const bool owner = tid < T;

  if (face == 0 && tid == 0) sm.scal[kScCounter] = 0;  // winner slots (read after 5 cluster barriers)
  for (int w = tid; w < NW; w += kThreads) sm.bits[w] = 0u;

  // ---- the transform: levels 1-2 in registers, the rest by shuffles and warp 0
  float co[NR > 0 ? NR : 1][3];  // detail coefficients held in registers (RGB)
  haar_face_in_registers<S>(src, tid, co, sm.upper, sm.llg);
  // ---- this thread's 16 coefficients: NR in registers, one of the upper block
  constexpr int NK = F::NK;
  auto flat_of = [&](int u) -> int { return flat_in_face<S>(tid, u); };
  uint32_t key[NK];
#pragma unroll
  for (int u = 0; u < NR; ++u) key[u] = wavelet_key_bits(co[u][0], co[u][1], co[u][2]);
  float ur = 0.f, ug = 0.f, ub = 0.f;
  if (owner) {
    ur = sm.upper[tid * 3];
    ug = sm.upper[tid * 3 + 1];
    ub = sm.upper[tid * 3 + 2];
  }
  key[NR] = wavelet_key_bits(ur, ug, ub);

  // ---- 4-pass radix select of the K-th largest key over the whole cluster
  uint32_t prefix = 0, mask = 0;
  int remaining = K;
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = 24 - 8 * pass;
    uint32_t* h = sm.hist + (pass & 1) * 256;
    // buffer (pass & 1) was last read remotely in pass - 2, before the previous cluster barrier
    h[tid] = 0u;
    __syncthreads();
    if (owner)
#pragma unroll
      for (int u = 0; u < NK; ++u)
        if ((key[u] & mask) == prefix) atomicAdd(&h[(key[u] >> shift) & 255u], 1u);
    cluster.sync();
    const int digit = 255 - tid;  // thread order = digits from the top
    uint32_t v[6], tot = 0;
#pragma unroll
    for (int g = 0; g < 6; ++g) v[g] = cluster.map_shared_rank(h, g)[digit];
#pragma unroll
    for (int g = 0; g < 6; ++g) tot += v[g];
    uint32_t all;
    const uint32_t incl = block_inclusive_sum(tot, sm.warp_tot, &all);
    if (incl >= (uint32_t)remaining && incl - tot < (uint32_t)remaining) {
      sm.scal[kScPrefix] = (int)(prefix | ((uint32_t)digit << shift));
      sm.scal[kScMask] = (int)(mask | (255u << shift));
      sm.scal[kScRemaining] = remaining - (int)(incl - tot);
      if (pass == 3)
#pragma unroll
        for (int g = 0; g < 6; ++g) sm.scal[kScEq + g] = (int)v[g];
    }
    __syncthreads();
    prefix = (uint32_t)sm.scal[kScPrefix];
    mask = (uint32_t)sm.scal[kScMask];
    remaining = sm.scal[kScRemaining];
  }
  // ---- ties at the threshold, taken in flat-index order (faces in order)
  const uint32_t thr = prefix;
  int eq_before = 0;
  for (int g = 0; g < face; ++g) eq_before += sm.scal[kScEq + g];
  if (owner)
#pragma unroll
    for (int u = 0; u < NK; ++u)
      if (key[u] == thr) {
        const int f = flat_of(u);
        atomicOr(&sm.bits[f >> 5], 1u << (f & 31));
      }
  __syncthreads();
  {
    uint32_t all;
    const uint32_t c = tid < NW ? (uint32_t)__popc(sm.bits[tid]) : 0u;
    const uint32_t incl = block_inclusive_sum(c, sm.warp_tot, &all);
    if (tid < NW) sm.wpre[tid] = incl - c;
  }
  __syncthreads();
  // ---- winners: slots from CTA 0's counter (one atomic per warp), stored in every CTA
  uint32_t selmask = 0;
  int n_sel = 0;
  if (owner)
#pragma unroll
    for (int u = 0; u < NK; ++u) {
      bool sel = key[u] > thr;
      if (key[u] == thr) {
        const int f = flat_of(u), w = f >> 5;
        const int rank = eq_before + (int)sm.wpre[w] + __popc(sm.bits[w] & ((1u << (f & 31)) - 1u));
        sel = rank < remaining;
      }
      if (sel) {
        selmask |= 1u << u;
        ++n_sel;
      }
    }
  int incl_w = n_sel;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl_w, o);
    if (lane >= o) incl_w += t;
  }
  int base = 0;
  if (lane == 31 && incl_w > 0) base = atomicAdd(cluster.map_shared_rank(&sm.scal[kScCounter], 0), incl_w);
  base = __shfl_sync(0xffffffffu, base, 31);
  int slot = base + incl_w - n_sel;
  if (selmask) {
#pragma unroll
    for (int u = 0; u < NK; ++u)
      if (selmask & (1u << u)) {
        const int32_t gflat = face * SS + flat_of(u);
        // composite key: larger key first, then smaller index first
        const uint64_t ck = ((uint64_t)key[u] << 32) | (uint64_t)(0xFFFFFFFFu - (uint32_t)gflat);
        Winner wv;
        if (u < NR) {
          wv = Winner{co[u][0], co[u][1], co[u][2], gflat};
        } else {
          wv = Winner{ur, ug, ub, gflat};
        }
#pragma unroll
        for (int g = 0; g < 6; ++g) {
          cluster.map_shared_rank(sm.gkey, g)[slot] = ck;
          cluster.map_shared_rank(sm.gval, g)[slot] = wv;
        }
        ++slot;
      }
  }
  cluster.sync();
  // ---- rank the K winners: CTA f takes winners f, f + 6, ...; one warp per winner
  for (int e = face + 6 * warp; e < K; e += 6 * kWarps) {
    const uint64_t me = sm.gkey[e];
    int rank = 0;
    for (int o = lane; o < K; o += 32) rank += sm.gkey[o] > me;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) rank += __shfl_xor_sync(0xffffffffu, rank, o);
    if (lane == 0) {
      const Winner wv = sm.gval[e];
      const size_t out = (size_t)env * K + rank;
      idx_out[out] = wv.idx;
      st_out[out * 3 + 0] = wv.r;
      st_out[out * 3 + 1] = wv.g;
      st_out[out * 3 + 2] = wv.b;
    }
  }
}

// ------------------------------------------------------------------ batched form
// One persistent CTA per map at a time (no cluster): for large batches, whole maps in flight
// per SM beat the cluster's one sixth of a map each, and no step crosses an SM.  Faces are
// transformed one after another with the same register code; the keys of all six stay in
// shared memory (uint4 of four keys, thread-fastest: conflict-free).  Of the coefficients
// only each thread's upper-block entry is kept, in this CTA's slice of a global scratch
// buffer ([face][channel][thread], 18 KB at S = 64, so it stays in L2); the K winners' other
// coefficients are recomputed from their texel blocks (block_coef), which costs far less
// than writing and re-reading all 6 * S * S of them.  The select is block-local: a first
// histogram pass over a window of 16 binades below the map's largest key; when that finds the
// K-th largest key's bin, one scan sorts the keys above it (winners) from those in it
// (candidates, ranked directly); otherwise radix passes, a bitmap of ties over the 6*S*S flat
// indices and winner slots from one block scan.  The winners are ordered by a counting pass
// over their key range.  The faces need no block barrier between them: levels 1-2 are
// thread-local, levels 3-4 (warp shuffles) write their details straight to the scratch slice,
// and the last levels of all six faces run after one barrier, in warps 0-5.

struct BatchSmem {
  uint4* keys;      // [6][NK/4][kThreads]
  uint32_t* whist;  // [kWarps][256] per-warp histograms of a pass
  uint32_t* bits;   // [6*S*S/32] ties (aliases whist after the passes)
  uint32_t* wpre;   // [6*S*S/32]
  uint64_t* gkey;   // [K]
  int* gid;         // [K] winner: (face * NK + u) * kThreads + thread
  float* llg;       // [6][16][3] each face's LL values left for its last levels
  int* warp_tot;
  int* scal;
};

__host__ __device__ inline size_t batch_smem_layout(int S, int K, char* base, BatchSmem* L) {
  const int nk = S >= 4 ? 16 : (S == 2 ? 4 : 1);
  const int nkq = (nk + 3) / 4;
  const int nw = (6 * S * S + 31) / 32;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o = align16(o + bytes); return at; };
  const size_t oK = take(sizeof(uint4) * 6 * nkq * kThreads);
  const size_t uA = sizeof(uint32_t) * kWarps * 256, uB = sizeof(uint32_t) * 2 * nw;
  const size_t oH = take(uA > uB ? uA : uB);
  const size_t oG = take(sizeof(uint64_t) * K);
  const size_t oI = take(sizeof(int) * K);
  const size_t oL = take(sizeof(float) * 3 * 16 * 6);
  const size_t oW = take(sizeof(int) * kWarps);
  const size_t oS = take(sizeof(int) * 32);
  if (L) {
    L->keys = (uint4*)(base + oK);
    L->whist = (uint32_t*)(base + oH);
    L->bits = (uint32_t*)(base + oH);
    L->wpre = (uint32_t*)(base + oH) + nw;
    L->gkey = (uint64_t*)(base + oG);
    L->gid = (int*)(base + oI);
    L->llg = (float*)(base + oL);
    L->warp_tot = (int*)(base + oW);
    L->scal = (int*)(base + oS);
  }
  return o;
}

template <int S>
__host__ __device__ constexpr size_t batch_scratch_floats_per_cta() {
  return (size_t)6 * 3 * kThreads;
}

template <int S>
__global__ void __launch_bounds__(kThreads, 2)
    haar_topk_batch_kernel(const float* __restrict__ faces, int n_env, int K, int32_t* __restrict__ idx_out,
                           float* __restrict__ st_out, float* __restrict__ scratch) {
  using F = FaceGeom<S>;
  constexpr int T = F::T, SS = F::SS, NR = F::NR, NK = F::NK;
  constexpr int NKQ = (NK + 3) / 4;
  constexpr int NW = (6 * SS + 31) / 32;
  static_assert(T <= kThreads, "one 4x4 block per thread");
  static_assert(kThreads == 256, "one thread per bin of the winners' counting pass");
  static_assert(512 * sizeof(uint32_t) + kMaxK * sizeof(uint16_t) <= kWarps * 256 * sizeof(uint32_t),
                "the winners' bins and order fit the histogram region");
  extern __shared__ __align__(16) char smem_raw[];
  BatchSmem sm;
  batch_smem_layout(S, K, smem_raw, &sm);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool owner = tid < T;
  // this CTA's upper-block entries, [face][channel][thread]
  float* up = scratch + (size_t)blockIdx.x * batch_scratch_floats_per_cta<S>();

  for (int env = blockIdx.x; env < n_env; env += gridDim.x) {
    // ---- the six transforms, with no block barrier between faces: levels 1-2 in registers
    // (their 15 keys straight to shared memory), levels 3-4 by warp shuffles whose details go
    // to this face's scratch slice, the LL values left over to shared staging.  After all six,
    // warp f finishes face f's last levels; then every thread reads its own six upper-block
    // entries and forms their keys.  Each thread keeps the largest key it formed.
    uint32_t kmax = 0;
    constexpr int G = F::G;
    constexpr int NL = G >= 8 ? G / 4 : 1;  // side of the LL grid left after levels 3-4
    for (int f = 0; f < 6; ++f) {
      const float* src = faces + ((size_t)env * 6 + f) * (size_t)SS * 3;
      // the next face (after the sixth: this CTA's next map's first) into L2 meanwhile
      if (tid == 0 && (SS * 12) % 16 == 0) {
        const long long nxt = (long long)env * 6 + f + 1 + (f == 5 ? (long long)(gridDim.x - 1) * 6 : 0);
        const float* pf = faces + (size_t)nxt * SS * 3;
        if (nxt < (long long)n_env * 6 && (reinterpret_cast<uintptr_t>(pf) & 15) == 0)
          asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(pf), "r"((uint32_t)(SS * 12)) : "memory");
      }
      float* upf = up + f * 3 * kThreads;
      uint32_t k[NKQ * 4];
#pragma unroll
      for (int u = 0; u < NKQ * 4; ++u) k[u] = 0u;
      float ll[3];
      {
        float px[F::B][F::B][3];
        float co[NR > 0 ? NR : 1][3];
        block_load<S>(src, tid, px);
        block_levels<S>(px, tid, co, ll);
        if (owner)
#pragma unroll
          for (int u = 0; u < NR; ++u) {
            k[u] = wavelet_key_bits(co[u][0], co[u][1], co[u][2]);
            kmax = max(kmax, k[u]);
          }
      }
#pragma unroll
      for (int q = 0; q < NKQ; ++q)
        sm.keys[((size_t)f * NKQ + q) * kThreads + tid] = make_uint4(k[4 * q], k[4 * q + 1], k[4 * q + 2], k[4 * q + 3]);
      int n = G, st_ = 1;
#pragma unroll
      for (int lev = 0; lev < 2; ++lev)
        if (n >= 2) {
          shuffle_level_scratch(ll, lane, st_, tid / (4 * st_), n / 2, owner, upf, G);
          n /= 2;
          st_ *= 4;
        }
      if (n >= 2) {
        if (owner && (tid & (st_ - 1)) == 0)
#pragma unroll
          for (int c = 0; c < 3; ++c) sm.llg[(f * 16 + tid / st_) * 3 + c] = ll[c];
      } else if (tid == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) upf[c * kThreads] = ll[c];  // the DC term
      }
    }
    __syncthreads();  // every face's level-3/4 details and LL staging are written
    if constexpr (NL >= 2) {
      if (warp < 6) {
        const int f = warp;
        float* upf = up + f * 3 * kThreads;
        const bool live = lane < NL * NL;
        float ll[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) ll[c] = live ? sm.llg[(f * 16 + lane) * 3 + c] : 0.f;
        int n = NL, s2 = 1;
#pragma unroll
        for (int lev = 0; lev < 2; ++lev)
          if (n >= 2) {
            shuffle_level_scratch(ll, lane, s2, lane / (4 * s2), n / 2, live, upf, G);
            n /= 2;
            s2 *= 4;
          }
        if (lane == 0)
#pragma unroll
          for (int c = 0; c < 3; ++c) upf[c * kThreads] = ll[c];  // the DC term
      }
      __syncthreads();  // the last levels' details are written
    }
    if (owner)
      for (int f = 0; f < 6; ++f) {
        const float* upf = up + f * 3 * kThreads;
        const uint32_t kk = wavelet_key_bits(upf[tid], upf[kThreads + tid], upf[2 * kThreads + tid]);
        kmax = max(kmax, kk);
        reinterpret_cast<uint32_t*>(&sm.keys[((size_t)f * NKQ + NR / 4) * kThreads + tid])[NR % 4] = kk;
      }
    __syncthreads();  // the keys are complete
    // ---- radix select of the K-th largest key.  The keys' top bits are mostly exponent, so a
    // plain first pass piles 24K keys into a few bins (serialised shared atomics).  Instead the
    // first pass histograms only keys within 16 binades of the largest key, at 1/16 binade
    // (256 bins on bits 30..19; keys are non-negative, bit 31 is 0).  If that window holds K
    // keys or more, the K-th largest is in it and the remaining 19 bits take passes of 8, 8
    // and 3 bits over the few keys that match the prefix; otherwise four 8-bit passes.
    uint32_t prefix = 0, mask = 0;
    int remaining = K;
    int shifts[4] = {24, 16, 8, 0}, widths[4] = {8, 8, 8, 8}, n_pass = 4;
    {
      kmax = __reduce_max_sync(0xffffffffu, kmax);  // then over the block: the map's largest key
      if (lane == 0) sm.warp_tot[warp] = (int)kmax;
      for (int i = tid; i < kWarps * 256; i += kThreads) sm.whist[i] = 0u;
      __syncthreads();
#pragma unroll
      for (int w = 0; w < kWarps; ++w) kmax = max(kmax, (uint32_t)sm.warp_tot[w]);
      const int e_lo = (int)(kmax >> 23) - 15;
      if (owner) {
        uint32_t* h = sm.whist + warp * 256;
        for (int f = 0; f < 6; ++f)
#pragma unroll
          for (int q = 0; q < NKQ; ++q) {
            const uint4 v = sm.keys[((size_t)f * NKQ + q) * kThreads + tid];
            const uint32_t kk[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const int e = (int)(kk[i] >> 23);
              if (4 * q + i < NK && e >= e_lo) atomicAdd(&h[((e - e_lo) << 4) | ((kk[i] >> 19) & 15u)], 1u);
            }
          }
      }
      __syncthreads();
      const int bin = 255 - tid;
      uint32_t tot = 0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) tot += sm.whist[w * 256 + bin];
      uint32_t all;
      const uint32_t incl = block_inclusive_sum(tot, sm.warp_tot, &all);  // its barriers order the reads above
      if (tid == 0) sm.scal[kScRemaining] = -1;  // stays -1 when the window holds fewer than K keys
      __syncthreads();
      if (incl >= (uint32_t)K && incl - tot < (uint32_t)K) {
        sm.scal[kScPrefix] = (int)((uint32_t)(((e_lo + (bin >> 4)) << 4) | (bin & 15)) << 19);
        sm.scal[kScRemaining] = K - (int)(incl - tot);
      }
      __syncthreads();
      if (sm.scal[kScRemaining] >= 0) {
        prefix = (uint32_t)sm.scal[kScPrefix];
        mask = 0xFFF80000u;
        remaining = sm.scal[kScRemaining];
        shifts[0] = 11;
        shifts[1] = 3;
        shifts[2] = 0;
        widths[2] = 3;
        n_pass = 3;
      }
    }
    // ---- the window's bin was found: every key above it wins, the keys in it are candidates.
    // Two scans sort them without atomics: the first counts each thread's keys above the bin
    // and in it, one block scan of both counts (packed in one word; each total is below 2^16)
    // gives every thread its slots, and the second writes them.  A group of four keys below
    // the bin (almost all of them) costs one compare per scan.  The candidates, usually a few
    // dozen, are ranked among themselves.  More candidates than fit: the general passes below.
    bool fast = false;
    if (n_pass == 3) {
      uint64_t* ckey = reinterpret_cast<uint64_t*>(sm.whist);
      int* cid = reinterpret_cast<int*>(ckey + kCandCap);
      const uint32_t lo_key = prefix, hi_key = prefix + (1u << 19);  // the bin is [lo_key, hi_key)
      uint32_t n_up = 0, n_in = 0;
      if (owner)
        for (int f = 0; f < 6; ++f)
#pragma unroll
          for (int q = 0; q < NKQ; ++q) {
            const uint4 v = sm.keys[((size_t)f * NKQ + q) * kThreads + tid];
            if (max(max(v.x, v.y), max(v.z, v.w)) < lo_key) continue;
            const uint32_t kk[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const bool live = 4 * q + i < NK;
              n_up += live && kk[i] >= hi_key;
              n_in += live && kk[i] >= lo_key && kk[i] < hi_key;
            }
          }
      uint32_t all;
      const uint32_t packed = n_up | (n_in << 16);
      const uint32_t excl = block_inclusive_sum(packed, sm.warp_tot, &all) - packed;  // barriers inside
      uint32_t slot_up = excl & 0xFFFFu, slot_in = excl >> 16;
      if (owner && packed)
        for (int f = 0; f < 6; ++f)
#pragma unroll
          for (int q = 0; q < NKQ; ++q) {
            const uint4 v = sm.keys[((size_t)f * NKQ + q) * kThreads + tid];
            if (max(max(v.x, v.y), max(v.z, v.w)) < lo_key) continue;
            const uint32_t kk[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const int u = 4 * q + i;
              if (u >= NK || kk[i] < lo_key) continue;
              const int g = f * SS + flat_in_face<S>(tid, u);
              const uint64_t ck = ((uint64_t)kk[i] << 32) | (uint64_t)(0xFFFFFFFFu - (uint32_t)g);
              const int id = (f * NK + u) * kThreads + tid;
              if (kk[i] >= hi_key) {
                sm.gkey[slot_up] = ck;
                sm.gid[slot_up] = id;
                ++slot_up;
              } else {
                if (slot_in < (uint32_t)kCandCap) {
                  ckey[slot_in] = ck;
                  cid[slot_in] = id;
                }
                ++slot_in;
              }
            }
          }
      if (tid == 0) {
        sm.scal[kScNAbove] = (int)(all & 0xFFFFu);
        sm.scal[kScNCand] = (int)(all >> 16);
      }
      __syncthreads();
      const int n_cand = sm.scal[kScNCand];
      if (n_cand <= kCandCap) {
        fast = true;
        const int n_above = sm.scal[kScNAbove];  // == K - remaining
        for (int c = tid; c < n_cand; c += kThreads) {
          const uint64_t me = ckey[c];
          int rank = 0;
          for (int o = 0; o < n_cand; ++o) rank += ckey[o] > me;
          if (rank < remaining) {
            sm.gkey[n_above + rank] = me;
            sm.gid[n_above + rank] = cid[c];
          }
        }
        __syncthreads();
      }
    }
    if (!fast) {
      for (int pass = 0; pass < n_pass; ++pass) {
        const int shift = shifts[pass];
        const uint32_t dmask = (1u << widths[pass]) - 1u;
        for (int i = tid; i < kWarps * 256; i += kThreads) sm.whist[i] = 0u;
        __syncthreads();
        if (owner) {
          uint32_t* h = sm.whist + warp * 256;
          for (int f = 0; f < 6; ++f)
  #pragma unroll
            for (int q = 0; q < NKQ; ++q) {
              const uint4 v = sm.keys[((size_t)f * NKQ + q) * kThreads + tid];
              const uint32_t kk[4] = {v.x, v.y, v.z, v.w};
  #pragma unroll
              for (int i = 0; i < 4; ++i)
                if (4 * q + i < NK && (kk[i] & mask) == prefix) atomicAdd(&h[(kk[i] >> shift) & dmask], 1u);
            }
        }
        __syncthreads();
        const int digit = 255 - tid;  // digits above dmask hold no keys
        uint32_t tot = 0;
  #pragma unroll
        for (int w = 0; w < kWarps; ++w) tot += sm.whist[w * 256 + digit];
        uint32_t all;
        const uint32_t incl = block_inclusive_sum(tot, sm.warp_tot, &all);
        if (incl >= (uint32_t)remaining && incl - tot < (uint32_t)remaining) {
          sm.scal[kScPrefix] = (int)(prefix | ((uint32_t)digit << shift));
          sm.scal[kScMask] = (int)(mask | (dmask << shift));
          sm.scal[kScRemaining] = remaining - (int)(incl - tot);
        }
        __syncthreads();
        prefix = (uint32_t)sm.scal[kScPrefix];
        mask = (uint32_t)sm.scal[kScMask];
        remaining = sm.scal[kScRemaining];
      }
      // ---- ties at the threshold in flat-index order: a bitmap over face * S*S + flat
      const uint32_t thr = prefix;
      for (int w = tid; w < NW; w += kThreads) sm.bits[w] = 0u;
      __syncthreads();
      if (owner)
        for (int f = 0; f < 6; ++f)
  #pragma unroll
          for (int q = 0; q < NKQ; ++q) {
            const uint4 v = sm.keys[((size_t)f * NKQ + q) * kThreads + tid];
            const uint32_t kk[4] = {v.x, v.y, v.z, v.w};
  #pragma unroll
            for (int i = 0; i < 4; ++i)
              if (4 * q + i < NK && kk[i] == thr) {
                const int g = f * SS + flat_in_face<S>(tid, 4 * q + i);
                atomicOr(&sm.bits[g >> 5], 1u << (g & 31));
              }
          }
      __syncthreads();
      {
        // exclusive popcount prefix over the bitmap: thread t covers words [t*per, t*per + per)
        constexpr int PER = (NW + kThreads - 1) / kThreads;
        uint32_t pc[PER], mine = 0;
  #pragma unroll
        for (int i = 0; i < PER; ++i) {
          const int w = tid * PER + i;
          pc[i] = w < NW ? (uint32_t)__popc(sm.bits[w]) : 0u;
          mine += pc[i];
        }
        uint32_t all;
        uint32_t run = block_inclusive_sum(mine, sm.warp_tot, &all) - mine;
  #pragma unroll
        for (int i = 0; i < PER; ++i) {
          const int w = tid * PER + i;
          if (w < NW) sm.wpre[w] = run;
          run += pc[i];
        }
      }
      __syncthreads();
      // ---- winners: slots from one block scan of per-thread counts
      int n_sel = 0;
      if (owner)
        for (int f = 0; f < 6; ++f)
  #pragma unroll
          for (int q = 0; q < NKQ; ++q) {
            const uint4 v = sm.keys[((size_t)f * NKQ + q) * kThreads + tid];
            const uint32_t kk[4] = {v.x, v.y, v.z, v.w};
  #pragma unroll
            for (int i = 0; i < 4; ++i) {
              if (4 * q + i >= NK) continue;
              bool sel = kk[i] > thr;
              if (kk[i] == thr) {
                const int g = f * SS + flat_in_face<S>(tid, 4 * q + i), w = g >> 5;
                sel = (int)(sm.wpre[w] + __popc(sm.bits[w] & ((1u << (g & 31)) - 1u))) < remaining;
              }
              n_sel += sel;
            }
          }
      uint32_t all_sel;
      int slot = (int)block_inclusive_sum((uint32_t)n_sel, sm.warp_tot, &all_sel) - n_sel;
      if (owner && n_sel)
        for (int f = 0; f < 6; ++f)
  #pragma unroll
          for (int q = 0; q < NKQ; ++q) {
            const uint4 v = sm.keys[((size_t)f * NKQ + q) * kThreads + tid];
            const uint32_t kk[4] = {v.x, v.y, v.z, v.w};
  #pragma unroll
            for (int i = 0; i < 4; ++i) {
              if (4 * q + i >= NK) continue;
              const int u = 4 * q + i;
              const int g = f * SS + flat_in_face<S>(tid, u);
              bool sel = kk[i] > thr;
              if (kk[i] == thr) {
                const int w = g >> 5;
                sel = (int)(sm.wpre[w] + __popc(sm.bits[w] & ((1u << (g & 31)) - 1u))) < remaining;
              }
              if (sel) {
                sm.gkey[slot] = ((uint64_t)kk[i] << 32) | (uint64_t)(0xFFFFFFFFu - (uint32_t)g);
                sm.gid[slot] = (f * NK + u) * kThreads + tid;
                ++slot;
              }
            }
          }
      __syncthreads();
    }
    // ---- order the K winners.  Every winner's key lies in [prefix, kmax] (prefix: the window
    // bin's lower edge or the exact threshold), so a counting pass over 256 bins of that range
    // (bin 0 = the largest keys) places them, and each is ranked only among the few winners of
    // its own bin by the composite key.  The histogram region is free again here.
    uint32_t* bin_n = sm.whist;                                    // [256] winners per bin
    uint32_t* bin_end = sm.whist + 256;                            // [256] scatter cursor
    uint16_t* order = reinterpret_cast<uint16_t*>(sm.whist + 512);  // [K] winners by bin
    const uint32_t range = kmax - prefix;
    const int bshift = range < 256u ? 0 : 24 - __clz((int)range);  // (range >> bshift) < 256
    auto bin_of = [&](uint64_t ck) { return (kmax - (uint32_t)(ck >> 32)) >> bshift; };
    bin_n[tid] = 0u;  // kThreads == 256 bins
    __syncthreads();
    for (int e = tid; e < K; e += kThreads) atomicAdd(&bin_n[bin_of(sm.gkey[e])], 1u);
    __syncthreads();
    {
      uint32_t all;
      const uint32_t n = bin_n[tid];
      bin_end[tid] = block_inclusive_sum(n, sm.warp_tot, &all) - n;  // starts; ends after the scatter
    }
    __syncthreads();
    for (int e = tid; e < K; e += kThreads) order[atomicAdd(&bin_end[bin_of(sm.gkey[e])], 1u)] = (uint16_t)e;
    __syncthreads();
    for (int e = tid; e < K; e += kThreads) {
      const uint64_t me = sm.gkey[e];
      const uint32_t b = bin_of(me), end = bin_end[b];
      int rank = (int)(end - bin_n[b]);
      for (uint32_t i = end - bin_n[b]; i < end; ++i) rank += sm.gkey[order[i]] > me;
      const int id = sm.gid[e];
      const int t = id % kThreads, fu = id / kThreads, f = fu / NK, u = fu % NK;
      const size_t out = (size_t)env * K + rank;
      float v[3] = {0.f, 0.f, 0.f};
      if (u == NR) {
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = up[(f * 3 + c) * kThreads + t];
      } else if constexpr (NR > 0) {
        block_coef<S>(faces + ((size_t)env * 6 + f) * (size_t)SS * 3, t, u, v);
      }
      idx_out[out] = f * SS + flat_in_face<S>(t, u);
      st_out[out * 3 + 0] = v[0];
      st_out[out * 3 + 1] = v[1];
      st_out[out * 3 + 2] = v[2];
    }
    __syncthreads();  // the next map reuses every shared array and the scratch slice
  }
}

// Batches of at least this many maps use the batched kernel; smaller ones the cluster form,
// whose six CTAs per map give the lower latency for a single map.
constexpr int kBatchMinMaps = 32;

// A stream-ordered pool per device for the batched kernel's scratch.  It keeps its memory
// between calls (release threshold = max), so a steady stream of batches allocates once.
std::mutex g_pool_mu;
cudaMemPool_t g_pool[64] = {};

cudaMemPool_t scratch_pool(int dev) {
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (dev < 0 || dev >= 64) fail(NWPRT_UNSUPPORTED, "haar_topk: device ordinal beyond the pool table");
  if (!g_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    NWPRT_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = ~0ull;
    NWPRT_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pool[dev] = pool;
  }
  return g_pool[dev];
}

template <int S>
void launch_s(const float* faces, int n_env, int K, int32_t* idx, float* strength, cudaStream_t st) {
  int dev = 0, sms = 0, max_smem = 0;
  NWPRT_CUDA(cudaGetDevice(&dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const size_t bsmem = batch_smem_layout(S, K, nullptr, nullptr);
  if (n_env >= kBatchMinMaps && bsmem <= (size_t)max_smem) {
    NWPRT_CUDA(cudaFuncSetAttribute(haar_topk_batch_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsmem));
    int per_sm = 0;
    NWPRT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, haar_topk_batch_kernel<S>, kThreads, bsmem));
    const long long slots = (long long)sms * (per_sm > 0 ? per_sm : 1);
    const int grid = (int)(n_env < slots ? n_env : slots);
    void* scratch = nullptr;
    const size_t bytes = (size_t)grid * batch_scratch_floats_per_cta<S>() * sizeof(float);
    if (cudaMallocFromPoolAsync(&scratch, bytes, scratch_pool(dev), st) == cudaSuccess) {
      haar_topk_batch_kernel<S><<<grid, kThreads, bsmem, st>>>(faces, n_env, K, idx, strength, (float*)scratch);
      const cudaError_t launch = cudaGetLastError();
      NWPRT_CUDA(cudaFreeAsync(scratch, st));
      NWPRT_CUDA(launch);
      return;
    }
    (void)cudaGetLastError();  // no scratch: the cluster form needs none
  }
  const size_t smem = smem_layout(S, K, nullptr, nullptr);
  NWPRT_CUDA(cudaFuncSetAttribute(haar_topk_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  haar_topk_kernel<S><<<6 * n_env, kThreads, smem, st>>>(faces, K, idx, strength);
  NWPRT_CUDA(cudaGetLastError());
}

}  // namespace

size_t haar_topk_smem_bytes(int S, int K) { return smem_layout(S, K, nullptr, nullptr); }

void launch_haar_topk(const float* faces, int n_env, int S, int K, int32_t* idx, float* strength,
                      uint32_t* /*err: the kernel has no waits that could time out*/, cudaStream_t st) {
  if (n_env < 1 || n_env > (1 << 28)) fail(NWPRT_INVALID_ARG, "haar_topk: n_env out of range");
  if (S < 1 || S > kMaxS || (S & (S - 1)))
    fail(S > kMaxS ? NWPRT_UNSUPPORTED : NWPRT_INVALID_ARG,
         "haar_topk: face size must be a power of two <= 64");
  if (K < 1 || K > 6 * S * S || K > kMaxK)
    fail(NWPRT_INVALID_ARG, "haar_topk: K must be in [1, min(6*S*S, 1024)]");
  if (!faces || !idx || !strength) fail(NWPRT_INVALID_ARG, "haar_topk: null pointer");
  switch (S) {
    case 1: launch_s<1>(faces, n_env, K, idx, strength, st); break;
    case 2: launch_s<2>(faces, n_env, K, idx, strength, st); break;
    case 4: launch_s<4>(faces, n_env, K, idx, strength, st); break;
    case 8: launch_s<8>(faces, n_env, K, idx, strength, st); break;
    case 16: launch_s<16>(faces, n_env, K, idx, strength, st); break;
    case 32: launch_s<32>(faces, n_env, K, idx, strength, st); break;
    default: launch_s<64>(faces, n_env, K, idx, strength, st); break;
  }
}

}  // namespace nwprt

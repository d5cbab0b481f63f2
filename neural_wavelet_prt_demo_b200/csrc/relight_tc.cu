// tcgen05 tensor-core relight kernel: BF16 operands, FP32 accumulation in TMEM.
//
// Same computation as the FP32 path (prt_network.h:73-154 + utils_kernels.h:52-127):
// per pixel p and wavelet k, cp = hash(p) * E[:, idx_k] -> out_prd MLP -> [o || aux]
// -> cmp_net MLP -> T_k, and sum_k max(L_k * T_k, 0).  Every hidden dense layer of a
// 128-pixel x 1-wavelet row block is one tcgen05.mma chain (M=128, N<=64, K=16 steps);
// the final 3-output layer runs in FP32 on the CUDA cores inside the epilogue of the
// layer before it, straight from the FP32 accumulator.
//
// Design, from measurements on B200: a tcgen05.mma costs >= ~60 cycles whatever N <= 64,
// so these 64-wide layers are bound by MMA issue at ~53% of the tensor peak; keeping the
// activations in shared memory made the kernel shared-memory-bandwidth bound instead
// (operand reads + epilogue stores ~266 KB per tile and wavelet).  So activations live
// in TMEM: the A operand of every layer is read by the MMA straight from tensor memory
// (the ".kind::f16 [d], [a], b_desc" form), and the epilogue writes it back with a
// single tcgen05.st.  Only the weights (B) and the per-tile aux block come from shared
// memory.
//
// Organisation (one persistent CTA per SM): kNWG warpgroups, one 128-pixel tile each,
// 128 TMEM columns per tile: [0,32) the BF16 A operand (2 values per 32-bit column),
// [64,128) the FP32 accumulator.  Thread (warp w, lane l) owns tile row 32*(w%4)+l, the
// TMEM lane it may access.  Per layer: wait on the tile's commit barrier -> tcgen05.ld
// -> ReLU + cvt.rn.relu.bf16x2 -> tcgen05.st into the A columns -> warpgroup barrier
// (bar.red.and carrying the "no timeout" vote) -> one elected thread issues the next
// layer's MMAs and commits them.  The final layer's epilogue forms T_k, does the
// clamped Kahan sum and writes the next wavelet's first-layer operand hash(p) * E_k+1.
// Every wait is bounded by %globaltimer (2 s); on expiry the kernel records
// kDevWaitTimeout and the warpgroup unwinds together.
#include <cmath>
#include <cstring>

#include "nwprt_internal.cuh"

namespace nwprt {
namespace {

constexpr int kNWG = 4;                    // warpgroups per CTA, one tile each
constexpr int kThreads = 128 * kNWG;
constexpr int kTile = 128;                 // pixels per tile (MMA M)
constexpr int kAuxBytes = kTile * 16 * 2;  // 128 x 16 bf16 aux operand
constexpr int kMaxTcLayers = 12;
constexpr int kTmemCols = 512;
constexpr int kTileCols = 128;             // TMEM columns per tile
constexpr int kAcol = 0;                   // A operand columns [0, 32)
constexpr int kDcol = 64;                  // accumulator columns [64, 128)
constexpr int kVlastFloats = 3 * 64;
constexpr uint64_t kWaitNs = 2000000000ull;
static_assert(kNWG * kTileCols <= kTmemCols, "TMEM budget");

struct TcLayer {
  uint32_t b_off;  // byte offset of B (N x K, canonical K-major) in the weight blob
  uint32_t b_sbo;  // B stride between 8-row groups (= K * 16 bytes)
  int k;           // reduction length (multiple of 16)
  int n;           // output width: 32 or 64
  int relu;
  int aux;         // also accumulate aux (K=16) x aux block of B at aux_off
  uint32_t aux_off;
  int fin;         // the epilogue forms T_k = V_last relu(h) from this layer's output
};

struct TcParams {
  HashLevels hl;
  const float* hash;
  const uint4* wblob;
  uint32_t wblob_bytes;
  uint32_t vlast_off;  // byte offset of V_last (FP32 [3][64]) in the blob
  TcLayer layers[kMaxTcLayers];
  int n_layers;
  int enc_dims;  // D, multiple of 16, <= 32
  const TcJob* jobs;
  int n_jobs;
  long long total_tiles;
  int kahan, clamp;
  uint32_t* err;
};

// ------------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(a), "r"(parity)
      : "memory");
  return done != 0;
}

// Wait for the phase with `parity`, bounded by kWaitNs of wall time.
__device__ __forceinline__ bool wait_bounded(uint64_t* bar, uint32_t parity, uint32_t* err) {
  const uint32_t a = smem_u32(bar);
  if (mbar_try(a, parity)) return true;
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 1; it < (1u << 30); ++it) {
    if (mbar_try(a, parity)) return true;
    if ((it & 255u) == 0 && globaltimer() - t0 > kWaitNs) break;
  }
  atomicCAS(err, 0u, (uint32_t)kDevWaitTimeout);
  return false;
}

// Warpgroup barrier (named barrier 1+g, 128 threads) that also ANDs a predicate.
__device__ __forceinline__ bool wg_barrier_and(int g, bool pred) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(out)
      : "r"((uint32_t)pred), "r"(1 + g)
      : "memory");
  return out != 0;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1, no swizzle
}

// kind::f16 instruction descriptor: D=F32, A=B=BF16, both K-major, M=128.
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// D[tmem] (+)= A[tmem] * B[smem]^T
__device__ __forceinline__ void mma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T
__device__ __forceinline__ void mma_ss(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

#define NWPRT_R8(i) "=r"(r[i]), "=r"(r[i + 1]), "=r"(r[i + 2]), "=r"(r[i + 3]), "=r"(r[i + 4]), \
                    "=r"(r[i + 5]), "=r"(r[i + 6]), "=r"(r[i + 7])
#define NWPRT_W8(i) "r"(r[i]), "r"(r[i + 1]), "r"(r[i + 2]), "r"(r[i + 3]), "r"(r[i + 4]), \
                    "r"(r[i + 5]), "r"(r[i + 6]), "r"(r[i + 7])

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : NWPRT_R8(0), NWPRT_R8(8), NWPRT_R8(16), NWPRT_R8(24)
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
      NWPRT_W8(0), NWPRT_W8(8), NWPRT_W8(16), NWPRT_W8(24)
      : "memory");
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t* r) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr),
      NWPRT_W8(0), NWPRT_W8(8)
      : "memory");
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t* r) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr),
               NWPRT_W8(0)
               : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}
__device__ __forceinline__ uint32_t pack_bf16_relu(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}
__device__ __forceinline__ float bf16_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d)
               : "memory");
}

// Byte offset of (row, 16-byte K chunk) in a canonical no-swizzle K-major tile whose
// 8-row groups are `sbo` bytes apart.
__device__ __forceinline__ uint32_t core_off(int row, int chunk, uint32_t sbo) {
  return (uint32_t)(row >> 3) * sbo + (uint32_t)chunk * 128u + (uint32_t)(row & 7) * 16u;
}

// 32 FP32 TMEM values -> 16 BF16 pairs.
template <bool RELU>
__device__ __forceinline__ void pack32(const uint32_t (&v)[32], uint32_t* out) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const float lo = __uint_as_float(v[2 * j]), hi = __uint_as_float(v[2 * j + 1]);
    out[j] = RELU ? pack_bf16_relu(lo, hi) : pack_bf16(lo, hi);
  }
}

// T += V_last[:, j0:j0+32] relu(h[j0:j0+32]) in FP32 (ascending j).
__device__ __forceinline__ void final_dot32(const uint32_t (&v)[32], const float* __restrict__ sV, int j0,
                                            float& t0, float& t1, float& t2) {
#pragma unroll
  for (int j4 = 0; j4 < 8; ++j4) {
    const float4 a = *reinterpret_cast<const float4*>(sV + 0 * 64 + j0 + 4 * j4);
    const float4 b = *reinterpret_cast<const float4*>(sV + 1 * 64 + j0 + 4 * j4);
    const float4 c = *reinterpret_cast<const float4*>(sV + 2 * 64 + j0 + 4 * j4);
    const float h0 = fmaxf(__uint_as_float(v[4 * j4 + 0]), 0.f), h1 = fmaxf(__uint_as_float(v[4 * j4 + 1]), 0.f);
    const float h2 = fmaxf(__uint_as_float(v[4 * j4 + 2]), 0.f), h3 = fmaxf(__uint_as_float(v[4 * j4 + 3]), 0.f);
    t0 = fmaf(a.x, h0, t0); t0 = fmaf(a.y, h1, t0); t0 = fmaf(a.z, h2, t0); t0 = fmaf(a.w, h3, t0);
    t1 = fmaf(b.x, h0, t1); t1 = fmaf(b.y, h1, t1); t1 = fmaf(b.z, h2, t1); t1 = fmaf(b.w, h3, t1);
    t2 = fmaf(c.x, h0, t2); t2 = fmaf(c.y, h1, t2); t2 = fmaf(c.z, h2, t2); t2 = fmaf(c.w, h3, t2);
  }
}

// Hash-grid encoding (same arithmetic as the FP32 path), kept as BF16 pairs.
template <int DMAX>
__device__ __forceinline__ void hash_encode_bf16(const HashLevels& hl, const float* __restrict__ table,
                                                 float px, float py, float pz, uint32_t (&enc)[DMAX / 2]) {
  const float p[3] = {fminf(fmaxf(px, 0.f), 1.f), fminf(fmaxf(py, 0.f), 1.f), fminf(fmaxf(pz, 0.f), 1.f)};
#pragma unroll
  for (int l = 0; l < DMAX / 2; ++l) {
    float a0 = 0.f, a1 = 0.f;
    if (l < hl.n_levels) {
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
      const float2* lvl = reinterpret_cast<const float2*>(table) + hl.offset[l];
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
        const float2 v = __ldg(lvl + e);
        a0 = fmaf(wc, v.x, a0);
        a1 = fmaf(wc, v.y, a1);
      }
    }
    enc[l] = pack_bf16(a0, a1);
  }
}

// First-layer operand of wavelet k (hash(p) * E_k, rounded once to BF16) -> TMEM A columns.
template <int DMAX>
__device__ __forceinline__ void store_cp(const uint32_t (&enc)[DMAX / 2], const float* __restrict__ ek,
                                         uint32_t a_taddr) {
  uint32_t cp[DMAX / 2];
#pragma unroll
  for (int c = 0; c < DMAX / 8; ++c) {
    const float4 e0 = __ldg(reinterpret_cast<const float4*>(ek + c * 8));
    const float4 e1 = __ldg(reinterpret_cast<const float4*>(ek + c * 8 + 4));
    const uint32_t h0 = enc[c * 4 + 0], h1 = enc[c * 4 + 1], h2 = enc[c * 4 + 2], h3 = enc[c * 4 + 3];
    cp[c * 4 + 0] = pack_bf16(__fmul_rn(bf16_lo(h0), e0.x), __fmul_rn(bf16_hi(h0), e0.y));
    cp[c * 4 + 1] = pack_bf16(__fmul_rn(bf16_lo(h1), e0.z), __fmul_rn(bf16_hi(h1), e0.w));
    cp[c * 4 + 2] = pack_bf16(__fmul_rn(bf16_lo(h2), e1.x), __fmul_rn(bf16_hi(h2), e1.y));
    cp[c * 4 + 3] = pack_bf16(__fmul_rn(bf16_lo(h3), e1.z), __fmul_rn(bf16_hi(h3), e1.w));
  }
  if constexpr (DMAX == 32) tmem_st16(a_taddr, cp);
  else tmem_st8(a_taddr, cp);
}

__device__ __forceinline__ int find_job(const TcJob* jobs, int n_jobs, long long tile) {
  int lo = 0, hi = n_jobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].tile_begin <= tile) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct __align__(8) TcBarriers {
  uint64_t acc_full[kNWG];  // MMA commit -> epilogue of that warpgroup's tile
  uint64_t done[kNWG];      // final commit before TMEM is released
  uint32_t tmem_base;
};

// Issues layer L of warpgroup g's tile: A from TMEM (and the aux block from shared memory).
__device__ __forceinline__ void issue_layer(const TcLayer& L, uint32_t wbase, uint32_t a_tmem, uint32_t aux_base,
                                            uint32_t d_tmem, uint64_t* bar) {
  tc_fence_after();
  const uint32_t id = idesc_bf16(L.n);
  for (int s = 0; s < L.k / 16; ++s) {
    const uint64_t bd = smem_desc(wbase + L.b_off + (uint32_t)s * 256u, 128u, L.b_sbo);
    mma_ts(d_tmem, a_tmem + (uint32_t)s * 8u, bd, id, s > 0 ? 1u : 0u);
  }
  if (L.aux) {
    const uint64_t ad = smem_desc(aux_base, 128u, 256u);
    const uint64_t bd = smem_desc(wbase + L.aux_off, 128u, 256u);
    mma_ss(d_tmem, ad, bd, id, 1u);
  }
  mma_commit(bar);
}

template <int DMAX>
__global__ void __launch_bounds__(kThreads, 1) relight_tc_kernel(const __grid_constant__ TcParams p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* wsm = smem;                                       // weight blob (+ V_last)
  uint8_t* aux = smem + ((p.wblob_bytes + 1023u) & ~1023u);  // [kNWG][kAuxBytes]
  TcBarriers* bars = reinterpret_cast<TcBarriers*>(aux + kNWG * kAuxBytes);
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = warp >> 2;  // warpgroup
  const int q = warp & 3;   // TMEM lane quarter this warp may access
  const int row = q * 32 + lane;
  const bool leader = (tid & 127) == 0;

  // ---- weights -> shared memory (generic proxy), barriers, TMEM
  for (uint32_t i = tid; i < p.wblob_bytes / 16u; i += kThreads)
    reinterpret_cast<uint4*>(wsm)[i] = __ldg(p.wblob + i);
  if (tid == 0) {
    for (int w = 0; w < kNWG; ++w) {
      mbar_init(&bars->acc_full[w], 1);
      mbar_init(&bars->done[w], 1);
    }
    fence_barrier_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&bars->tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = bars->tmem_base;
  const uint32_t wbase = smem_u32(wsm);
  const float* sV = reinterpret_cast<const float*>(wsm + p.vlast_off);
  const long long stride = (long long)gridDim.x * kNWG;
  const uint32_t col0 = tmem + (uint32_t)(g * kTileCols);
  const uint32_t a_tmem = col0 + kAcol;                                 // MMA operand address (lane 0)
  const uint32_t d_tmem = col0 + kDcol;
  const uint32_t a_taddr = a_tmem + ((uint32_t)(q * 32) << 16);         // this warp's lanes
  const uint32_t d_taddr = d_tmem + ((uint32_t)(q * 32) << 16);
  const uint32_t aux_base = smem_u32(aux + g * kAuxBytes);
  const uint32_t aux_row = aux_base + core_off(row, 0, 256u);
  uint64_t* acc_bar = &bars->acc_full[g];

  uint32_t ph = 0;
  bool ok = true;
  for (long long t = (long long)blockIdx.x * kNWG + g; t < p.total_tiles && ok; t += stride) {
    // ---- tile set-up: hash encoding, aux operand, first-layer operand of wavelet 0
    const int jid = find_job(p.jobs, p.n_jobs, t);
    const TcJob& J = p.jobs[jid];
    const int K = J.K;
    const long long px = J.px_begin + (t - J.tile_begin) * kTile + row;
    const bool valid = px < J.n_px;
    uint32_t enc[DMAX / 2];
    if (valid) {
      const float4* pr = reinterpret_cast<const float4*>(J.packed) + px * 4;
      const float4 r0 = __ldg(pr), r1 = __ldg(pr + 1), r2 = __ldg(pr + 2), r3 = __ldg(pr + 3);
      hash_encode_bf16<DMAX>(p.hl, p.hash, r0.x, r0.y, r0.z, enc);
      // aux operand: the 13 remapped G-buffer values followed by ones
      st_shared_v4(aux_row, pack_bf16(r0.w, r1.x), pack_bf16(r1.y, r1.z), pack_bf16(r1.w, r2.x),
                   pack_bf16(r2.y, r2.z));
      st_shared_v4(aux_row + 128u, pack_bf16(r2.w, r3.x), pack_bf16(r3.y, r3.z), pack_bf16(r3.w, 1.f),
                   pack_bf16(1.f, 1.f));
    } else {
#pragma unroll
      for (int i = 0; i < DMAX / 2; ++i) enc[i] = 0u;
      st_shared_v4(aux_row, 0, 0, 0, 0);
      st_shared_v4(aux_row + 128u, 0, 0, 0, 0);
    }
    store_cp<DMAX>(enc, J.emb_k, a_taddr);
    tmem_wait_st();
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
    // hand the first layer to the tensor core
    tc_fence_before();
    fence_proxy_async_smem();
    ok = wg_barrier_and(g, ok);
    if (ok && leader) issue_layer(p.layers[0], wbase, a_tmem, aux_base, d_tmem, acc_bar);
    for (int k = 0; k < K && ok; ++k) {
      for (int l = 0; l < p.n_layers; ++l) {
        const TcLayer& L = p.layers[l];
        const bool waited = __all_sync(0xffffffffu, wait_bounded(acc_bar, ph, p.err));
        ph ^= 1u;
        if (waited) {
          tc_fence_after();
          uint32_t v[32];
          if (!L.fin) {
            uint32_t a[32];
            tmem_ld32(d_taddr, v);
            tmem_wait_ld();
            if (L.relu) pack32<true>(v, a);
            else pack32<false>(v, a);
            if (L.n > 32) {
              tmem_ld32(d_taddr + 32u, v);
              tmem_wait_ld();
              if (L.relu) pack32<true>(v, a + 16);
              else pack32<false>(v, a + 16);
              tmem_st32(a_taddr, a);
            } else {
              tmem_st16(a_taddr, a);
            }
            tmem_wait_st();
          } else {
            float t0 = 0.f, t1 = 0.f, t2 = 0.f;
            tmem_ld32(d_taddr, v);
            tmem_wait_ld();
            final_dot32(v, sV, 0, t0, t1, t2);
            tmem_ld32(d_taddr + 32u, v);
            tmem_wait_ld();
            final_dot32(v, sV, 32, t0, t1, t2);
            const float* Lk = J.strength + (size_t)k * 3;
            float u0 = __fmul_rn(__ldg(Lk + 0), t0);
            float u1 = __fmul_rn(__ldg(Lk + 1), t1);
            float u2 = __fmul_rn(__ldg(Lk + 2), t2);
            if (p.clamp) { u0 = fmaxf(u0, 0.f); u1 = fmaxf(u1, 0.f); u2 = fmaxf(u2, 0.f); }
            if (p.kahan) {
              float y, z;
              y = __fsub_rn(u0, c0); z = __fadd_rn(s0, y); c0 = __fsub_rn(__fsub_rn(z, s0), y); s0 = z;
              y = __fsub_rn(u1, c1); z = __fadd_rn(s1, y); c1 = __fsub_rn(__fsub_rn(z, s1), y); s1 = z;
              y = __fsub_rn(u2, c2); z = __fadd_rn(s2, y); c2 = __fsub_rn(__fsub_rn(z, s2), y); s2 = z;
            } else {
              s0 = __fadd_rn(s0, u0); s1 = __fadd_rn(s1, u1); s2 = __fadd_rn(s2, u2);
            }
            if (k + 1 < K) {
              store_cp<DMAX>(enc, J.emb_k + (size_t)(k + 1) * p.enc_dims, a_taddr);
              tmem_wait_st();
            }
          }
        }
        ok = ok && waited;
        if (l + 1 == p.n_layers && k + 1 == K) break;  // the tile's last layer: no hand-off
        const int nl = (l + 1 == p.n_layers) ? 0 : l + 1;
        tc_fence_before();
        ok = wg_barrier_and(g, ok);
        if (!ok) break;
        if (leader) issue_layer(p.layers[nl], wbase, a_tmem, aux_base, d_tmem, acc_bar);
      }
    }
    if (valid && ok) {
      const float4 ind = J.flag[px] ? make_float4(s0, s1, s2, 1.f) : make_float4(0.f, 0.f, 0.f, 1.f);
      const float4 dl = __ldg(reinterpret_cast<const float4*>(J.direct) + px);
      reinterpret_cast<float4*>(J.indirect)[px] = ind;
      reinterpret_cast<float4*>(J.with_direct)[px] =
          make_float4(__fadd_rn(ind.x, dl.x), __fadd_rn(ind.y, dl.y), __fadd_rn(ind.z, dl.z), 1.f);
    }
    // every thread of the warpgroup agrees on the outcome before the next tile
    ok = wg_barrier_and(g, ok);
  }
  // every MMA this warpgroup issued has completed before TMEM is released
  if (leader) {
    mma_commit(&bars->done[g]);
    wait_bounded(&bars->done[g], 0, p.err);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                 : "memory");
}

// ------------------------------------------------------------------ host-side packing
uint16_t to_bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return 0x7fc0;
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

int pad16(int x) { return (x + 15) & ~15; }

// Writes the N x K (row-major [out][in]) block src[:, col0:col0+kc] as a canonical
// K-major tile of np x kp BF16 (zero padded) at byte offset `off` of the blob.
void put_b(std::vector<uint16_t>* blob, size_t off, const float* src, int n, int k_total, int col0, int kc,
           int np, int kp) {
  const size_t need = off / 2 + (size_t)np * kp;
  if (blob->size() < need) blob->resize(need, 0);
  const uint32_t sbo = (uint32_t)kp * 16u;
  for (int r = 0; r < np; ++r)
    for (int c = 0; c < kp; ++c) {
      const float v = (r < n && c < kc) ? src[(size_t)r * k_total + col0 + c] : 0.f;
      const size_t byte = off + (size_t)(r >> 3) * sbo + (size_t)(c >> 3) * 128 + (size_t)(r & 7) * 16 +
                          (size_t)(c & 7) * 2;
      (*blob)[byte / 2] = to_bf16(v);
    }
}

struct Plan {
  TcLayer layers[kMaxTcLayers];
  int n_layers = 0;
  uint32_t vlast_off = 0;
  std::vector<uint16_t> blob;
};

bool plan_supported(const NetDims& d, std::string* why) {
  auto no = [&](const char* m) { if (why) *why = m; return false; };
  if (d.aux_width != 16) return no("tensor-core path needs a 16-wide aux encoding");
  if (d.enc_dims() % 16 || d.enc_dims() > 32) return no("tensor-core path needs 16 or 32 hash features");
  if (d.op_out > 64) return no("tensor-core path needs out_prd outputs <= 64");
  if (d.cn_hidden < 1) return no("tensor-core path needs a hidden cmp_net layer");
  if (d.cn_neurons > 64 || pad16(d.cn_neurons) != 64) return no("tensor-core path needs 64-wide cmp_net layers");
  if (d.op_nl + d.cn_nl - 1 > kMaxTcLayers) return no("too many layers for the tensor-core path");
  for (int i = 0; i < d.op_nl; ++i) {
    const int n = pad16(d.op_outs[i]);
    if (n != 32 && n != 64) return no("out_prd widths must pad to 32 or 64");
    if (i > 0 && pad16(d.op_in[i]) > 64) return no("tensor-core path needs widths <= 64");
  }
  return true;
}

Plan make_plan(const NetDims& d, const float* op, const float* cn) {
  Plan P;
  size_t off = 0;
  const bool fill = op && cn;
  auto add = [&](const float* W, int n, int k_total, int col0, int kc, bool relu) {
    TcLayer L{};
    const int np = pad16(n), kp = pad16(kc);
    L.b_off = (uint32_t)off;
    L.b_sbo = (uint32_t)kp * 16u;
    L.k = kp;
    L.n = np;
    L.relu = relu;
    if (fill) put_b(&P.blob, off, W, n, k_total, col0, kc, np, kp);
    off += (size_t)np * kp * 2;
    off = (off + 127) & ~size_t(127);
    P.layers[P.n_layers++] = L;
    return P.n_layers - 1;
  };
  const float* w = op;
  for (int i = 0; i < d.op_nl; ++i) {
    add(w, d.op_outs[i], d.op_in[i], 0, d.op_in[i], i + 1 < d.op_nl);
    if (w) w += (size_t)d.op_in[i] * d.op_outs[i];
  }
  w = cn;
  for (int i = 0; i + 1 < d.cn_nl; ++i) {
    int li;
    if (i == 0) {
      li = add(w, d.cn_outs[0], d.cn_in[0], 0, d.op_out, true);
      // aux block: columns [op_out, op_out + 16) of cmp_net's first layer
      P.layers[li].aux = 1;
      P.layers[li].aux_off = (uint32_t)off;
      const int np = pad16(d.cn_outs[0]);
      if (fill) put_b(&P.blob, off, w, d.cn_outs[0], d.cn_in[0], d.op_out, 16, np, 16);
      off += (size_t)np * 16 * 2;
      off = (off + 127) & ~size_t(127);
    } else {
      li = add(w, d.cn_outs[i], d.cn_in[i], 0, d.cn_in[i], true);
    }
    if (w) w += (size_t)d.cn_in[i] * d.cn_outs[i];
  }
  P.layers[P.n_layers - 1].fin = 1;
  // V_last: the 3 x 64 output layer in FP32, [c][j]
  P.vlast_off = (uint32_t)off;
  const size_t vbytes = kVlastFloats * 4;
  P.blob.resize((off + vbytes) / 2, 0);
  if (fill) {
    const int n_in = d.cn_in[d.cn_nl - 1];
    for (int c = 0; c < 3; ++c)
      for (int j = 0; j < 64; ++j) {
        const float v = j < n_in ? w[(size_t)c * n_in + j] : 0.f;
        std::memcpy(reinterpret_cast<char*>(P.blob.data()) + off + (c * 64 + j) * 4, &v, 4);
      }
  }
  off += vbytes;
  off = (off + 127) & ~size_t(127);
  P.blob.resize(off / 2, 0);
  return P;
}

}  // namespace

bool relight_tc_supported(const NetDims& d, std::string* why) { return plan_supported(d, why); }

size_t tc_weight_bytes(const NetDims& d) { return make_plan(d, nullptr, nullptr).blob.size() * 2; }

void pack_tc_weights(const NetDims& d, const float* op, const float* cn, std::vector<uint16_t>* out) {
  *out = make_plan(d, op, cn).blob;
}

size_t relight_tc_smem_bytes(const NetDims& d) {
  return ((tc_weight_bytes(d) + 1023) & ~size_t(1023)) + (size_t)kNWG * kAuxBytes + sizeof(TcBarriers);
}

void launch_relight_tc(const NetDims& d, const HashLevels& hl, const float* hash, const uint16_t* tc_weights_dev,
                       const TcJob* jobs, int n_jobs, TcJob* jobs_dev, int kahan, int clamp, uint32_t* err,
                       cudaStream_t st) {
  std::string why;
  if (!plan_supported(d, &why)) fail(NWPRT_UNSUPPORTED, why);
  if (n_jobs <= 0) return;
  Plan P = make_plan(d, nullptr, nullptr);
  TcParams p{};
  p.hl = hl;
  p.hash = hash;
  p.wblob = reinterpret_cast<const uint4*>(tc_weights_dev);
  p.wblob_bytes = (uint32_t)(P.blob.size() * 2);
  p.vlast_off = P.vlast_off;
  std::memcpy(p.layers, P.layers, sizeof(P.layers));
  p.n_layers = P.n_layers;
  p.enc_dims = d.enc_dims();
  p.n_jobs = n_jobs;
  p.kahan = kahan;
  p.clamp = clamp;
  p.err = err;
  // tile prefix over the jobs, then one copy of the job table (stream ordered)
  std::vector<TcJob> J(jobs, jobs + n_jobs);
  long long tiles = 0;
  for (auto& j : J) {
    j.tile_begin = tiles;
    tiles += (j.n_px - j.px_begin + kTile - 1) / kTile;
  }
  if (tiles == 0) return;
  p.total_tiles = tiles;
  p.jobs = jobs_dev;
  NWPRT_CUDA(cudaMemcpyAsync(jobs_dev, J.data(), sizeof(TcJob) * J.size(), cudaMemcpyHostToDevice, st));
  int dev = 0, sms = 0, max_smem = 0;
  NWPRT_CUDA(cudaGetDevice(&dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const size_t smem = relight_tc_smem_bytes(d);
  if (smem > (size_t)max_smem) fail(NWPRT_UNSUPPORTED, "tensor-core relight: shared memory budget exceeded");
  const long long groups = (tiles + kNWG - 1) / kNWG;
  const int grid = (int)(groups < sms ? groups : sms);
  if (d.enc_dims() <= 16) {
    auto k = relight_tc_kernel<16>;
    NWPRT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<grid, kThreads, smem, st>>>(p);
  } else {
    auto k = relight_tc_kernel<32>;
    NWPRT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<grid, kThreads, smem, st>>>(p);
  }
  NWPRT_CUDA(cudaGetLastError());
}

}  // namespace nwprt

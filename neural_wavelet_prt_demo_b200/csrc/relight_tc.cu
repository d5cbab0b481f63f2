// tcgen05 tensor-core relight kernel: BF16 operands, FP32 accumulation in TMEM.
//
// Same computation as the FP32 path (prt_network.h:73-154 + utils_kernels.h:52-127):
// per pixel p and wavelet k, cp = hash(p) * E[:, idx_k] -> out_prd MLP -> [o || aux]
// -> cmp_net MLP -> T_k, and sum_k max(L_k * T_k, 0).  Every hidden dense layer of a
// 128-pixel x 1-wavelet row block is one tcgen05.mma chain (M=128, N<=64, K=16 steps);
// out_prd's linear output layer is folded into cmp_net's first layer on the host (one
// round trip less per wavelet).  The final 3-output layer is one more tensor-core step in the
// BF16 kernels with a fixed layer sequence: the last hidden layer's ReLU'd activations go back
// to TMEM as FP16 pairs and meet V_last in FP16 (N = 16, FP32 accumulation; FP16 keeps 11
// significant bits where BF16 keeps 8, so the output layer loses nothing measurable).  The
// FP8, calibration and generic forms run it in FP32 on the CUDA cores inside the epilogue of
// the layer before it, straight from the FP32 accumulator.
//
// Design, from measurements on B200: an M=128 N=64 tcgen05.mma issued back to back from an
// elected lane of a converged warp takes ~36 cycles (~90% of the tensor peak), and five
// independent 4-MMA layer chains saturate the pipe; issued from a lone lane of a diverged
// warp the same MMAs take ~75 cycles.  Keeping the activations in shared memory made the
// kernel shared-memory-bandwidth bound (operand reads + epilogue stores ~266 KB per tile and
// wavelet).  So activations live in TMEM: the A operand of every layer is read by the MMA
// straight from tensor memory (the ".kind::f16 [d], [a], b_desc" form), and the epilogue
// writes it back with a single tcgen05.st.  Only the weights (B, loaded once per CTA by TMA)
// and the per-tile aux block come from shared memory; the FP32-dot forms take V_last, the
// output layer, from the kernel parameters.
//
// Organisation (one persistent CTA per SM): kNWG = 5 warpgroups, one 128-pixel tile each,
// 96 TMEM columns per tile (480 of 512): [0,32) the BF16 A operand (2 values per 32-bit
// column), [32,96) the FP32 accumulator.  Each tile is an independent chain of MMA ->
// epilogue round trips, and the kernel is bound by their latency, so five chains beat
// four (640 threads leave ~96 registers each: the hash features of a tile live in shared
// memory, and each half of an accumulator is packed and stored back before the next).
// Thread (warp w, lane l) owns tile row 32*(w%4)+l, the TMEM lane it may access.  Per
// layer: wait on the tile's commit barrier -> tcgen05.ld -> ReLU + cvt.rn.relu.bf16x2 ->
// tcgen05.st into the A columns -> warpgroup barrier (bar.red.and carrying the "no
// timeout" vote) -> an elected lane of warp g % 4 of warpgroup g issues the next layer's MMAs
// and commits them (so the five issuing warps spread over the SM's four sub-partitions).  In the BF16 fixed-sequence kernels the last hidden layer's FP16 operand goes to
// accumulator columns [64, 96), the next wavelet's first-layer operand hash(p) * E_k+1 is
// written into the A columns while the output MMA runs, and T_k's clamped Kahan sum is formed
// after the hand-off to that next wavelet; the FP32-dot forms do all three in the last hidden
// layer's epilogue.  In the BF16 fixed-sequence kernels the embedding rows and strengths those
// two steps read come from per-warpgroup shared-memory rings that a non-issuing warp fills by
// cp.async, eight wavelets ahead of use: read from L2 they put two L2 latencies on every
// wavelet's chain.  Warpgroups take tiles from a per-launch counter, so tiles of different
// cost (requests of different K) balance across the SMs.  The two standard networks run
// kernels specialised on their layer sequence (ShapeOf), every other supported network a
// generic form that reads the sequence from the plan.  Every wait is bounded by
// %globaltimer (2 s); on expiry the kernel records kDevWaitTimeout and the warpgroup
// unwinds together.
#include <cuda.h>  // CUtensorMap; cuTensorMapEncodeTiled is resolved through the runtime

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "nwprt_internal.cuh"

namespace nwprt {
namespace {

constexpr int kNWG = 5;                    // warpgroups per CTA, one tile each
constexpr int kThreads = 128 * kNWG;
constexpr int kTile = 128;                 // pixels per tile (MMA M)
constexpr int kAuxBytes = kTile * 16 * 2;  // 128 x 16 bf16 aux operand
constexpr int kTmemCols = 512;
constexpr int kTileCols = 96;              // TMEM columns per tile
constexpr int kAcol = 0;                   // A operand columns [0, 32)
constexpr int kDcol = 32;                  // accumulator columns [32, 96)
constexpr uint64_t kWaitNs = 2000000000ull;
// The job table travels inside the kernel parameters (sm_100 takes up to 32 KB): a launch
// needs no host->device copy that could queue behind an unrelated bulk transfer.  Larger
// batches are split into several launches.
constexpr int kInlineJobs = 256;
static_assert(kNWG * kTileCols <= kTmemCols, "TMEM budget");

// The weight blob is loaded with TMA through a 2-D view: rows of kWRowBytes bytes, in
// w_boxes boxes of w_box_rows rows (the last box may extend past the blob; its rows read as
// zeros and land inside the shared-memory weight region, which holds whole boxes).
constexpr uint32_t kWRowBytes = 256;
constexpr uint32_t kWMaxBoxRows = 256;

struct TcParams {
  CUtensorMap wmap;  // the weight blob, [rows][kWRowBytes / 4] uint32
  HashLevels hl;
  const float* hash;
  uint32_t wblob_bytes;
  uint32_t w_boxes, w_box_rows;
  uint32_t out_b_off, out_sbo;  // BF16: the output layer's FP16 B tile (V_last) in the blob
  TcLayer layers[kMaxTcLayers];
  int n_layers;
  int enc_dims;  // D, multiple of 16, <= 32
  TcJob jobs[kInlineJobs];
  int n_jobs;
  long long total_tiles;
  int kahan, clamp;
  float cp_scale;   // FP8: scale of the first layer's operand
  uint32_t* amax;   // calibration: per-layer activation maxima (float bits)
  uint32_t* err;
  int* tile_ctr;    // the next 128-pixel tile to take (zeroed before the launch)
  // Shared-memory descriptors of every layer's B tile, its aux block and the output layer's
  // FP16 tile, formed on the host with the weight region at address 0: the kernel adds the
  // region's address (>> 4, no carry out of the 14-bit field below 256 KB) in one step.
  uint64_t bdesc[kMaxTcLayers], auxdesc[kMaxTcLayers], outdesc;
  // V_last, the FP32 3 x 64 output layer.  From the parameter space every output-dot FMA
  // takes its weight pair as an operand, without a shared-memory load.
  float vlast[3][64];
};
static_assert(sizeof(TcParams) <= 32764, "kernel parameters are limited to 32,764 bytes");

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

// Wait for the phase with `parity`, bounded by limit_ns of wall time (kWaitNs in the kernels).
__device__ __forceinline__ bool wait_bounded(uint64_t* bar, uint32_t parity, uint32_t* err,
                                             uint64_t limit_ns = kWaitNs) {
  const uint32_t a = smem_u32(bar);
  if (mbar_try(a, parity)) return true;
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 1; it < (1u << 30); ++it) {
    if (mbar_try(a, parity)) return true;
    if ((it & 255u) == 0 && globaltimer() - t0 > limit_ns) break;
  }
  atomicCAS(err, 0u, (uint32_t)kDevWaitTimeout);
  return false;
}

// One lane of a converged warp (elect.sync).  Issuing tcgen05.mma from an elected lane of a
// converged warp is about twice as fast as from a lone lane whose warp has diverged: back to
// back M=128 N=64 MMAs take ~36 cycles each instead of ~75.
__device__ __forceinline__ bool elect_one() {
  uint32_t e;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "elect.sync _|p, 0xffffffff;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(e));
  return e != 0;
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

__host__ __device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1, no swizzle
}

// kind::f16 instruction descriptor: D=F32, A=B=BF16, both K-major, M=128.
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
// kind::f16 instruction descriptor: D=F32, A=B=F16 (format code 0), both K-major, M=128.
__host__ __device__ constexpr uint32_t idesc_f16(int n) {
  return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
// kind::f8f6f4 instruction descriptor: D=F32, A=B=E4M3 (format code 0), both K-major, M=128.
__host__ __device__ constexpr uint32_t idesc_e4m3(int n) {
  return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
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

// D[tmem] (+)= A[tmem] * B[smem]^T with E4M3 operands (K = 32 per instruction)
__device__ __forceinline__ void mma_ts_e4m3(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
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


__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
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
// ReLU(lo), ReLU(hi) -> an FP16 pair (round to nearest even, saturated to the largest finite
// FP16), lo in the low half.
__device__ __forceinline__ uint32_t pack_f16_relu(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.satfinite.relu.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}
// Four FP32 values -> four E4M3 bytes (round to nearest even, saturated to +-448), x0 in
// the lowest byte: the K order of an 8-bit operand in one 32-bit TMEM column.
template <bool RELU>
__device__ __forceinline__ uint32_t pack_e4m3x4(float x0, float x1, float x2, float x3) {
  unsigned short lo, hi;
  if (RELU) {
    asm("cvt.rn.satfinite.relu.e4m3x2.f32 %0, %1, %2;" : "=h"(lo) : "f"(x1), "f"(x0));
    asm("cvt.rn.satfinite.relu.e4m3x2.f32 %0, %1, %2;" : "=h"(hi) : "f"(x3), "f"(x2));
  } else {
    asm("cvt.rn.satfinite.e4m3x2.f32 %0, %1, %2;" : "=h"(lo) : "f"(x1), "f"(x0));
    asm("cvt.rn.satfinite.e4m3x2.f32 %0, %1, %2;" : "=h"(hi) : "f"(x3), "f"(x2));
  }
  return (uint32_t)lo | ((uint32_t)hi << 16);
}
__device__ __forceinline__ float bf16_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }

// Asynchronous global -> shared copies (cp.async): 16 bytes bypassing L1, or 4 bytes.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d)
               : "memory");
}

// Byte offset of (row, 16-byte K chunk) in a canonical no-swizzle K-major tile whose
// 8-row groups are `sbo` bytes apart.
__device__ __forceinline__ uint32_t core_off(int row, int chunk, uint32_t sbo) {
  return (uint32_t)(row >> 3) * sbo + (uint32_t)chunk * 128u + (uint32_t)(row & 7) * 16u;
}

// 32 FP32 TMEM values (times `scale`, a uniform per-layer value) -> 8 E4M3 quads.
template <bool RELU>
__device__ __forceinline__ void pack32_e4m3(const uint32_t (&v)[32], float scale, uint32_t* out) {
  if (scale == 1.f) {
#pragma unroll
    for (int j = 0; j < 8; ++j)
      out[j] = pack_e4m3x4<RELU>(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]),
                                 __uint_as_float(v[4 * j + 2]), __uint_as_float(v[4 * j + 3]));
  } else {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float x[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) x[i] = __fmul_rn(__uint_as_float(v[4 * j + i]), scale);
      out[j] = pack_e4m3x4<RELU>(x[0], x[1], x[2], x[3]);
    }
  }
}

// Largest value this warp passes to the next layer (ReLU'd, or |v| for a linear layer),
// folded into the layer's calibration maximum.  Non-negative floats order like their bits.
__device__ __forceinline__ uint32_t amax32(const uint32_t (&v)[32], bool relu) {
  float m = 0.f;
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    const float x = __uint_as_float(v[i]);
    m = fmaxf(m, relu ? x : fabsf(x));
  }
  return __float_as_uint(m);
}
__device__ __forceinline__ void record_amax(uint32_t* slot, uint32_t bits) {
  bits = __reduce_max_sync(0xffffffffu, bits);
  if ((threadIdx.x & 31) == 0) atomicMax(slot, bits);
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

// 32 FP32 TMEM values -> 16 ReLU'd FP16 pairs.
__device__ __forceinline__ void pack32_f16_relu(const uint32_t (&v)[32], uint32_t* out) {
#pragma unroll
  for (int j = 0; j < 16; ++j) out[j] = pack_f16_relu(__uint_as_float(v[2 * j]), __uint_as_float(v[2 * j + 1]));
}

// Two FP32 values in one 64-bit register, for the packed f32x2 arithmetic of sm_100.
__device__ __forceinline__ unsigned long long pk2(float x, float y) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ void fma2(unsigned long long& acc, unsigned long long a, unsigned long long b) {
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(a), "l"(b));
}
__device__ __forceinline__ float sum2(unsigned long long x) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(x));
  return __fadd_rn(lo, hi);
}
// T += V_last[:, j0:j0+32] relu(h[j0:j0+32]) in FP32 with packed FMAs: q_c holds the
// partial sums of channel c over even and odd j, added once at the end (sum2).  V is the
// kernel-parameter copy of V_last.
__device__ __forceinline__ void final_dot32x2(const uint32_t (&v)[32], const float (&V)[3][64], int j0,
                                              unsigned long long& q0, unsigned long long& q1, unsigned long long& q2) {
#pragma unroll
  for (int j2 = 0; j2 < 16; ++j2) {
    const int j = j0 + 2 * j2;
    const unsigned long long h =
        pk2(fmaxf(__uint_as_float(v[2 * j2]), 0.f), fmaxf(__uint_as_float(v[2 * j2 + 1]), 0.f));
    fma2(q0, pk2(V[0][j], V[0][j + 1]), h);
    fma2(q1, pk2(V[1][j], V[1][j + 1]), h);
    fma2(q2, pk2(V[2][j], V[2][j + 1]), h);
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

// A tile's hash features in shared memory: one row of DMAX / 2 BF16 pairs per pixel, in
// 16-byte chunks whose order within the row is XOR-swizzled by the row, so that a warp's
// 16-byte loads of one chunk index (32 consecutive rows) are free of bank conflicts.
template <int DMAX>
struct EncRow {
  static constexpr int kChunks = DMAX / 8;  // 16-byte chunks per row: 4 or 2
  uint4* base;                              // this row
  int swz;
  __device__ __forceinline__ EncRow(uint32_t* tile_encs, int row)
      : base(reinterpret_cast<uint4*>(tile_encs) + row * kChunks),
        swz(kChunks == 4 ? (row >> 1) & 3 : (row >> 2) & 1) {}
  __device__ __forceinline__ uint4 get(int c) const { return base[c ^ swz]; }
  __device__ __forceinline__ void put(int c, uint4 v) const { base[c ^ swz] = v; }
};

// First-layer operand of wavelet k, hash(p) * E_k -> TMEM A columns.  BF16: one packed
// bf16x2 multiply per feature pair of the BF16 hash features and the BF16 embedding row eh
// (the exact product, rounded once).  Calibration: the same product from the FP32 row ek,
// recording max |hash(p) * E_k| in amax[0].  FP8: from the FP32 row, scaled by cp_scale and
// rounded to E4M3, zero-padded to K = 32.
template <int DMAX, int MODE>
__device__ __forceinline__ void store_cp(const EncRow<DMAX>& enc, const float* __restrict__ ek,
                                         const uint32_t* __restrict__ eh, uint32_t a_taddr, float cp_scale,
                                         uint32_t* amax) {
  constexpr int NW = MODE == kTcFp8 ? 8 : DMAX / 2;
  uint32_t cp[NW];
  if constexpr (MODE == kTcBf16) {
#pragma unroll
    for (int c = 0; c < DMAX / 8; ++c) {
      const uint4 e = __ldg(reinterpret_cast<const uint4*>(eh) + c);
      const uint4 h = enc.get(c);
      const uint32_t ev[4] = {e.x, e.y, e.z, e.w}, hv[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
      for (int i = 0; i < 4; ++i) asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(cp[c * 4 + i]) : "r"(hv[i]), "r"(ev[i]));
    }
    if constexpr (DMAX == 32) tmem_st16(a_taddr, cp);
    else tmem_st8(a_taddr, cp);
    return;
  }
  float m = 0.f;
#pragma unroll
  for (int c = 0; c < DMAX / 8; ++c) {
    const float4 e0 = __ldg(reinterpret_cast<const float4*>(ek + c * 8));
    const float4 e1 = __ldg(reinterpret_cast<const float4*>(ek + c * 8 + 4));
    const uint4 h = enc.get(c);
    const uint32_t h0 = h.x, h1 = h.y, h2 = h.z, h3 = h.w;
    const float x0 = __fmul_rn(bf16_lo(h0), e0.x), x1 = __fmul_rn(bf16_hi(h0), e0.y);
    const float x2 = __fmul_rn(bf16_lo(h1), e0.z), x3 = __fmul_rn(bf16_hi(h1), e0.w);
    const float x4 = __fmul_rn(bf16_lo(h2), e1.x), x5 = __fmul_rn(bf16_hi(h2), e1.y);
    const float x6 = __fmul_rn(bf16_lo(h3), e1.z), x7 = __fmul_rn(bf16_hi(h3), e1.w);
    if constexpr (MODE == kTcFp8) {
      cp[c * 2] = pack_e4m3x4<false>(__fmul_rn(x0, cp_scale), __fmul_rn(x1, cp_scale), __fmul_rn(x2, cp_scale),
                                     __fmul_rn(x3, cp_scale));
      cp[c * 2 + 1] = pack_e4m3x4<false>(__fmul_rn(x4, cp_scale), __fmul_rn(x5, cp_scale), __fmul_rn(x6, cp_scale),
                                         __fmul_rn(x7, cp_scale));
    } else {
      cp[c * 4 + 0] = pack_bf16(x0, x1);
      cp[c * 4 + 1] = pack_bf16(x2, x3);
      cp[c * 4 + 2] = pack_bf16(x4, x5);
      cp[c * 4 + 3] = pack_bf16(x6, x7);
    }
    if constexpr (MODE == kTcCalibrate)
      m = fmaxf(m, fmaxf(fmaxf(fmaxf(fabsf(x0), fabsf(x1)), fmaxf(fabsf(x2), fabsf(x3))),
                         fmaxf(fmaxf(fabsf(x4), fabsf(x5)), fmaxf(fabsf(x6), fabsf(x7)))));
  }
  if constexpr (MODE == kTcFp8) {
#pragma unroll
    for (int i = DMAX / 4; i < 8; ++i) cp[i] = 0u;
    tmem_st8(a_taddr, cp);
  } else {
    if constexpr (DMAX == 32) tmem_st16(a_taddr, cp);
    else tmem_st8(a_taddr, cp);
  }
  if constexpr (MODE == kTcCalibrate) record_amax(amax, __float_as_uint(m));
}

// store_cp's BF16 form with the embedding row taken from shared memory.
template <int DMAX>
__device__ __forceinline__ void store_cp_smem(const EncRow<DMAX>& enc, const uint4* e_row, uint32_t a_taddr) {
  uint32_t cp[DMAX / 2];
#pragma unroll
  for (int c = 0; c < DMAX / 8; ++c) {
    const uint4 e = e_row[c], h = enc.get(c);
    const uint32_t ev[4] = {e.x, e.y, e.z, e.w}, hv[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(cp[c * 4 + i]) : "r"(hv[i]), "r"(ev[i]));
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

constexpr int kBatch = 8, kRing = 2 * kBatch;
struct __align__(16) TcBarriers {
  // Per warpgroup, rings of kRing slots: the BF16 embedding rows E_j (read for wavelet j's
  // first-layer operand) and the strengths L_j (read after wavelet j's output layer), copied
  // in by cp.async kBatch wavelets at a time (slot j % kRing).
  uint4 e_ring[kNWG][kRing][4];
  float4 l_ring[kNWG][kRing];
  uint64_t acc_full[kNWG];  // MMA commit -> epilogue of that warpgroup's tile
  uint64_t done[kNWG];      // final commit before TMEM is released
  uint64_t wload;           // the weight blob's TMA load
  uint32_t tmem_base;
  int tile_slot[kNWG];      // the tile each warpgroup took from the launch's counter
};

// Shared-memory bytes of the weight region: whole TMA boxes, rounded to 1 KB.
__host__ __device__ inline uint32_t weight_region_bytes(uint32_t boxes, uint32_t box_rows) {
  return (boxes * box_rows * kWRowBytes + 1023u) & ~1023u;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Layer sequences fixed at compile time, so that the per-layer flags are constants and the
// layer loop unrolls (the plan still supplies offsets, strides and scales).  kShapePlan: the
// sequence is read from the plan at run time.  Both fixed shapes have 64-wide ReLU layers,
// one of them with the aux block and the last one fin:
//   kShapeSix: out_prd 32->64->64->64, folded cmp_net first layer (+aux), two 64->64 layers;
//   kShapeTwo: folded cmp_net first layer (+aux) on 16 hash features, one 64->64 layer.
enum TcShape { kShapePlan = 0, kShapeSix = 1, kShapeTwo = 2 };
template <int SHAPE> struct ShapeOf { static constexpr int nl = 0, aux = -1; };
template <> struct ShapeOf<kShapeSix> { static constexpr int nl = 6, aux = 3; };
template <> struct ShapeOf<kShapeTwo> { static constexpr int nl = 2, aux = 0; };

// S K-steps of one layer, unrolled: step s reads 8 more TMEM columns of A and the next two
// 128-byte core-matrix columns of B (+16 in the descriptor's address field, which counts
// 16-byte units).
template <int MODE, int S>
__device__ __forceinline__ void issue_steps(uint32_t d_tmem, uint32_t a_tmem, uint64_t b0, uint32_t id) {
#pragma unroll
  for (int s = 0; s < S; ++s) {
    if constexpr (MODE == kTcFp8)
      mma_ts_e4m3(d_tmem, a_tmem + (uint32_t)s * 8u, b0 + (uint64_t)(s * 16), id, s > 0 ? 1u : 0u);
    else
      mma_ts(d_tmem, a_tmem + (uint32_t)s * 8u, b0 + (uint64_t)(s * 16), id, s > 0 ? 1u : 0u);
  }
}

// Issues layer L of warpgroup g's tile: A from TMEM (and the aux block from shared memory).
// A K step covers 32 bytes of a row in both precisions (16 BF16 or 32 E4M3 values): 8 TMEM
// columns of A and two 128-byte core-matrix columns of B.  The aux block stays BF16 in both;
// its MMA accumulates into the same FP32 accumulator.  The K loop is unrolled for each step
// count the plans produce (1, 2 or 4): issuing with descriptors computed in a run-time loop
// made every layer's round trip measurably longer.
template <int MODE>
__device__ __forceinline__ void issue_layer(const TcLayer& L, bool with_aux, uint32_t wbase, uint32_t a_tmem,
                                            uint32_t aux_base, uint32_t d_tmem, uint64_t* bar) {
  tc_fence_after();
  const uint64_t b0 = smem_desc(wbase + L.b_off, 128u, L.b_sbo);
  const uint32_t id = MODE == kTcFp8 ? idesc_e4m3(L.n) : idesc_bf16(L.n);
  const int steps = L.k / (MODE == kTcFp8 ? 32 : 16);
  if (steps == 4) issue_steps<MODE, 4>(d_tmem, a_tmem, b0, id);
  else if (steps == 2) issue_steps<MODE, 2>(d_tmem, a_tmem, b0, id);
  else if (steps == 1) issue_steps<MODE, 1>(d_tmem, a_tmem, b0, id);
  else issue_steps<MODE, 3>(d_tmem, a_tmem, b0, id);
  if (with_aux) {
    const uint64_t ad = smem_desc(aux_base, 128u, 256u);
    const uint64_t bd = smem_desc(wbase + L.aux_off, 128u, 256u);
    mma_ss(d_tmem, ad, bd, idesc_bf16(L.n), 1u);
  }
  mma_commit(bar);
}

// Layer L of a fixed layer sequence: every layer is 64 wide, the step count and the aux flag
// are compile-time, and the descriptors come precomputed (b0, bd: the weight region's
// address already added; ad: the warpgroup's aux block).  Nothing between the warpgroup
// barrier and the first MMA but the fence and the descriptor add.
template <int MODE, int S, bool AUX>
__device__ __forceinline__ void issue_fixed(uint64_t b0, uint64_t ad, uint64_t bd, uint32_t a_tmem, uint32_t d_tmem,
                                            uint64_t* bar) {
  tc_fence_after();
  issue_steps<MODE, S>(d_tmem, a_tmem, b0, MODE == kTcFp8 ? idesc_e4m3(64) : idesc_bf16(64));
  if (AUX) mma_ss(d_tmem, ad, bd, idesc_bf16(64), 1u);
  mma_commit(bar);
}

template <int DMAX, int MODE, int SHAPE>
__global__ void __launch_bounds__(kThreads, 1) relight_tc_kernel(const __grid_constant__ TcParams p) {
  using Sh = ShapeOf<SHAPE>;
  // BF16 with a fixed layer sequence: the 64 -> 3 output layer is one more tensor-core step
  // (FP16 operands, FP32 accumulation) instead of an FP32 dot on the CUDA cores
  constexpr bool OUT_TC = MODE == kTcBf16 && SHAPE != kShapePlan;
  const int n_layers = SHAPE ? Sh::nl : p.n_layers;
  const int n_steps = n_layers + (OUT_TC ? 1 : 0);  // tensor-core steps per wavelet
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* wsm = smem;                                                  // weight blob
  uint8_t* aux = smem + weight_region_bytes(p.w_boxes, p.w_box_rows);  // [kNWG][kAuxBytes]
  uint32_t* encs = reinterpret_cast<uint32_t*>(aux + kNWG * kAuxBytes);  // [kNWG][kTile][DMAX/2], swizzled
  TcBarriers* bars = reinterpret_cast<TcBarriers*>(encs + kNWG * (DMAX / 2) * kTile);
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = warp >> 2;  // warpgroup
  const int q = warp & 3;   // TMEM lane quarter this warp may access
  const int row = q * 32 + lane;

  // ---- barriers, then the weights -> shared memory by TMA (one load per box), and TMEM
  if (tid == 0) {
    for (int w = 0; w < kNWG; ++w) {
      mbar_init(&bars->acc_full[w], 1);
      mbar_init(&bars->done[w], 1);
    }
    mbar_init(&bars->wload, 1);
    fence_barrier_init();
    mbar_arrive_expect_tx(&bars->wload, p.w_boxes * p.w_box_rows * kWRowBytes);
    for (uint32_t b = 0; b < p.w_boxes; ++b)
      tma_load_2d(wsm + b * p.w_box_rows * kWRowBytes, &p.wmap, 0, (int)(b * p.w_box_rows), &bars->wload);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&bars->tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  // the weights have landed (every thread sees the barrier complete before any MMA reads them)
  bool ok = wait_bounded(&bars->wload, 0, p.err);
  const uint32_t tmem = bars->tmem_base;
  const uint32_t wbase = smem_u32(wsm);
  const uint32_t col0 = tmem + (uint32_t)(g * kTileCols);
  const uint32_t a_tmem = col0 + kAcol;                                 // MMA operand address (lane 0)
  const uint32_t d_tmem = col0 + kDcol;
  const uint32_t a_taddr = a_tmem + ((uint32_t)(q * 32) << 16);         // this warp's lanes
  const uint32_t d_taddr = d_tmem + ((uint32_t)(q * 32) << 16);
  const uint32_t aux_base = smem_u32(aux + g * kAuxBytes);
  const uint32_t aux_row = aux_base + core_off(row, 0, 256u);
  uint64_t* acc_bar = &bars->acc_full[g];
  // The warp that issues this warpgroup's MMAs.  Warp w runs on SM sub-partition w % 4, so
  // taking warp g % 4 of warpgroup g spreads the five issuing warps over the four
  // sub-partitions instead of stacking them on one.
  const int lead = g & 3;
  const int fetcher = (g + 1) & 3;  // the warp that fills the warpgroup's rings (never the issuer)
  const uint64_t wb16 = (uint64_t)(wbase >> 4);
  const uint64_t aux_desc = smem_desc(aux_base, 128u, 256u);
  // fixed sequences: K steps of the first layer (hash features) and of the 64-wide ones
  constexpr int kS0 = MODE == kTcFp8 ? 1 : DMAX / 16;
  constexpr int kS1 = MODE == kTcFp8 ? 2 : 4;
  auto issue_next = [&](int nl) {
    if constexpr (SHAPE != kShapePlan) {
      if (OUT_TC && nl == n_layers) {
        tc_fence_after();
        issue_steps<kTcBf16, 4>(d_tmem, d_tmem + 32u, p.outdesc + wb16, idesc_f16(16));
        mma_commit(acc_bar);
      } else if (nl == 0) {
        issue_fixed<MODE, kS0, Sh::aux == 0>(p.bdesc[0] + wb16, aux_desc, p.auxdesc[0] + wb16, a_tmem, d_tmem,
                                              acc_bar);
      } else if (nl == Sh::aux) {
        issue_fixed<MODE, kS1, true>(p.bdesc[nl] + wb16, aux_desc, p.auxdesc[nl] + wb16, a_tmem, d_tmem, acc_bar);
      } else {
        issue_fixed<MODE, kS1, false>(p.bdesc[nl] + wb16, aux_desc, 0ull, a_tmem, d_tmem, acc_bar);
      }
    } else {
      issue_layer<MODE>(p.layers[nl], Sh::aux >= 0 ? Sh::aux == nl : p.layers[nl].aux != 0, wbase, a_tmem, aux_base,
                        d_tmem, acc_bar);
    }
  };

  uint32_t ph = 0;
  // Tiles come from the launch's counter, one atomic per tile and warpgroup, so that tiles of
  // different cost (jobs of different K or pixel count; the host puts the longest tiles first)
  // balance across the SMs.  The slot is read after a warpgroup barrier and rewritten only after
  // the next one (every tile has at least one).
  if (q == 0 && lane == 0) bars->tile_slot[g] = atomicAdd(p.tile_ctr, 1);
  ok = wg_barrier_and(g, ok);
  for (long long t = bars->tile_slot[g]; t < p.total_tiles && ok; t = bars->tile_slot[g]) {
    // ---- tile set-up: hash encoding, aux operand, first-layer operand of wavelet 0
    const int jid = find_job(p.jobs, p.n_jobs, t);
    const TcJob& J = p.jobs[jid];
    const int K = J.K;
    const long long px = J.px_begin + (t - J.tile_begin) * kTile + row;
    const bool valid = px < J.n_px;
    const EncRow<DMAX> enc_s(encs + g * (DMAX / 2) * kTile, row);  // this pixel's features
    if (valid) {
      uint32_t enc[DMAX / 2];
      const float4* pr = reinterpret_cast<const float4*>(J.packed) + px * 4;
      const float4 r0 = __ldg(pr), r1 = __ldg(pr + 1), r2 = __ldg(pr + 2), r3 = __ldg(pr + 3);
      hash_encode_bf16<DMAX>(p.hl, p.hash, r0.x, r0.y, r0.z, enc);
#pragma unroll
      for (int c = 0; c < DMAX / 8; ++c)
        enc_s.put(c, make_uint4(enc[4 * c], enc[4 * c + 1], enc[4 * c + 2], enc[4 * c + 3]));
      // aux operand: the 13 remapped G-buffer values followed by ones
      st_shared_v4(aux_row, pack_bf16(r0.w, r1.x), pack_bf16(r1.y, r1.z), pack_bf16(r1.w, r2.x),
                   pack_bf16(r2.y, r2.z));
      st_shared_v4(aux_row + 128u, pack_bf16(r2.w, r3.x), pack_bf16(r3.y, r3.z), pack_bf16(r3.w, 1.f),
                   pack_bf16(1.f, 1.f));
    } else {
#pragma unroll
      for (int c = 0; c < DMAX / 8; ++c) enc_s.put(c, make_uint4(0u, 0u, 0u, 0u));
      st_shared_v4(aux_row, 0, 0, 0, 0);
      st_shared_v4(aux_row + 128u, 0, 0, 0, 0);
    }
    store_cp<DMAX, MODE>(enc_s, J.emb_k, J.emb_h, a_taddr, p.cp_scale, p.amax);
    tmem_wait_st();
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
    // hand the first layer to the tensor core
    tc_fence_before();
    fence_proxy_async_smem();
    ok = wg_barrier_and(g, ok);
    if (ok && q == lead && elect_one()) issue_next(0);
    // T_k -> clamped Kahan sums, then the next wavelet's first-layer operand
    auto finish_wavelet = [&](int k, float t0, float t1, float t2) {
      float L0, L1, L2;
      if constexpr (OUT_TC) {
        const float4 Lk = bars->l_ring[g][k % kRing];
        L0 = Lk.x; L1 = Lk.y; L2 = Lk.z;
      } else {
        const float* Lk = J.strength + (size_t)k * 3;
        L0 = __ldg(Lk + 0); L1 = __ldg(Lk + 1); L2 = __ldg(Lk + 2);
      }
      float u0 = __fmul_rn(L0, t0);
      float u1 = __fmul_rn(L1, t1);
      float u2 = __fmul_rn(L2, t2);
      if (p.clamp) { u0 = fmaxf(u0, 0.f); u1 = fmaxf(u1, 0.f); u2 = fmaxf(u2, 0.f); }
      if (p.kahan) {
        float y, z;
        y = __fsub_rn(u0, c0); z = __fadd_rn(s0, y); c0 = __fsub_rn(__fsub_rn(z, s0), y); s0 = z;
        y = __fsub_rn(u1, c1); z = __fadd_rn(s1, y); c1 = __fsub_rn(__fsub_rn(z, s1), y); s1 = z;
        y = __fsub_rn(u2, c2); z = __fadd_rn(s2, y); c2 = __fsub_rn(__fsub_rn(z, s2), y); s2 = z;
      } else {
        s0 = __fadd_rn(s0, u0); s1 = __fadd_rn(s1, u1); s2 = __fadd_rn(s2, u2);
      }
      if (!OUT_TC && k + 1 < K) {  // OUT_TC: written while the output layer's MMA runs
        store_cp<DMAX, MODE>(enc_s, J.emb_k + (size_t)(k + 1) * p.enc_dims,
                             J.emb_h + (size_t)(k + 1) * (p.enc_dims / 2), a_taddr, p.cp_scale, p.amax);
        tmem_wait_st();
      }
    };
    float tk0 = 0.f, tk1 = 0.f, tk2 = 0.f;  // OUT_TC: T_k, summed during the next wavelet
    for (int k = 0; k < K && ok; ++k) {
#pragma unroll(SHAPE ? Sh::nl + (OUT_TC ? 1 : 0) : 1)
      for (int l = 0; l < n_steps; ++l) {
        const TcLayer& L = p.layers[l < n_layers ? l : 0];
        const bool is_out = OUT_TC && l == n_layers;       // the output layer's accumulator
        const bool pre_out = OUT_TC && l == n_layers - 1;  // the last hidden layer, packed as FP16
        const bool fin = !OUT_TC && (SHAPE ? l == Sh::nl - 1 : L.fin != 0);
        const bool relu = SHAPE ? true : L.relu != 0;
        const bool wide_out = SHAPE ? true : L.n > 32;
        const bool waited = __all_sync(0xffffffffu, wait_bounded(acc_bar, ph, p.err));
        ph ^= 1u;
        if (waited) {
          tc_fence_after();
          uint32_t v[32];
          if (is_out) {
            uint32_t t[4];
            tmem_ld4(d_taddr, t);
            tmem_wait_ld();
            tk0 = __uint_as_float(t[0]);
            tk1 = __uint_as_float(t[1]);
            tk2 = __uint_as_float(t[2]);
          } else if (pre_out) {
            // the output layer's operand goes to accumulator columns [64, 96) (the second half
            // is read before its columns are overwritten), leaving the A columns free for the
            // next wavelet's first-layer operand while the output MMA runs
            uint32_t a[16];
            tmem_ld32(d_taddr + 32u, v);
            tmem_wait_ld();
            pack32_f16_relu(v, a);
            tmem_st16(d_taddr + 48u, a);
            tmem_ld32(d_taddr, v);
            tmem_wait_ld();
            pack32_f16_relu(v, a);
            tmem_st16(d_taddr + 32u, a);
            tmem_wait_st();
          } else if (!fin && MODE == kTcFp8) {
            uint32_t a[8];
            tmem_ld32(d_taddr, v);
            tmem_wait_ld();
            if (relu) pack32_e4m3<true>(v, L.scale, a);
            else pack32_e4m3<false>(v, L.scale, a);
            tmem_st8(a_taddr, a);
            if (wide_out) {
              tmem_ld32(d_taddr + 32u, v);
              tmem_wait_ld();
              if (relu) pack32_e4m3<true>(v, L.scale, a);
              else pack32_e4m3<false>(v, L.scale, a);
              tmem_st8(a_taddr + 8u, a);
            }
            tmem_wait_st();
          } else if (!fin) {
            uint32_t a[16];
            uint32_t m = 0;
            tmem_ld32(d_taddr, v);
            tmem_wait_ld();
            if constexpr (MODE == kTcCalibrate) m = amax32(v, relu);
            if (relu) pack32<true>(v, a);
            else pack32<false>(v, a);
            tmem_st16(a_taddr, a);
            if (wide_out) {
              tmem_ld32(d_taddr + 32u, v);
              tmem_wait_ld();
              if constexpr (MODE == kTcCalibrate) m = max(m, amax32(v, relu));
              if (relu) pack32<true>(v, a);
              else pack32<false>(v, a);
              tmem_st16(a_taddr + 16u, a);
            }
            if constexpr (MODE == kTcCalibrate) record_amax(p.amax + l + 1, m);
            tmem_wait_st();
          } else {
            float t0 = 0.f, t1 = 0.f, t2 = 0.f;
            uint32_t m = 0;
            tmem_ld32(d_taddr, v);
            tmem_wait_ld();
            if constexpr (MODE == kTcCalibrate) m = amax32(v, true);
            unsigned long long q0 = 0ull, q1 = 0ull, q2 = 0ull;
            final_dot32x2(v, p.vlast, 0, q0, q1, q2);
            tmem_ld32(d_taddr + 32u, v);
            tmem_wait_ld();
            if constexpr (MODE == kTcCalibrate) record_amax(p.amax + n_layers, max(m, amax32(v, true)));
            final_dot32x2(v, p.vlast, 32, q0, q1, q2);
            t0 = sum2(q0); t1 = sum2(q1); t2 = sum2(q2);
            finish_wavelet(k, t0, t1, t2);
          }
        }
        ok = ok && waited;
        if (l + 1 == n_steps && k + 1 == K) {  // the tile's last step: no hand-off
          if (is_out && waited) finish_wavelet(k, tk0, tk1, tk2);
          break;
        }
        const int nl = (l + 1 == n_steps) ? 0 : l + 1;
        if (pre_out && q == fetcher) cp_async_wait_all();  // the rings, before this barrier
        tc_fence_before();
        ok = wg_barrier_and(g, ok);
        if (!ok) break;
        if (q == lead && elect_one()) issue_next(nl);
        if (OUT_TC && l == 0 && q == fetcher && k % kBatch == 0) {
          // E_k+1..k+8 and L_k..k+7 into the rings, by a warp that would otherwise only wait
          // for this layer's MMAs; waited for before this wavelet's last hidden-layer barrier
          constexpr int C = DMAX / 8;
          const int j = lane / C;
          if (j < kBatch && k + 1 + j < K)
            cp_async16(smem_u32(&bars->e_ring[g][(k + 1 + j) % kRing][lane % C]),
                       J.emb_h + (size_t)(k + 1 + j) * (p.enc_dims / 2) + (lane % C) * 4);
          if (lane < 3 * kBatch && k + lane / 3 < K)
            cp_async4(smem_u32(reinterpret_cast<float*>(&bars->l_ring[g][(k + lane / 3) % kRing]) + lane % 3),
                      J.strength + (size_t)k * 3 + lane);
          cp_async_commit();
        }
        // T_k's clamped Kahan update waits one more step: under the next wavelet's second layer,
        // whose MMAs take longer than its first layer's, so that it stays off the chain
        if (OUT_TC && l == 1 && k > 0) finish_wavelet(k - 1, tk0, tk1, tk2);
        if (OUT_TC && nl == n_layers && k + 1 < K) {
          // the next wavelet's first-layer operand into the A columns, which the output MMA
          // (operand in [64, 96), accumulator in [32, 48)) does not touch
          store_cp_smem<DMAX>(enc_s, bars->e_ring[g][(k + 1) % kRing], a_taddr);
          tmem_wait_st();
        }
      }
    }
    if (valid && ok) {
      const float4 ind = J.flag[px] ? make_float4(s0, s1, s2, 1.f) : make_float4(0.f, 0.f, 0.f, 1.f);
      const float4 dl = __ldg(reinterpret_cast<const float4*>(J.direct) + px);
      reinterpret_cast<float4*>(J.indirect)[px] = ind;
      reinterpret_cast<float4*>(J.with_direct)[px] =
          make_float4(__fadd_rn(ind.x, dl.x), __fadd_rn(ind.y, dl.y), __fadd_rn(ind.z, dl.z), 1.f);
    }
    // every thread of the warpgroup agrees on the outcome (and sees the next tile) before it
    if (q == 0 && lane == 0) bars->tile_slot[g] = atomicAdd(p.tile_ctr, 1);
    ok = wg_barrier_and(g, ok);
  }
  if (OUT_TC && q == fetcher) cp_async_wait_all();  // no ring copy outlives the CTA (a timed-out exit)
  // every MMA this warpgroup issued has completed before TMEM is released
  if (q == lead && elect_one()) {  // the same lane that issued: a commit tracks its own thread's MMAs
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

// FP32 -> E4M3 (1 sign, 4 exponent bits with bias 7, 3 mantissa bits; no infinities; max
// finite 448), round to nearest even, saturated to +-448 like cvt.rn.satfinite.
uint8_t to_e4m3(float f) {
  if (std::isnan(f)) return 0x7f;
  const uint8_t sign = std::signbit(f) ? 0x80 : 0x00;
  const double a = std::fabs((double)f);
  if (a >= 464.0) return sign | 0x7e;  // 464 = halfway between 448 and the next step
  if (a < std::ldexp(1.0, -6)) {       // subnormal: multiples of 2^-9
    const double q = std::nearbyint(a * 512.0);
    return sign | (uint8_t)q;          // q == 8 is the smallest normal, code 0x08
  }
  int e;
  const double m = std::frexp(a, &e);  // a = m * 2^e, m in [0.5, 1)
  double q = std::nearbyint((m * 2.0 - 1.0) * 8.0);
  int E = e - 1;
  if (q >= 8.0) {
    q = 0.0;
    ++E;
  }
  if (E > 8 || (E == 8 && q > 6.0)) return sign | 0x7e;
  return sign | (uint8_t)(((E + 7) << 3) | (int)q);
}

// FP32 -> FP16 (1 sign, 5 exponent bits with bias 15, 10 mantissa bits), round to nearest
// even, overflow to infinity.
uint16_t to_f16(float f) {
  if (std::isnan(f)) return 0x7e00;
  const uint16_t sign = std::signbit(f) ? 0x8000 : 0x0000;
  const double a = std::fabs((double)f);
  if (a >= 65520.0) return sign | 0x7c00;  // 65520 = halfway between 65504 and the next step
  if (a < std::ldexp(1.0, -14)) return sign | (uint16_t)std::nearbyint(a * 16777216.0);  // multiples of 2^-24
  int e;
  const double m = std::frexp(a, &e);  // a = m * 2^e, m in [0.5, 1)
  double q = std::nearbyint((m * 2.0 - 1.0) * 1024.0);
  int E = e - 1;
  if (q >= 1024.0) {
    q = 0.0;
    ++E;
  }
  return sign | (uint16_t)(((E + 15) << 10) | (int)q);
}

int pad16(int x) { return (x + 15) & ~15; }
int pad32(int x) { return (x + 31) & ~31; }

// Writes the N x K (row-major [out][in]) block src[:, col0:col0+kc] * scale as a canonical
// K-major tile of np x kp elements (zero padded) of `eb` bytes each at byte offset `off`.
// Core matrices are 8 rows x 16 bytes; K-adjacent ones are 128 bytes apart, 8-row groups
// kp * eb * 8 bytes apart.
void put_b(std::vector<uint8_t>* blob, size_t off, const float* src, int n, int k_total, int col0, int kc,
           int np, int kp, int eb, float scale, bool f16 = false) {
  const size_t need = off + (size_t)np * kp * eb;
  if (blob->size() < need) blob->resize(need, 0);
  const size_t sbo = (size_t)kp * eb * 8;
  for (int r = 0; r < np; ++r)
    for (int c = 0; c < kp; ++c) {
      const float v = (r < n && c < kc) ? src[(size_t)r * k_total + col0 + c] * scale : 0.f;
      const size_t cb = (size_t)c * eb;  // byte column within the row
      const size_t byte = off + (size_t)(r >> 3) * sbo + (cb >> 4) * 128 + (size_t)(r & 7) * 16 + (cb & 15);
      if (eb == 2) {
        const uint16_t h = f16 ? to_f16(v) : to_bf16(v);
        std::memcpy(blob->data() + byte, &h, 2);
      } else {
        (*blob)[byte] = to_e4m3(v);
      }
    }
}

// Weights of one tensor-core layer: [n][k] row-major, plus [n][16] for the aux block.
struct LayerMat {
  int n, k;
  bool relu, aux;
  std::vector<float> w, waux;
};

// The tensor-core chain: out_prd's hidden layers; cmp_net's first layer with out_prd's
// output layer folded in; cmp_net's remaining hidden layers (the last one marked fin by the
// plan).  out_prd's output layer is linear (prt_network.h:49-53: no output activation) and
// feeds cmp_net's first layer directly (prt_network.h:116-131), so
//   relu(Wc [Wo h ; aux]) = relu((Wc[:, :m] Wo) h + Wc[:, m:] aux)        (m = op_out)
// exactly; the product Wc[:, :m] Wo is formed here in double, which saves one layer per
// wavelet.  With op or cn null only the shapes are filled.
std::vector<LayerMat> layer_mats(const NetDims& d, const float* op, const float* cn) {
  const bool fill = op && cn;
  std::vector<LayerMat> v;
  const float* w = op;
  for (int i = 0; i + 1 < d.op_nl; ++i) {
    LayerMat L{d.op_outs[i], d.op_in[i], true, false, {}, {}};
    if (fill) L.w.assign(w, w + (size_t)d.op_in[i] * d.op_outs[i]);
    v.push_back(std::move(L));
    if (w) w += (size_t)d.op_in[i] * d.op_outs[i];
  }
  const int lo = d.op_nl - 1;  // out_prd's output layer: [op_out][op_in[lo]]
  const int n0 = d.cn_outs[0], k0 = d.op_in[lo], m = d.op_out, kt = d.cn_in[0];
  LayerMat F{n0, k0, true, true, {}, {}};
  if (fill) {
    const float* wo = w;
    F.w.resize((size_t)n0 * k0);
    for (int r = 0; r < n0; ++r)
      for (int c = 0; c < k0; ++c) {
        double acc = 0.0;
        for (int j = 0; j < m; ++j) acc += (double)cn[(size_t)r * kt + j] * (double)wo[(size_t)j * k0 + c];
        F.w[(size_t)r * k0 + c] = (float)acc;
      }
    F.waux.resize((size_t)n0 * 16);
    for (int r = 0; r < n0; ++r)
      for (int c = 0; c < 16; ++c) F.waux[(size_t)r * 16 + c] = cn[(size_t)r * kt + m + c];
  }
  v.push_back(std::move(F));
  w = cn ? cn + (size_t)d.cn_in[0] * d.cn_outs[0] : nullptr;
  for (int i = 1; i + 1 < d.cn_nl; ++i) {
    LayerMat L{d.cn_outs[i], d.cn_in[i], true, false, {}, {}};
    if (fill) L.w.assign(w, w + (size_t)d.cn_in[i] * d.cn_outs[i]);
    v.push_back(std::move(L));
    if (w) w += (size_t)d.cn_in[i] * d.cn_outs[i];
  }
  return v;
}
const float* vlast_src(const NetDims& d, const float* cn) {
  if (!cn) return nullptr;
  const float* w = cn;
  for (int i = 0; i + 1 < d.cn_nl; ++i) w += (size_t)d.cn_in[i] * d.cn_outs[i];
  return w;
}

// Builds the blob for one precision.  eb = 2: BF16, every scale 1.  eb = 1: E4M3 with
// layer scales g[l] (B = W * g[l]), aux scales (the aux block stays BF16, times dscale of
// its layer) and V_last divided by the fin layer's accumulator scale.
TcPlan make_plan(const NetDims& d, const float* op, const float* cn, int eb, const std::vector<float>& g,
                 const std::vector<float>& dscale, std::vector<uint8_t>* blob) {
  TcPlan P;
  size_t off = 0;
  const bool fill = op && cn;
  const std::vector<LayerMat> src = layer_mats(d, op, cn);
  for (size_t li = 0; li < src.size(); ++li) {
    const LayerMat& ls = src[li];
    TcLayer L{};
    const int np = pad16(ls.n), kp = eb == 2 ? pad16(ls.k) : pad32(ls.k);
    L.b_off = (uint32_t)off;
    L.b_sbo = (uint32_t)(kp * eb * 8);
    L.k = kp;
    L.n = np;
    L.relu = ls.relu;
    L.scale = 1.f;
    if (fill) put_b(blob, off, ls.w.data(), ls.n, ls.k, 0, ls.k, np, kp, eb, eb == 2 ? 1.f : g[li]);
    off += (size_t)np * kp * eb;
    off = (off + 127) & ~size_t(127);
    if (ls.aux) {
      // aux block: columns [op_out, op_out + 16) of cmp_net's first layer, BF16
      L.aux = 1;
      L.aux_off = (uint32_t)off;
      if (fill) put_b(blob, off, ls.waux.data(), ls.n, 16, 0, 16, np, 16, 2, eb == 2 ? 1.f : dscale[li]);
      off += (size_t)np * 16 * 2;
      off = (off + 127) & ~size_t(127);
    }
    P.layers[P.n_layers++] = L;
  }
  P.layers[P.n_layers - 1].fin = 1;
  // V_last: the 3 x 64 output layer in FP32, [c][j]; it travels in the kernel parameters
  if (fill) {
    const float* w = vlast_src(d, cn);
    const int n_in = d.cn_in[d.cn_nl - 1];
    const float inv = eb == 2 ? 1.f : 1.f / dscale[P.n_layers - 1];
    for (int c = 0; c < 3; ++c)
      for (int j = 0; j < 64; ++j) P.vlast[c][j] = j < n_in ? w[(size_t)c * n_in + j] * inv : 0.f;
  }
  // BF16: V_last as the FP16 B tile of the output layer on the tensor core (N = 16, channel c in
  // row c; FP16 keeps 11 significant bits of ReLU(h) and V_last, where BF16 keeps 8)
  if (eb == 2) {
    const int n_in = d.cn_in[d.cn_nl - 1], kp = pad16(n_in);
    P.out_b_off = (uint32_t)off;
    P.out_sbo = (uint32_t)(kp * 2 * 8);
    P.out_k = kp;
    if (fill) put_b(blob, off, vlast_src(d, cn), 3, n_in, 0, n_in, 16, kp, 2, 1.f, true);
    off += (size_t)16 * kp * 2;
    off = (off + 127) & ~size_t(127);
  }
  if (blob) blob->resize(off, 0);
  P.blob_bytes = (uint32_t)off;
  return P;
}

TcPlan plan_bf16(const NetDims& d, const float* op, const float* cn, std::vector<uint8_t>* blob) {
  return make_plan(d, op, cn, 2, {}, {}, blob);
}

bool plan_supported(const NetDims& d, std::string* why) {
  auto no = [&](const char* m) { if (why) *why = m; return false; };
  if (d.aux_width != 16) return no("tensor-core path needs a 16-wide aux encoding");
  if (d.enc_dims() % 16 || d.enc_dims() > 32) return no("tensor-core path needs 16 or 32 hash features");
  if (d.op_out > 64) return no("tensor-core path needs out_prd outputs <= 64");
  if (d.cn_hidden < 1) return no("tensor-core path needs a hidden cmp_net layer");
  if (d.cn_neurons > 64 || pad16(d.cn_neurons) != 64) return no("tensor-core path needs 64-wide cmp_net layers");
  if (d.op_nl + d.cn_nl - 2 > kMaxTcLayers) return no("too many layers for the tensor-core path");
  for (int i = 0; i < d.op_nl; ++i) {
    const int n = pad16(d.op_outs[i]);
    if (n != 32 && n != 64) return no("out_prd widths must pad to 32 or 64");
    if (i > 0 && pad16(d.op_in[i]) > 64) return no("tensor-core path needs widths <= 64");
  }
  return true;
}

}  // namespace

bool relight_tc_supported(const NetDims& d, std::string* why) { return plan_supported(d, why); }

namespace {
// One warp waits, through the relight kernel's bounded wait, on a barrier that nothing ever
// arrives on; the wait gives up after limit_ns and records kDevWaitTimeout in err.
__global__ void wait_selftest_kernel(uint64_t limit_ns, uint32_t* err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  (void)__all_sync(0xffffffffu, wait_bounded(&bar, 0, err, limit_ns));
}
}  // namespace

void launch_wait_selftest(int timeout_ms, uint32_t* err, cudaStream_t st) {
  if (timeout_ms < 1 || timeout_ms > 2000) fail(NWPRT_INVALID_ARG, "wait self-test: timeout_ms must be in [1, 2000]");
  wait_selftest_kernel<<<1, 32, 0, st>>>((uint64_t)timeout_ms * 1000000ull, err);
  NWPRT_CUDA(cudaGetLastError());
}

bool relight_tc_fp8_supported(const NetDims& d, std::string* why) {
  if (!plan_supported(d, why)) return false;
  // every FP8 operand pads to K = 32 (zero columns); the widths above already do
  return true;
}

int tc_layer_count(const NetDims& d) { return d.op_nl + d.cn_nl - 2; }

size_t tc_weight_bytes(const NetDims& d) { return plan_bf16(d, nullptr, nullptr, nullptr).blob_bytes; }

TcPlan pack_tc_weights(const NetDims& d, const float* op, const float* cn, std::vector<uint16_t>* out) {
  std::vector<uint8_t> b;
  const TcPlan P = plan_bf16(d, op, cn, &b);
  out->assign(b.size() / 2, 0);
  std::memcpy(out->data(), b.data(), b.size());
  return P;
}

// Per-layer FP8 scales.  h[l] = kTarget / amax[l] maps layer l's input activations to
// E4M3 with kTarget (half the format's range) at the calibrated maximum, leaving headroom
// for values the calibration batch did not reach.  Layer l's weights carry
// g[l] = h[l+1] / h[l], so its FP32 accumulator already equals the next layer's scaled
// input and the epilogue converts it without a multiply; when that would push the weights
// outside E4M3's range, g[l] is clamped and the epilogue multiplies by the remainder.
// The fin layer's weights use the full range; V_last absorbs its accumulator scale.
TcPlan pack_tc_weights_fp8(const NetDims& d, const float* op, const float* cn, const float* amax,
                           std::vector<uint8_t>* out) {
  constexpr float kTarget = 240.f, kWmax = 240.f, kWmin = 1.f / 16.f;
  const std::vector<LayerMat> src = layer_mats(d, op, cn);
  const int n = (int)src.size();
  std::vector<float> h(n), g(n), epi(n, 1.f), dscale(n);
  for (int l = 0; l < n; ++l) h[l] = amax[l] > 0.f && std::isfinite(amax[l]) ? kTarget / amax[l] : 1.f;
  for (int l = 0; l < n; ++l) {
    float wmax = 0.f;
    for (float x : src[l].w) wmax = std::max(wmax, std::fabs(x));
    if (wmax == 0.f) wmax = 1.f;
    if (l + 1 < n) {
      g[l] = h[l + 1] / h[l];
      const float lo = kWmin / wmax, hi = kWmax / wmax;
      const float gc = std::min(std::max(g[l], lo), hi);
      epi[l] = g[l] / gc;  // 1 unless clamped
      g[l] = gc;
    } else {
      g[l] = kWmax / wmax;
    }
    dscale[l] = h[l] * g[l];  // accumulator = true pre-activation * dscale
  }
  out->clear();
  TcPlan P = make_plan(d, op, cn, 1, g, dscale, out);
  for (int l = 0; l < n; ++l) P.layers[l].scale = epi[l];
  P.cp_scale = h[0];
  return P;
}

// The compile-time layer sequence that matches plan P (kShapePlan if none does).
int shape_of(const TcPlan& P, const NetDims& d) {
  auto fixed = [&](int nl, int aux, int enc) {
    if (P.n_layers != nl || d.enc_dims() != enc) return false;
    for (int l = 0; l < nl; ++l) {
      const TcLayer& L = P.layers[l];
      if (L.n != 64 || !L.relu || (L.aux != 0) != (l == aux) || (L.fin != 0) != (l == nl - 1)) return false;
      // the fixed kernels issue K = the hash features (padded to one FP8 step) first, then 64
      if (l == 0 ? (L.k < enc || L.k > 32) : L.k != 64) return false;
    }
    return true;
  };
  if (fixed(ShapeOf<kShapeSix>::nl, ShapeOf<kShapeSix>::aux, 32)) return kShapeSix;
  if (fixed(ShapeOf<kShapeTwo>::nl, ShapeOf<kShapeTwo>::aux, 16)) return kShapeTwo;
  return kShapePlan;
}

size_t enc_smem_bytes(const NetDims& d) { return (size_t)kNWG * (d.enc_dims() <= 16 ? 8 : 16) * kTile * 4; }

// Rows of the weight blob's TMA view and their split into boxes of at most kWMaxBoxRows rows.
void weight_boxes(uint32_t blob_bytes, uint32_t* rows, uint32_t* boxes, uint32_t* box_rows) {
  *rows = (blob_bytes + kWRowBytes - 1) / kWRowBytes;
  *boxes = (*rows + kWMaxBoxRows - 1) / kWMaxBoxRows;
  *box_rows = (*rows + *boxes - 1) / *boxes;
}

size_t smem_for_blob(const NetDims& d, uint32_t blob_bytes) {
  uint32_t rows, boxes, box_rows;
  weight_boxes(blob_bytes, &rows, &boxes, &box_rows);
  return weight_region_bytes(boxes, box_rows) + (size_t)kNWG * kAuxBytes + enc_smem_bytes(d) + sizeof(TcBarriers);
}

size_t relight_tc_smem_bytes(const NetDims& d) { return smem_for_blob(d, (uint32_t)tc_weight_bytes(d)); }

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime.
EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  if (!fn) fail(NWPRT_CUDA_ERROR, "cuTensorMapEncodeTiled is unavailable from the driver");
  return fn;
}

// The weight blob (a device allocation of tc_blob_alloc_bytes(blob_bytes): whole rows) as a
// [rows][kWRowBytes / 4] uint32 tensor; no swizzle, so shared memory receives the blob's
// byte layout unchanged.
void encode_weight_map(CUtensorMap* map, const void* blob_dev, uint32_t blob_bytes, uint32_t* boxes,
                       uint32_t* box_rows) {
  uint32_t rows;
  weight_boxes(blob_bytes, &rows, boxes, box_rows);
  if ((reinterpret_cast<uintptr_t>(blob_dev) & 15) != 0) fail(NWPRT_INVALID_ARG, "weight blob not 16-byte aligned");
  const cuuint64_t dims[2] = {kWRowBytes / 4, rows};
  const cuuint64_t strides[1] = {kWRowBytes};
  const cuuint32_t box[2] = {kWRowBytes / 4, *box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_tiled()(map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<void*>(blob_dev), dims, strides,
                                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(NWPRT_CUDA_ERROR, "cuTensorMapEncodeTiled failed for the weight blob");
}

void launch_relight_tc(const NetDims& d, const HashLevels& hl, const float* hash, const void* blob_dev,
                       const TcPlan* plan, int mode, const TcJob* jobs, int n_jobs, int kahan, int clamp,
                       uint32_t* amax, uint32_t* err, int* tile_ctr, cudaStream_t st) {
  std::string why;
  if (!plan_supported(d, &why)) fail(NWPRT_UNSUPPORTED, why);
  if (n_jobs <= 0) return;
  if (mode == kTcFp8 && !plan) fail(NWPRT_NOT_READY, "FP8 relight without a calibrated plan");
  if (!plan) fail(NWPRT_NOT_READY, "tensor-core relight without packed weights");
  if (mode == kTcCalibrate && !amax) fail(NWPRT_INVALID_ARG, "calibration needs an amax buffer");
  if (!tile_ctr) fail(NWPRT_INVALID_ARG, "tensor-core relight needs a tile counter");
  if (n_jobs > kInlineJobs) {
    for (int j0 = 0; j0 < n_jobs; j0 += kInlineJobs)
      launch_relight_tc(d, hl, hash, blob_dev, plan, mode, jobs + j0, std::min(kInlineJobs, n_jobs - j0), kahan,
                        clamp, amax, err, tile_ctr, st);
    return;
  }
  const TcPlan& P = *plan;
  TcParams p{};
  p.hl = hl;
  p.hash = hash;
  p.wblob_bytes = P.blob_bytes;
  p.out_b_off = P.out_b_off;
  p.out_sbo = P.out_sbo;
  for (int l = 0; l < P.n_layers; ++l) {
    p.bdesc[l] = smem_desc(P.layers[l].b_off, 128u, P.layers[l].b_sbo);
    p.auxdesc[l] = P.layers[l].aux ? smem_desc(P.layers[l].aux_off, 128u, 256u) : 0ull;
  }
  p.outdesc = P.out_sbo ? smem_desc(P.out_b_off, 128u, P.out_sbo) : 0ull;
  encode_weight_map(&p.wmap, blob_dev, P.blob_bytes, &p.w_boxes, &p.w_box_rows);
  std::memcpy(p.vlast, P.vlast, sizeof(p.vlast));
  std::memcpy(p.layers, P.layers, sizeof(P.layers));
  p.n_layers = P.n_layers;
  p.enc_dims = d.enc_dims();
  p.n_jobs = n_jobs;
  p.kahan = kahan;
  p.clamp = clamp;
  p.cp_scale = P.cp_scale;
  p.amax = amax;
  p.err = err;
  // tile prefix over the jobs, longest tiles (largest K) first: the warpgroups take tiles in
  // this order, so the cheap ones fill the end of the launch
  int order[kInlineJobs];
  for (int i = 0; i < n_jobs; ++i) order[i] = i;
  std::stable_sort(order, order + n_jobs, [&](int a, int b) { return jobs[a].K > jobs[b].K; });
  long long tiles = 0;
  for (int i = 0; i < n_jobs; ++i) {
    p.jobs[i] = jobs[order[i]];
    p.jobs[i].tile_begin = tiles;
    tiles += (p.jobs[i].n_px - p.jobs[i].px_begin + kTile - 1) / kTile;
  }
  if (tiles == 0) return;
  p.total_tiles = tiles;
  int dev = 0, sms = 0, max_smem = 0;
  NWPRT_CUDA(cudaGetDevice(&dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  NWPRT_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const size_t smem = smem_for_blob(d, P.blob_bytes);
  if (smem > (size_t)max_smem) fail(NWPRT_UNSUPPORTED, "tensor-core relight: shared memory budget exceeded");
  const long long groups = (tiles + kNWG - 1) / kNWG;
  const int grid = (int)(groups < sms ? groups : sms);
  p.tile_ctr = tile_ctr;
  auto go = [&](auto kern) {
    NWPRT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    NWPRT_CUDA(cudaMemsetAsync(tile_ctr, 0, sizeof(int), st));
    kern<<<grid, kThreads, smem, st>>>(p);
  };
  const int shape = shape_of(P, d);
  if (mode == kTcBf16 && shape != kShapePlan && (P.out_k != 64 || P.out_sbo == 0))
    fail(NWPRT_INVALID_ARG, "tensor-core relight: the BF16 plan lacks its 64-wide FP16 output tile");
  auto pick = [&](auto mode_tag) {
    constexpr int M = decltype(mode_tag)::value;
    if (shape == kShapeSix) go(relight_tc_kernel<32, M, kShapeSix>);
    else if (shape == kShapeTwo) go(relight_tc_kernel<16, M, kShapeTwo>);
    else if (d.enc_dims() > 16) go(relight_tc_kernel<32, M, kShapePlan>);
    else go(relight_tc_kernel<16, M, kShapePlan>);
  };
  switch (mode) {
    case kTcBf16: pick(std::integral_constant<int, kTcBf16>{}); break;
    case kTcCalibrate: pick(std::integral_constant<int, kTcCalibrate>{}); break;
    case kTcFp8: pick(std::integral_constant<int, kTcFp8>{}); break;
    default: fail(NWPRT_INVALID_ARG, "unknown tensor-core mode");
  }
  NWPRT_CUDA(cudaGetLastError());
}

}  // namespace nwprt

// tcgen05 complex GEMM with split-TF32 products (sm_100a).
//
// C[z] (m x n, complex64) = A[z] (m x k) . B[z] (k x n) for every batch z.
// Operands arrive packed (k_pack_tiled / k_pack_planar) as K-major fp32 planes
// [re_hi | re_lo | im_hi | im_lo][z][rows][k] (rows padded to 128, k padded
// to 16): every value x is stored as hi = x rounded to the nearest TF32 value
// and lo = x - hi (exact in FP32) rounded likewise, so hi + lo carries x to
// about 2^-23 relative with no bias.  The split happens once, in the pack, so
// the GEMM's shared memory serves only TMA writes and tensor-core reads.  The
// 4M complex product is 12 TF32 MMAs per 8-wide K step into TMEM accumulators:
//   Cr += Ar*Br - Ai*Bi,  Ci += Ar*Bi + Ai*Br   for (hi,hi), (hi,lo), (lo,hi),
// the minus through the instruction's negate-A bit.  Accumulation is FP32: short
// chains in TMEM (32 or 64 of K), summed across chains in registers.
//
// Persistent: one CTA per SM walks a list of 128x128 output tiles (work items).
// Warp roles (512 threads, four warpgroups):
//   warp 0        TMA producer: 8 plane tiles per stage, 3-stage ring, across items
//   warp 1        TMEM allocation + single-thread MMA issue into two TMEM buffers
//   warps 4..11   drain: each finished buffer -> FP32 registers (round-to-nearest adds),
//                 then stage the finished tile, 32 rows at a time, in shared memory
//   warps 2..15   epilogue stores of every staged pass (staging -> HBM), while the
//                 MMA thread already fills TMEM for the next item
// Every mbarrier wait is bounded (about one second of global time); on expiry
// the kernel records a code in *err, drains what it issued and returns.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"

namespace ab2 {
namespace tc {

constexpr int BM = 128, BN = 128, BK = 16, STAGES = 3;
constexpr int PLANES = 4;                          // re_hi, re_lo, im_hi, im_lo
constexpr int PLANE_BYTES = BM * BK * 4;          // 8 KB: 128 rows x 64 B
constexpr int STAGE_BYTES = 2 * PLANES * PLANE_BYTES;  // A planes then B planes: 64 KB
// The epilogue stages one TMEM lane quadrant (32 output rows of complex64, rows padded by one element)
// in its own buffer, so the operand ring keeps feeding the next work item meanwhile.
constexpr int kStageRows = 32;
constexpr int STAGING_BYTES = kStageRows * BN * 8;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + STAGING_BYTES + 1024 /*barriers*/ + 1024 /*align*/;
static_assert(SMEM_BYTES <= 232448, "shared memory above the 227 KB a block may use");
// Two TMEM buffers of (Cr, Ci), 128 columns each: buffer b at columns [256 b, 256 b + 256).  The MMA
// thread fills one buffer with kChunkTiles K tiles (all 12 products per 8-wide K step) while the drain
// warps read the other and add it into FP32 registers with round-to-nearest.  The tensor core's FP32
// accumulation truncates once per MMA, so keeping each TMEM chain short (24 MMAs per accumulator at
// kChunkTiles = 2, the format default; TcArgs::chunk_tiles doubles it for forward programs) bounds that
// biased error; the long sum over K happens in the drain registers.
constexpr uint32_t TMEM_COLS = 512;
constexpr int kChunkTiles = 2;

// Operand formats of the kernel body.  FMT_TF32X3: each value as a TF32 pair (hi, lo) in 4-byte planes,
// 3 products per real product.  FMT_BF16X3: a BF16 pair, 3 products.  FMT_BF16X6: three BF16 pieces
// x = h + m + l (h = bf16(x), m = bf16(x - h), l = bf16(x - h - m); each difference is exact in FP32), which
// carry x to about 2^-26, and the 6 products hh, hm, mh, hl, lh, mm -- every dropped term (ml, lm, ll) is at
// most about 2^-24 of the product, so the result matches FP32 arithmetic; at the BF16 rate, 6 BF16 MMAs of
// K = 16 take as long as 3 TF32 MMAs of K = 8 over the same K.  Its 6 planes per operand fill a 96 KB stage,
// so the ring holds 2 stages, and one stage (32 of K) per TMEM chunk keeps 24 MMAs per accumulator chain.
enum : int { FMT_TF32X3 = 0, FMT_BF16X3 = 1, FMT_BF16X6 = 2 };
// The streaming epilogue (kStream): two staging buffers, so that the next 32-row pass is staged while the
// previous one is stored, with per-buffer mbarriers in place of block-wide barriers; its smem comes from a
// two-stage operand ring.  Meant for GEMMs whose epilogue outweighs their MMA work (short K).
constexpr int kStreamStages = 2;
constexpr int kStreamSmemBytes = kStreamStages * STAGE_BYTES + 2 * STAGING_BYTES + 1024 + 1024;
static_assert(kStreamSmemBytes <= 232448, "shared memory above the 227 KB a block may use");
// The deep-ring variant (kDeep, split-TF32): 8 of K per stage (32-byte operand rows, 32-byte swizzle), so the
// same 192 KB ring holds six stages and keeps five in flight instead of two -- more time to hide TMA latency
// on long-K steps.  A TMEM chunk spans four stages, the same 32 of K as otherwise.
constexpr int kDeepBK = 8, kDeepStages = 6;
constexpr int kDeepStageBytes = 2 * PLANES * BM * kDeepBK * 4;  // 32 KB
constexpr int kDeepSmemBytes = kDeepStages * kDeepStageBytes + STAGING_BYTES + 1024 + 1024;
static_assert(kDeepSmemBytes <= 232448, "shared memory above the 227 KB a block may use");
// The CTA-pair variant (kPair, split-TF32): two CTAs of a cluster share a 256 x 128 tile through
// tcgen05.mma.cta_group::2, each holding its 128 rows of A and half of B (64 output columns).  A stage is
// then 32 KB of A and 16 KB of B per CTA: a quarter less operand traffic per MMA and four stages in the ring.
constexpr int kPairStages = 4;
constexpr int kPairStageBytes = PLANES * PLANE_BYTES + PLANES * PLANE_BYTES / 2;  // 48 KB
constexpr int kPairSmemBytes = kPairStages * kPairStageBytes + STAGING_BYTES + 1024 + 1024;
static_assert(kPairSmemBytes <= 232448, "shared memory above the 227 KB a block may use");
// CTA pairs with the streaming epilogue: the pair's smaller stages leave room for both staging buffers beside
// a three-stage ring.
constexpr int kPairStreamStages = 3;
constexpr int kPairStreamSmemBytes = kPairStreamStages * kPairStageBytes + 2 * STAGING_BYTES + 1024 + 1024;
static_assert(kPairStreamSmemBytes <= 232448, "shared memory above the 227 KB a block may use");
template <int F>
struct Fmt {
  static constexpr bool kBF16 = F != FMT_TF32X3;
  static constexpr int kPieces = F == FMT_BF16X6 ? 3 : 2;
  static constexpr int kPlanes = 2 * kPieces;  // re pieces, then im pieces
  static constexpr int kStages = F == FMT_BF16X6 ? 2 : STAGES;
  static constexpr int kStageBytes = 2 * kPlanes * PLANE_BYTES;
  static constexpr int kChunkTiles = F == FMT_BF16X6 ? 1 : tc::kChunkTiles;
  static constexpr int kSmemBytes = kStages * kStageBytes + STAGING_BYTES + 1024 + 1024;
  static_assert(kSmemBytes <= 232448, "shared memory above the 227 KB a block may use");
};
// 16 warps in four warpgroups.  Warpgroup 0: TMA producer (warp 0), TMEM owner + MMA issuer (warp 1),
// store helpers (warps 2, 3).  Warpgroups 1 and 2: the 8 drain warps (4..11), which hold the FP32
// accumulators in registers.  Warpgroup 3: store helpers (12..15).  The block launches at 128 registers
// a thread; setmaxnreg then moves registers from warpgroups 0 and 3 (down to kLowRegs) to the drain
// warpgroups (up to kDrainRegs): 2 x 128 x kLowRegs + 2 x 128 x kDrainRegs equals 512 x 128 exactly.
constexpr int kThreads = 512, kLaunchRegs = 128, kLowRegs = 56, kDrainRegs = 200;
static_assert(2 * 128 * kLowRegs + 2 * 128 * kDrainRegs == kThreads * kLaunchRegs, "register split must use the launch total");
constexpr int kDrainWarps = 8, kDrainThreads = kDrainWarps * 32;
constexpr int kEpiWarps = 14, kEpiThreads = kEpiWarps * 32;  // warps 2..15 share the epilogue stores
constexpr int kHalfCols = BN / 2;             // columns one drain thread owns
constexpr unsigned long long kWaitNs = 1000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Nearest TF32 value of a finite FP32 bit pattern, ties away from zero: adding half of the dropped
// 13-bit field to the sign-magnitude pattern rounds the magnitude, a carry out of the mantissa moves
// to the next binade, and the mask clears the dropped field.  The result is exact as a TF32 operand,
// so the tensor core's own input conversion cannot change it.
__host__ __device__ __forceinline__ uint32_t tf32_round(uint32_t bits) { return (bits + 0x1000u) & 0xFFFFE000u; }
// x - hi, exact in FP32 (hi is within half a TF32 unit of x, so the subtraction is Sterbenz-exact).
__device__ __forceinline__ uint32_t tf32_residual(uint32_t x, uint32_t hi) {
  return __float_as_uint(__uint_as_float(x) - __uint_as_float(hi));
}
// Stores x as its TF32 pair: hi at dst[o], lo at dst[plane + o].
__device__ __forceinline__ void put_split(float* dst, ll plane, ll o, float x) {
  const uint32_t b = __float_as_uint(x), h = tf32_round(b);
  dst[o] = __uint_as_float(h);
  dst[plane + o] = __uint_as_float(tf32_round(tf32_residual(b, h)));
}
// Split-BF16 planes: hi = x rounded to BF16, lo = (x - hi) rounded to BF16.  x - hi is exact in FP32 (hi is
// within half a BF16 unit of x), so hi + lo carries x to about 2^-18 relative.
__device__ __forceinline__ void put_split(__nv_bfloat16* dst, ll plane, ll o, float x) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  dst[o] = h;
  dst[plane + o] = __float2bfloat16_rn(x - __bfloat162float(h));
}
// Split-BF16 with three pieces: the plane element of FMT_BF16X6 packs (2 bytes, like __nv_bfloat16).  put_split
// writes h, m, l to planes 0, 1, 2 (plane floats apart).
struct __align__(2) bf16p3 {
  __nv_bfloat16 v;
};
__device__ __forceinline__ void put_split(bf16p3* dst, ll plane, ll o, float x) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(h);  // exact: h is within half a BF16 unit of x
  const __nv_bfloat16 m = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(m);  // exact likewise
  dst[o].v = h;
  dst[plane + o].v = m;
  dst[2 * plane + o].v = __float2bfloat16_rn(r2);
}
// Pieces per value of a plane element type (the imaginary part's planes start this many planes later).
template <typename PT> __host__ __device__ constexpr int pieces_of() { return 2; }
template <> __host__ __device__ constexpr int pieces_of<bf16p3>() { return 3; }

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait; false (and *err = code) once about a second has passed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = now_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try(bar, parity)) return true;
    if ((i & 255) == 0) {
      if (now_ns() - t0 > kWaitNs) {
        atomicCAS(err, 0, code);
        return false;
      }
      __nanosleep(128);
    }
  }
}

__device__ __forceinline__ void tma_load_3d(const CUtensorMap* map, uint64_t* bar, void* dst, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(smem_u32(dst)), "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// K-major operand tile, 64-byte swizzle: rows of 64 B, 8-row groups 512 B apart.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFF) >> 4) | (1ull << 16) | ((uint64_t)(512 >> 4) << 32) | (1ull << 46) |
         (4ull << 61);
}
// K-major operand tile, 32-byte swizzle: rows of 32 B, 8-row groups 256 B apart (the deep-ring stages).
__device__ __forceinline__ uint64_t sw32_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFF) >> 4) | (1ull << 16) | ((uint64_t)(256 >> 4) << 32) | (1ull << 46) |
         (6ull << 61);
}
// kind::tf32, FP32 accumulate, K-major A and B, M = 128, N = 128.
__host__ __device__ constexpr uint32_t idesc_tf32(bool neg_a) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}
// kind::f16 with A and B both BF16 (one format code for both operands), FP32 accumulate, K-major, M = N = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(bool neg_a) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}
template <bool kBF16>
__host__ __device__ constexpr uint32_t idesc_for(bool neg_a) { return kBF16 ? idesc_bf16(neg_a) : idesc_tf32(neg_a); }

// One MMA: TF32 operands cover 8 of K in the 32 bytes of each operand row it reads, BF16 operands 16.
template <bool kBF16>
__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  if constexpr (kBF16) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc));
  } else {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc));
  }
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// ---- CTA pairs (cta_group::2): a cluster of two CTAs on one TPC computes a 256 x 128 tile; CTA rank r holds
// A rows 128 r .. + 127 and B rows (output columns) 64 r .. + 63 of the tile in its shared memory, and its own
// TMEM receives output rows 128 r .. + 127.  Rank 0 (the leader) issues the MMAs for both.
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// The shared::cluster address of the same shared variable in CTA `rank` of this cluster.
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
  return a;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// TMA load into this CTA's shared memory whose completion is counted on the leader's barrier (bar: a
// shared::cluster address).  No multicast.
__device__ __forceinline__ void tma_load_3d_pair(const CUtensorMap* map, uint32_t bar, void* dst, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(smem_u32(dst)), "l"(map), "r"(bar), "r"(x), "r"(y), "r"(z)
      : "memory");
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t bar) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_cluster(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on a local barrier that CTAs of the cluster arrive on (acquire at cluster scope).
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity, int* err, int code) {
  if (mbar_try_cluster(bar, parity)) return true;
  const unsigned long long t0 = now_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_cluster(bar, parity)) return true;
    if ((i & 255) == 0) {
      if (now_ns() - t0 > kWaitNs) {
        atomicCAS(err, 0, code);
        return false;
      }
      __nanosleep(128);
    }
  }
}
// kind::tf32 over the pair: M = 256 (128 rows in each CTA), N = 128 (64 B rows in each CTA).
__host__ __device__ constexpr uint32_t idesc_tf32_pair(bool neg_a) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)((2 * BM) >> 4) << 24);
}
__device__ __forceinline__ void umma_pair(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
// Arrive on the barrier at bar's offset in both CTAs of the pair once the leader's MMAs so far complete.
__device__ __forceinline__ void umma_commit_pair_both(uint64_t* bar) {
  const uint16_t mask = 3;
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;"
      ::"r"(smem_u32(bar)), "h"(mask)
      : "memory");
}
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

#define AB2_TMEM_LD32(taddr, r)                                                                                   \
  asm volatile(                                                                                                   \
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18," \
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"                                             \
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),          \
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),    \
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),  \
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])   \
      : "r"(taddr))

struct TcArgs {
  cf32* C;
  ll m, n;           // logical output rows / complex columns
  int k_tiles;       // padded K / BK
  int za, zb;        // plane batches of A and B (plane p of batch z sits at z + p * za / z + p * zb)
  int bt;            // GEMM batch per slice
  int a_var, b_var;  // operand differs per slice (else it is shared by all slices)
  int* err;
  // Split K: CTA blockIdx.z = split * zc + z accumulates k-tiles [split*kt_chunk, ...) in TMEM and
  // writes its FP32 partial to part[split][z][m][n]; k_splitk_reduce sums the splits in order.  The
  // tensor core's FP32 accumulation loses about one unit in the last place per addition, so its
  // error grows with the number of K steps one accumulator takes; bounding that number bounds it.
  int kt_chunk = 0;  // 0: one CTA takes all of K and writes C
  int zc = 0;        // output batches
  cf32* part = nullptr;
  // Persistent schedule: CTA b takes work items b, b + gridDim.x, ...; item it is output tile
  // it % tiles of batch-and-split it / tiles (split * zc + z).  Tiles enumerate the m_tiles x n_tiles
  // grid with the m-tile fastest when m_fast (A's tiles stay in L2 while B streams through once),
  // else the n-tile fastest.
  int n_items = 0, tiles = 1;
  int m_tiles = 1;
  int m_fast = 1;
  // Fused consumer pack: instead of C, write the output as the next GEMM's 4-plane operand pack.  The
  // packed offset of element (z = slice * bt + b, i, j) is slice * pk_slice + pk_b[b] + pk_i[i] + pk_j[j];
  // plane p sits p * pk_plane floats further.  Inside one output tile the packed offsets form chunks of
  // 32 consecutive floats with a common shape: chunk q starts at tile position (r0, c0) = pk_chunk[q].x
  // (r0 << 16 | c0) and packed offset pk_chunk[q].y past the tile's base, and its element l sits at
  // (r0, c0) + pk_lane[l] (dr << 16 | dc).  A warp stores one chunk per step: 128 contiguous bytes per plane.
  float* pk = nullptr;
  const ll* pk_i = nullptr;
  const ll* pk_j = nullptr;
  const ll* pk_b = nullptr;
  const int2* pk_chunk = nullptr;  // grouped by lane quadrant: quadrant q owns [pk_qbeg[q], pk_qbeg[q+1])
  const int* pk_lane = nullptr;
  int pk_qbeg[5] = {0, 0, 0, 0, 0};
  ll pk_plane = 0, pk_slice = 0;
  // Every packed offset a tile's chunks start at, the tile bases, the slice and plane strides and the pack's
  // address are multiples of 4 floats: a quarter-warp then stores one chunk with 16-byte stores (4 chunks
  // per warp step, 4 stores per element quadruple instead of 16).
  int pk_vec = 0;
  // K tiles per TMEM accumulation chunk (0: the format's default, 32 of K).  Longer chunks drain TMEM less
  // often and let the MMA run further ahead of an epilogue, at a longer truncated-FP32 chain per chunk.
  int chunk_tiles = 0;
};

#define AB2_TMEM_LD16(taddr, r)                                                                                   \
  asm volatile(                                                                                                   \
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"    \
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),          \
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])     \
      : "r"(taddr))

// Bounded wait for the drain warps: also gives up as soon as another role aborted.
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t* bar, uint32_t parity, int* err, int code,
                                                   volatile int* abort_flag) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = now_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try(bar, parity)) return true;
    if ((i & 63) == 0) {
      if (*abort_flag) return false;
      if (now_ns() - t0 > kWaitNs) {
        atomicCAS(err, 0, code);
        return false;
      }
      __nanosleep(64);
    }
  }
}

// Bounded wait until a shared-memory arrival counter reaches target (acquire); same exits as above.
__device__ __forceinline__ bool count_wait_or_abort(const volatile uint32_t* c, uint32_t target, int* err,
                                                    int code, volatile int* abort_flag) {
  const unsigned long long t0 = now_ns();
  for (uint32_t i = 1; *c < target; ++i) {
    if ((i & 63) == 0) {
      if (*abort_flag) return false;
      if (now_ns() - t0 > kWaitNs) {
        atomicCAS(err, 0, code);
        return false;
      }
      __nanosleep(64);
    }
  }
  __threadfence_block();
  return true;
}

// Staging layout of 32 output rows x 128 complex columns: row r, column c sits at r * BN + (c ^ g(r mod 16)),
// g(q) = (q & 3) << 2 | q >> 2.  A stager warp (lanes = 32 rows, one column) and a row reader (lanes = 32
// columns) both meet 16 distinct 8-byte bank pairs per half-warp, and so does a packed chunk spanning
// 4 rows x 4 columns.
__device__ __forceinline__ int stage_at(int r, int c) {
  const int q = r & 15;
  return r * BN + (c ^ (((q & 3) << 2) | (q >> 2)));
}

// Per-thread epilogue state.  For the fused pack: the lane's chunk pattern (dr, dc) and this warp's
// chunk entries, loaded once per kernel (the chunk table is the same for every tile): storer warp ew of nw
// takes chunks qbeg[q] + ew + nw * k of quadrant q, slot s = q * kq + k, held by lane s % 32 in e0
// (s < 32) or e1; entries past a quadrant's end hold r0 = 0x7FFF (out of every tile).  A quadrant has at
// most 32 x 128 / 32 = 128 chunks, so kq <= 10 for 14 storers and kq <= 16 for 8: 64 slots suffice.
struct EpiState {
  int dr = 0, dc = 0, kq = 0;
  int2 e0 = make_int2(0x7FFF0000, 0), e1 = make_int2(0x7FFF0000, 0);
};
__device__ __forceinline__ EpiState epi_setup(const TcArgs& args, int ew, int lane, int nw = kEpiWarps) {
  EpiState st;
  if (!args.pk) return st;
  const int lp = __ldg(args.pk_lane + lane);
  st.dr = lp >> 16;
  st.dc = lp & 0xFFFF;

  int most = 0;
#pragma unroll
  for (int q = 0; q < BM / kStageRows; ++q) most = max(most, args.pk_qbeg[q + 1] - args.pk_qbeg[q]);
  st.kq = (most + nw - 1) / nw;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int slot = lane + 32 * h, q = st.kq ? slot / st.kq : 0, k = st.kq ? slot % st.kq : 0;
    int2 e = make_int2(0x7FFF0000, 0);
    if (q < BM / kStageRows) {
      const int ci = args.pk_qbeg[q] + ew + nw * k;
      if (ci < args.pk_qbeg[q + 1]) e = __ldg(args.pk_chunk + ci);
    }
    if (h == 0) st.e0 = e; else st.e1 = e;
  }
  return st;
}
// Where one tile's output goes: the four packed planes (fused) or its C / split-K partial block.
struct EpiTile {
  float* p0;
  float* p1;
  float* p2;
  float* p3;
  cf32* cbase;
};
__device__ __forceinline__ EpiTile epi_tile(const TcArgs& args, int z, int split, ll row0, ll col0, int lane) {
  EpiTile t;
  if (args.pk) {
    t.p0 = args.pk + (ll)(z / args.bt) * args.pk_slice + __ldg(args.pk_b + z % args.bt) + __ldg(args.pk_i + row0) +
           __ldg(args.pk_j + col0) + (args.pk_vec ? (lane & 7) * 4 : lane);
    t.p1 = t.p0 + args.pk_plane;
    t.p2 = t.p1 + args.pk_plane;
    t.p3 = t.p2 + args.pk_plane;
    t.cbase = nullptr;
  } else {
    t.p0 = t.p1 = t.p2 = t.p3 = nullptr;
    t.cbase = (args.part ? args.part + (ll)split * args.zc * args.m * args.n : args.C) + (ll)z * args.m * args.n +
              row0 * args.n + col0;
  }
  return t;
}
__device__ __forceinline__ void put_pair(float* hi, float* lo, ll o, float x) {
  const uint32_t b = __float_as_uint(x), h = tf32_round(b);
  hi[o] = __uint_as_float(h);
  lo[o] = __uint_as_float(tf32_round(tf32_residual(b, h)));
}

// One pass of the epilogue store: output rows [r_lo, r_lo + 32) of the tile, staged in `stage`, written
// by storer thread et of nthreads (the 14 epilogue warps; 8 in the streaming epilogue), either as C rows or
// as packed 32-float chunks (the warp's chunks are in es, from epi_setup with the same storer count).
__device__ __forceinline__ void store_pass(const TcArgs& args, const EpiState& es, const EpiTile& t, const cf32* stage,
                                           int q, int rows, int cols, int et, int nthreads = kEpiThreads) {
  const int r_lo = q * kStageRows;
  if (r_lo >= rows) return;
  if (args.pk && args.pk_vec) {
    // Quarter-warp g = lane / 8 takes chunk k0 + g of this warp's list; its lane stores floats 4 (lane % 8) ..
    // + 3 of the chunk: the four elements are read from staging, split, and written as one float4 per plane.
    const int lane = threadIdx.x & 31, g = lane >> 3;
    // (dr << 16 | dc) of chunk elements 4 (lane % 8) .. + 3, read per pass (L1-resident) so that the drain
    // warps, which hold a tile of accumulators meanwhile, keep no extra registers across passes
    const int4 vq = __ldg(reinterpret_cast<const int4*>(args.pk_lane) + (lane & 7));
    const int vp[4] = {vq.x, vq.y, vq.z, vq.w};
    for (int k0 = 0; k0 < es.kq; k0 += 4) {
      const int kk = k0 + g, slot = q * es.kq + kk;
      const int x0 = __shfl_sync(0xffffffffu, es.e0.x, slot & 31), y0 = __shfl_sync(0xffffffffu, es.e0.y, slot & 31);
      const int x1 = __shfl_sync(0xffffffffu, es.e1.x, slot & 31), y1 = __shfl_sync(0xffffffffu, es.e1.y, slot & 31);
      int cx = slot < 32 ? x0 : x1;
      const int cy = slot < 32 ? y0 : y1;
      if (kk >= es.kq) cx = 0x7FFF0000;
      const int rb = cx >> 16, cb = cx & 0xFFFF;
      cf32 v[4];
      bool in[4], all = true, any = false;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = rb + (vp[i] >> 16), c = cb + (vp[i] & 0xFFFF);
        in[i] = r < rows && c < cols;
        all = all && in[i];
        any = any || in[i];
        v[i] = in[i] ? stage[stage_at(r - r_lo, c)] : cf32{0.f, 0.f};
      }
      if (all) {
#pragma unroll
        for (int part = 0; part < 2; ++part) {  // real parts to planes 0 / 1, then imaginary parts to 2 / 3
          float4 h, l;
          float* hp = &h.x;
          float* lp = &l.x;
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const uint32_t b = __float_as_uint(part ? v[i].im : v[i].re), th = tf32_round(b);
            hp[i] = __uint_as_float(th);
            lp[i] = __uint_as_float(tf32_round(tf32_residual(b, th)));
          }
          *reinterpret_cast<float4*>((part ? t.p2 : t.p0) + cy) = h;
          *reinterpret_cast<float4*>((part ? t.p3 : t.p1) + cy) = l;
        }
      } else if (any) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if (!in[i]) continue;
          put_pair(t.p0, t.p1, cy + i, v[i].re);
          put_pair(t.p2, t.p3, cy + i, v[i].im);
        }
      }
    }
  } else if (args.pk) {
    constexpr int U = 4;
    for (int k0 = 0; k0 < es.kq; k0 += U) {
      int2 ch[U];
      cf32 v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int slot = q * es.kq + k0 + u;
        const int2 e = slot < 32 ? es.e0 : es.e1;
        ch[u].x = __shfl_sync(0xffffffffu, e.x, slot & 31);
        ch[u].y = __shfl_sync(0xffffffffu, e.y, slot & 31);
        if (k0 + u >= es.kq) ch[u].x = 0x7FFF0000;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int r = (ch[u].x >> 16) + es.dr, c = (ch[u].x & 0xFFFF) + es.dc;
        v[u] = (r < rows && c < cols) ? stage[stage_at(r - r_lo, c)] : cf32{0.f, 0.f};
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int r = (ch[u].x >> 16) + es.dr, c = (ch[u].x & 0xFFFF) + es.dc;
        if (r < rows && c < cols) {
          put_pair(t.p0, t.p1, ch[u].y, v[u].re);
          put_pair(t.p2, t.p3, ch[u].y, v[u].im);
        }
      }
    }
  } else {
    const int nr = rows - r_lo < kStageRows ? rows - r_lo : kStageRows;
    cf32* cbase = t.cbase + (ll)r_lo * args.n;
    constexpr int U = 4;
    for (int e0 = et; e0 < nr * BN; e0 += U * nthreads) {
      cf32 v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = e0 + u * nthreads, r = e / BN, c = e % BN;
        v[u] = (e < nr * BN && c < cols) ? stage[stage_at(r, c)] : cf32{0.f, 0.f};
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = e0 + u * nthreads, r = e / BN, c = e % BN;
        if (e < nr * BN && c < cols) cbase[(ll)r * args.n + c] = v[u];
      }
    }
  }
}

// The GEMM body for either operand format: split-TF32 (4-byte planes, 16 of K per 64-byte operand row) or
// split-BF16 (2-byte planes, 32 of K per row).  Shared-memory layout, swizzle, TMEM and epilogue are the same.
template <int F, bool kStream = false, bool kDeep = false, bool kPair = false>
__device__ __forceinline__ void tc_cgemm_body(const CUtensorMap& tmA, const CUtensorMap& tmB, const TcArgs& args) {
  using FM = Fmt<F>;
  static_assert(!kStream || F == FMT_TF32X3, "the streaming epilogue is built for split-TF32 operands");
  static_assert(!kDeep || (F == FMT_TF32X3 && !kStream), "the deep ring is built for split-TF32 operands");
  static_assert(!kPair || (F == FMT_TF32X3 && !kDeep), "the CTA pair is built for split-TF32 operands");
  constexpr bool kBF16 = FM::kBF16;
  constexpr int STAGES = kPair ? (kStream ? kPairStreamStages : kPairStages)
                               : kDeep ? kDeepStages : kStream ? kStreamStages : FM::kStages;
  constexpr int STAGE_BYTES = kPair ? kPairStageBytes : kDeep ? kDeepStageBytes : FM::kStageBytes;
  constexpr int PLANES = FM::kPlanes;
  constexpr int PLANE_BYTES = kDeep ? BM * kDeepBK * 4 : tc::PLANE_BYTES;
  constexpr int B_PLANE_BYTES = kPair ? PLANE_BYTES / 2 : PLANE_BYTES;  // B rows per CTA: 64 in a pair
  constexpr int kStagingBufs = kStream ? 2 : 1;
  const int kChunkTiles = args.chunk_tiles > 0 ? args.chunk_tiles : (kDeep ? 4 : FM::kChunkTiles);
  constexpr int KT_ELEMS = kDeep ? kDeepBK : kBF16 ? 2 * BK : BK;  // K per operand row of a stage
  constexpr int KSTEPS = kDeep ? 1 : BK / 8;                        // MMA K steps per stage (32 bytes each)
  auto sdesc = [](uint32_t a) { return kDeep ? sw32_desc(a) : sw64_desc(a); };
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* ring = smem;                                  // STAGES x {A planes, B planes}
  cf32* stage = reinterpret_cast<cf32*>(smem + STAGES * STAGE_BYTES);  // kStageRows x kTileStride
  uint64_t* bars = (uint64_t*)(smem + STAGES * STAGE_BYTES + kStagingBufs * STAGING_BYTES);
  uint64_t* full = bars;                     // TMA landed                  (count 1 + tx)
  uint64_t* empty = bars + STAGES;           // MMAs done reading a stage   (commit)
  uint64_t* accfull = bars + 2 * STAGES;     // [2] a TMEM buffer's chunk is complete (commit)
  uint64_t* accempty = accfull + 2;          // [2] the drain warps have read it      (count kDrainThreads)
  uint64_t* drain = accempty + 2;            // abort drain                 (commit)
  uint64_t* sfull = drain + 1;               // [2] kStream: a staging buffer holds its pass (the 2 stager warps)
  // [2] kStream: storer warps done with a staging buffer, counted over all its uses (8 per use).  A counter,
  // not an mbarrier: a buffer's consecutive uses are staged by different quadrants, which may drift two uses
  // apart, and a phase-parity wait cannot tell those apart.
  volatile uint32_t* sdone = (volatile uint32_t*)(sfull + 2);
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(sfull + 4);
  volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int n_tiles = (int)((args.n + BN - 1) / BN);
  // Items are taken per CTA, or per pair (items it0, it0 + it_step, ...); a pair's m-tiles are 256 rows and
  // CTA rank r writes rows 128 r .. + 127 of each.
  const int rank = kPair ? (int)cluster_rank() : 0;
  const int it0 = kPair ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
  const int it_step = kPair ? (int)(gridDim.x >> 1) : (int)gridDim.x;
  auto row0_of = [&](int tile_m) -> ll { return kPair ? (ll)tile_m * 2 * BM + rank * BM : (ll)tile_m * BM; };
  // Work item it: output tile it % tiles (raster as in TcArgs) of batch-and-split it / tiles.
  struct Item { int tile_m, tile_n, z, split, kt0, KT, zA, zB; };
  auto item_of = [&](int it) {
    Item w;
    const int x = it % args.tiles, zz = it / args.tiles;
    w.tile_m = args.m_fast ? x % args.m_tiles : x / n_tiles;
    w.tile_n = args.m_fast ? x / args.m_tiles : x % n_tiles;
    w.split = args.kt_chunk ? zz / args.zc : 0;
    w.z = args.kt_chunk ? zz % args.zc : zz;
    w.kt0 = args.kt_chunk ? w.split * args.kt_chunk : 0;
    const int kt1 = args.kt_chunk ? min(args.k_tiles, w.kt0 + args.kt_chunk) : args.k_tiles;
    w.KT = kt1 - w.kt0;                         // k-tile of iteration t is kt0 + t
    const int b_idx = w.z % args.bt;
    w.zA = args.a_var ? w.z : b_idx;
    w.zB = args.b_var ? w.z : b_idx;
    return w;
  };

  if (threadIdx.x == 0) {
    for (int i = 0; i < STAGES; ++i) { mbar_init(&full[i], 1); mbar_init(&empty[i], 1); }
    // accempty: every drain thread arrives, or in a pair one arrival per drain warp of both CTAs (the leader's)
    for (int i = 0; i < 2; ++i) { mbar_init(&accfull[i], 1); mbar_init(&accempty[i], kPair ? 2 * kDrainWarps : kDrainThreads); }
    mbar_init(drain, 1);
    for (int i = 0; i < 2; ++i) { mbar_init(&sfull[i], 2); sdone[i] = 0; }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    // a pair allocates collectively, one warp in each CTA: the same columns in both CTAs' TMEM
    if constexpr (kPair) {
      asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;"
                   ::"r"(smem_u32((const void*)tmem_slot)), "r"(TMEM_COLS));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    } else {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                   ::"r"(smem_u32((const void*)tmem_slot)), "r"(TMEM_COLS));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if constexpr (kPair) cluster_sync_all();  // the peer's barriers are initialised before any copy signals them
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // kStream: global pass gp (4 per item) uses staging buffer gp & 1 for the (gp >> 1)-th time, u.  A pass is
  // stored once sfull[b] completed use u, and its buffer is staged again once sdone[b] counts the stores of
  // uses 0..u-1; every wait is bounded and gives up at once after an abort.  A storer waits on sfull[b] only
  // after it stored use u-1 and before it stores use u, and use u+1 is staged only after that store, so the
  // barrier is never two phases away from its waiter and the parity wait is exact.
  // Storers of a streamed pass: the six helpers (ranks 0..5) and the two drain warps that staged it (ranks 6, 7).
  constexpr int kStreamStorers = 8;
  // epi_setup holds a storer's chunks of all four passes in the 64 slots of a warp's two int2 registers.
  static_assert(BM / kStageRows * ((kStageRows * BN / 32 + kStreamStorers - 1) / kStreamStorers) <= 64,
                "a streamed pass's packed chunks do not fit a storer warp's slots");
  auto stream_store = [&](const EpiState& es, const EpiTile& t, int gp, int rows, int cols, bool& dead, int srank) {
    const int b = gp & 1, u = gp >> 1;
    if (!dead && !mbar_wait_or_abort(&sfull[b], (uint32_t)(u & 1), args.err, 3, abort_flag)) {
      dead = true;
      *abort_flag = 1;
    }
    if (!dead)
      store_pass(args, es, t, stage + b * kStageRows * BN, gp & 3, rows, cols, srank * 32 + (threadIdx.x & 31),
                 kStreamStorers * 32);
    __syncwarp();
    if (!dead && (threadIdx.x & 31) == 0) {
      __threadfence_block();  // this warp's reads of the buffer come before the count
      atomicAdd((uint32_t*)&sdone[b], 1u);
    }
  };
  // Store helpers (warps 2, 3, 12..15): they follow the drain warps' items and barriers and share the
  // stores of every staged pass.
  auto helpers = [&]() {
    if constexpr (kStream) {
      const int srank = warp < 4 ? warp - 2 : warp - 10;  // warps 2, 3, 12..15 -> storer ranks 0..5
      const EpiState es = epi_setup(args, srank, lane, kStreamStorers);
      bool dead = false;
      int gp = 0;
      for (int it = it0; it < args.n_items; it += it_step, gp += BM / kStageRows) {
        const Item w = item_of(it);
        const ll row0 = row0_of(w.tile_m), col0 = (ll)w.tile_n * BN;
        const int rows = (int)(args.m - row0 < BM ? args.m - row0 : BM);
        const int cols = (int)(args.n - col0 < BN ? args.n - col0 : BN);
        const EpiTile t = epi_tile(args, w.z, w.split, row0 < args.m ? row0 : 0, col0, lane);  // rows <= 0: unused
        for (int q = 0; q < BM / kStageRows; ++q) {
          if (*abort_flag) dead = true;
          stream_store(es, t, gp + q, rows, cols, dead, srank);
        }
      }
      return;
    }
    const EpiState es = epi_setup(args, warp - 2, lane);
    bool dead = false;
    for (int it = it0; it < args.n_items; it += it_step) {
      const Item w = item_of(it);
      const ll row0 = row0_of(w.tile_m), col0 = (ll)w.tile_n * BN;
      const int rows = (int)(args.m - row0 < BM ? args.m - row0 : BM);
      const int cols = (int)(args.n - col0 < BN ? args.n - col0 : BN);
      const EpiTile t = epi_tile(args, w.z, w.split, row0 < args.m ? row0 : 0, col0, lane);  // rows <= 0: unused
#pragma unroll 1
      for (int q = 0; q < BM / kStageRows; ++q) {
        asm volatile("bar.sync 1, %0;" ::"n"(kEpiThreads) : "memory");
        asm volatile("bar.sync 1, %0;" ::"n"(kEpiThreads) : "memory");
        if (*abort_flag) dead = true;
        if (!dead) store_pass(args, es, t, stage, q, rows, cols, threadIdx.x - 64);
      }
    }
  };
  if (warp < 4) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kLowRegs));
    if (warp == 0) {
      // ------------------------------------------------------------ TMA producer
      // g counts k-tiles over all of this CTA's items: stage g % STAGES, phase (g / STAGES) & 1.
      if (lane == 0) {
        int g = 0, issued = 0;
        bool stop = false;
        for (int it = it0; it < args.n_items && !stop; it += it_step) {
          const Item w = item_of(it);
          for (int t = 0; t < w.KT; ++t, ++g) {
            const int s = g % STAGES;
            if (g >= STAGES && !mbar_wait(&empty[s], ((g / STAGES) - 1) & 1, args.err, 1)) {
              *abort_flag = 1;
              stop = true;
              break;
            }
            if (*abort_flag) { stop = true; break; }
            unsigned char* dst = ring + s * STAGE_BYTES;
            const int k0 = (w.kt0 + t) * KT_ELEMS;
            if constexpr (kPair) {
              // Both CTAs' copies count on the leader's full[s], which expects the pair's bytes.  Rows past the
              // operand (the upper half of a last 256-row tile) arrive as zeros and count all the same.
              const uint32_t fb = cluster_addr(&full[s], 0);
              if (rank == 0) mbar_expect_tx(&full[s], 2 * STAGE_BYTES);
              const int ya = (int)row0_of(w.tile_m), yb = w.tile_n * BN + rank * (BN / 2);
  #pragma unroll
              for (int p = 0; p < PLANES; ++p) {
                tma_load_3d_pair(&tmA, fb, dst + p * PLANE_BYTES, k0, ya, w.zA + p * args.za);
                tma_load_3d_pair(&tmB, fb, dst + PLANES * PLANE_BYTES + p * B_PLANE_BYTES, k0, yb, w.zB + p * args.zb);
              }
            } else {
              mbar_expect_tx(&full[s], STAGE_BYTES);
  #pragma unroll
              for (int p = 0; p < PLANES; ++p) {
                tma_load_3d(&tmA, &full[s], dst + p * PLANE_BYTES, k0, w.tile_m * BM, w.zA + p * args.za);
                tma_load_3d(&tmB, &full[s], dst + (PLANES + p) * PLANE_BYTES, k0, w.tile_n * BN, w.zB + p * args.zb);
              }
            }
            issued = g + 1;
          }
        }
        if (*abort_flag && rank == 0) {  // let issued copies land before the CTA retires (a pair's count on the leader)
          for (int t = (issued > STAGES ? issued - STAGES : 0); t < issued; ++t)
            mbar_wait(&full[t % STAGES], (t / STAGES) & 1, args.err, 7);
        }
      }
    } else if (warp == 1) {
      // ------------------------------------------------------------ MMA issuer
      // gc counts chunks over all items: TMEM buffer gc & 1.  The issuer runs up to two chunks ahead
      // of the drain warps, so the next item's first chunks overlap the previous item's epilogue.
      if (lane == 0 && rank == 0) {  // in a pair, the leader issues for both CTAs
        const uint32_t id_pos = kPair ? idesc_tf32_pair(false) : idesc_for<kBF16>(false);
        const uint32_t id_neg = kPair ? idesc_tf32_pair(true) : idesc_for<kBF16>(true);
        auto mma = [&](uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
          if constexpr (kPair) umma_pair(d, a, b, id, acc);
          else umma<kBF16>(d, a, b, id, acc);
        };
        auto commit = [&](uint64_t* bar) {  // a pair's stage and accumulator barriers are signalled in both CTAs
          if constexpr (kPair) umma_commit_pair_both(bar);
          else umma_commit(bar);
        };
        int g = 0, gc = 0;
        bool stop = false;
        for (int it = it0; it < args.n_items && !stop; it += it_step) {
          const Item w = item_of(it);
          const int n_chunks = (w.KT + kChunkTiles - 1) / kChunkTiles;
          for (int c = 0; c < n_chunks; ++c, ++gc) {
            if (*abort_flag) { stop = true; break; }
            const int b = gc & 1;
            if (gc >= 2 && !(kPair ? mbar_wait_cluster(&accempty[b], ((gc >> 1) - 1) & 1, args.err, 6)
                                   : mbar_wait(&accempty[b], ((gc >> 1) - 1) & 1, args.err, 6))) {
              *abort_flag = 1;
              stop = true;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t cr = tmem + b * 2 * BN, ci = cr + BN;
            const int t_end = min(w.KT, (c + 1) * kChunkTiles);
            bool first = true;
            for (int t = c * kChunkTiles; t < t_end; ++t, ++g) {
              const int s = g % STAGES;
              if (!mbar_wait(&full[s], (g / STAGES) & 1, args.err, 2)) {
                *abort_flag = 1;
                stop = true;
                break;
              }
              asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
              const uint32_t a0 = smem_u32(ring + s * STAGE_BYTES), b0 = a0 + PLANES * PLANE_BYTES;
              if constexpr (F == FMT_BF16X6) {
                // planes re_h, re_m, re_l, im_h, im_m, im_l; products (h,h), (h,m), (m,h), (h,l), (l,h), (m,m)
                constexpr int px[6] = {0, 0, 1, 0, 2, 1}, py[6] = {0, 1, 0, 2, 0, 1};
  #pragma unroll
                for (int kk = 0; kk < BK / 8; ++kk) {
                  const uint32_t o = kk * 32;
  #pragma unroll
                  for (int q = 0; q < 6; ++q) {
                    const uint32_t Ar = a0 + px[q] * PLANE_BYTES + o, Ai = Ar + 3 * PLANE_BYTES;
                    const uint32_t Br = b0 + py[q] * PLANE_BYTES + o, Bi = Br + 3 * PLANE_BYTES;
                    const uint32_t acc = (first && q == 0) ? 0u : 1u;
                    umma<true>(cr, sw64_desc(Ar), sw64_desc(Br), id_pos, acc);
                    umma<true>(ci, sw64_desc(Ar), sw64_desc(Bi), id_pos, acc);
                    umma<true>(cr, sw64_desc(Ai), sw64_desc(Bi), id_neg, 1);
                    umma<true>(ci, sw64_desc(Ai), sw64_desc(Br), id_pos, 1);
                  }
                  first = false;
                }
                umma_commit(&empty[s]);
                continue;
              }
              const uint32_t hAr = a0, lAr = a0 + PLANE_BYTES, hAi = a0 + 2 * PLANE_BYTES, lAi = a0 + 3 * PLANE_BYTES;
              const uint32_t hBr = b0, lBr = b0 + B_PLANE_BYTES, hBi = b0 + 2 * B_PLANE_BYTES, lBi = b0 + 3 * B_PLANE_BYTES;
  #pragma unroll
              for (int kk = 0; kk < KSTEPS; ++kk) {
                const uint32_t o = kk * 32;  // 8 tf32 or 16 bf16 = 32 bytes along the swizzled row
                const uint32_t acc = first ? 0u : 1u;
                // leading terms (hi,hi), then the corrections (lo,hi) and (hi,lo), all into this chunk's buffer
                mma(cr, sdesc(hAr + o), sdesc(hBr + o), id_pos, acc);
                mma(ci, sdesc(hAr + o), sdesc(hBi + o), id_pos, acc);
                mma(cr, sdesc(hAi + o), sdesc(hBi + o), id_neg, 1);
                mma(ci, sdesc(hAi + o), sdesc(hBr + o), id_pos, 1);
                mma(cr, sdesc(lAr + o), sdesc(hBr + o), id_pos, 1);
                mma(ci, sdesc(lAr + o), sdesc(hBi + o), id_pos, 1);
                mma(cr, sdesc(lAi + o), sdesc(hBi + o), id_neg, 1);
                mma(ci, sdesc(lAi + o), sdesc(hBr + o), id_pos, 1);
                mma(cr, sdesc(hAr + o), sdesc(lBr + o), id_pos, 1);
                mma(ci, sdesc(hAr + o), sdesc(lBi + o), id_pos, 1);
                mma(cr, sdesc(hAi + o), sdesc(lBi + o), id_neg, 1);
                mma(ci, sdesc(hAi + o), sdesc(lBr + o), id_pos, 1);
                first = false;
              }
              commit(&empty[s]);
            }
            if (stop) break;
            commit(&accfull[b]);
          }
        }
        if (*abort_flag) {
          if constexpr (kPair) umma_commit_pair(drain);
          else umma_commit(drain);
          mbar_wait(drain, 0, args.err, 8);
        }
      }
    } else {
      helpers();
    }
  } else if (warp < 12) {
    // ------------------------------------------------------------ drain + epilogue (8 warps)
    // Warp w reads TMEM lanes 32 * (w % 4) .. +31 (its output rows) and one half of the 128 columns.
    // Every epilogue warp walks the same items and meets the same named barriers; after an abort (dead)
    // it skips the waits and the stores but still meets the barriers.
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kDrainRegs));
    const int quad = warp % 4, half = (warp - 4) / 4;
    const EpiState es = epi_setup(args, warp - 2, lane);
    [[maybe_unused]] const EpiState es_stream = kStream ? epi_setup(args, 6 + half, lane, 8) : EpiState{};
    int gc = 0, gpass = 0;
    bool dead = false;
    for (int it = it0; it < args.n_items; it += it_step) {
      const Item w = item_of(it);
      const int n_chunks = (w.KT + kChunkTiles - 1) / kChunkTiles;
      const ll row0 = row0_of(w.tile_m), col0 = (ll)w.tile_n * BN;
      const EpiTile t = epi_tile(args, w.z, w.split, row0 < args.m ? row0 : 0, col0, lane);  // overlaps the drain
      float acc_re[kHalfCols], acc_im[kHalfCols];
#pragma unroll
      for (int j = 0; j < kHalfCols; ++j) acc_re[j] = acc_im[j] = 0.f;
      for (int c = 0; c < n_chunks; ++c, ++gc) {
        if (dead) continue;
        const int b = gc & 1;
        if (!mbar_wait_or_abort(&accfull[b], (gc >> 1) & 1, args.err, 5, abort_flag)) {
          dead = true;
          *abort_flag = 1;
          continue;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t ta = tmem + ((uint32_t)(quad * 32) << 16) + b * 2 * BN + half * kHalfCols;
#pragma unroll
        for (int c0 = 0; c0 < kHalfCols; c0 += 16) {
          uint32_t vr[16], vi[16];
          AB2_TMEM_LD16(ta + c0, vr);
          AB2_TMEM_LD16(ta + BN + c0, vi);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            acc_re[c0 + j] += __uint_as_float(vr[j]);
            acc_im[c0 + j] += __uint_as_float(vi[j]);
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        if constexpr (kPair) {  // one arrival per warp of either CTA, on the leader's barrier
          __syncwarp();
          if (lane == 0) mbar_arrive_remote(cluster_addr(&accempty[b], 0));
        } else {
          mbar_arrive(&accempty[b]);
        }
      }
      if (*abort_flag) dead = true;
      // Epilogue, one lane quadrant (32 output rows) at a time: its two drain warps stage their rows,
      // then all 14 epilogue warps store them.
      const int rows = (int)(args.m - row0 < BM ? args.m - row0 : BM);
      const int cols = (int)(args.n - col0 < BN ? args.n - col0 : BN);
      if constexpr (kStream) {
        // Pass q is staged by quadrant q's two drain warps into buffer gp & 1 once the pass that used it before
        // is stored, then stored by those two warps and the six helpers.  A drain warp's part of the epilogue
        // ends with its own quadrant's pass, so it goes on to drain the next item while the helpers still store
        // the later passes of this one.
        auto stage_pass = [&](int g) {
          const int b = g & 1, u = g >> 1;
          if (!dead && u > 0 &&
              !count_wait_or_abort(&sdone[b], (uint32_t)(kStreamStorers * u), args.err, 4, abort_flag)) {
            dead = true;
            *abort_flag = 1;
          }
          if (!dead) {
            cf32* sb = stage + b * kStageRows * BN;
#pragma unroll
            for (int j = 0; j < kHalfCols; ++j) sb[stage_at(lane, half * kHalfCols + j)] = cf32{acc_re[j], acc_im[j]};
          }
          __syncwarp();
          if (!dead && lane == 0) mbar_arrive(&sfull[b]);
        };
        if (*abort_flag) dead = true;
        stage_pass(gpass + quad);
        stream_store(es_stream, t, gpass + quad, rows, cols, dead, 6 + half);
        gpass += BM / kStageRows;
      } else {
#pragma unroll 1
        for (int q = 0; q < BM / kStageRows; ++q) {
          asm volatile("bar.sync 1, %0;" ::"n"(kEpiThreads) : "memory");  // the previous rows are out
          if (quad == q && !dead) {
#pragma unroll
            for (int j = 0; j < kHalfCols; ++j) stage[stage_at(lane, half * kHalfCols + j)] = cf32{acc_re[j], acc_im[j]};
          }
          asm volatile("bar.sync 1, %0;" ::"n"(kEpiThreads) : "memory");
          if (!dead) store_pass(args, es, t, stage, q, rows, cols, threadIdx.x - 64);
        }
      }
    }
  } else {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kLowRegs));
    helpers();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  // A pair retires together: the leader's MMAs read the peer's shared memory and write its TMEM, and the
  // peer's warps arrive on the leader's barriers.
  if constexpr (kPair) cluster_sync_all();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if constexpr (kPair)
      asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    else
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

static __global__ void __launch_bounds__(kThreads, 1) k_tc_cgemm_tf32x3(const __grid_constant__ CUtensorMap tmA,
                                                                const __grid_constant__ CUtensorMap tmB,
                                                                TcArgs args) {
  tc_cgemm_body<FMT_TF32X3>(tmA, tmB, args);
}
// Split-TF32 with the streaming epilogue (two-stage operand ring, double-buffered staging).
static __global__ void __launch_bounds__(kThreads, 1) k_tc_cgemm_tf32x3_stream(const __grid_constant__ CUtensorMap tmA,
                                                                       const __grid_constant__ CUtensorMap tmB,
                                                                       TcArgs args) {
  tc_cgemm_body<FMT_TF32X3, true>(tmA, tmB, args);
}
// Split-TF32 on CTA pairs (clusters of 2, cta_group::2 MMAs on 256 x 128 tiles, four 48 KB stages).
static __global__ void __launch_bounds__(kThreads, 1) k_tc_cgemm_tf32x3_pair(const __grid_constant__ CUtensorMap tmA,
                                                                     const __grid_constant__ CUtensorMap tmB,
                                                                     TcArgs args) {
  tc_cgemm_body<FMT_TF32X3, false, false, true>(tmA, tmB, args);
}
// Split-TF32 on CTA pairs with the streaming epilogue (three 48 KB stages, double-buffered staging).
static __global__ void __launch_bounds__(kThreads, 1) k_tc_cgemm_tf32x3_pair_stream(
    const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, TcArgs args) {
  tc_cgemm_body<FMT_TF32X3, true, false, true>(tmA, tmB, args);
}
// Split-TF32 with the deep ring (six 32 KB stages of 8 of K, 32-byte swizzle).
static __global__ void __launch_bounds__(kThreads, 1) k_tc_cgemm_tf32x3_deep(const __grid_constant__ CUtensorMap tmA,
                                                                     const __grid_constant__ CUtensorMap tmB,
                                                                     TcArgs args) {
  tc_cgemm_body<FMT_TF32X3, false, true>(tmA, tmB, args);
}
// Split-BF16: operands packed as BF16 hi/lo planes, 3 BF16 products per real product (kind::f16).
static __global__ void __launch_bounds__(kThreads, 1) k_tc_cgemm_bf16x3(const __grid_constant__ CUtensorMap tmA,
                                                                const __grid_constant__ CUtensorMap tmB,
                                                                TcArgs args) {
  tc_cgemm_body<FMT_BF16X3>(tmA, tmB, args);
}
// Three-piece split-BF16: 6 BF16 products per real product (kind::f16), FP32-level accuracy.
static __global__ void __launch_bounds__(kThreads, 1) k_tc_cgemm_bf16x6(const __grid_constant__ CUtensorMap tmA,
                                                                const __grid_constant__ CUtensorMap tmB,
                                                                TcArgs args) {
  tc_cgemm_body<FMT_BF16X6>(tmA, tmB, args);
}

// Leg-aware pack: the same gather as k_pack_planar, for operands whose legs are scattered (as in
// networks of dimension-2 legs).  The host picks tile legs -- those innermost in the source plus those
// innermost in the packed destination, at most kPackTile elements -- and numbers the tile's elements
// by destination address.  rd_rank[i] / rd_off[i] give the element with the i-th smallest source
// offset (its rank and its source offset), wr_off[r] the destination offset of rank r, so the read
// and the write of a tile both walk memory in address order.  Remaining legs are enumerated by
// src_base / dst_base.  Each thread keeps its share of the tables in registers; the tile is held as
// separate re / im planes with an XOR-folded index, which spreads the scattered writes over banks.
constexpr int kPackTile = 1024;
constexpr int kPackThreads = 256;
__device__ __forceinline__ int pack_swz(int e) { return e ^ ((e >> 5) & 31); }
template <typename PT>  // plane element: float (split-TF32), __nv_bfloat16 (split-BF16) or bf16p3 (three pieces)
static __global__ void __launch_bounds__(kPackThreads, 6) k_pack_tiled(
    const cf32* __restrict__ src, PT* __restrict__ dst, const int* __restrict__ rd_rank,
    const int* __restrict__ rd_off, const int* __restrict__ wr_off, int T, const ll* __restrict__ src_base,
    const ll* __restrict__ dst_base, ll n_outer, ll n_slices, ll dst_slice_stride, ll plane, SliceOff so, ll g0,
    int conj) {
  constexpr int PER = kPackTile / kPackThreads;
  __shared__ float t_re[kPackTile], t_im[kPackTile];
  const float im_sign = conj ? -1.f : 1.f;
  int rr[PER], ro[PER], wo[PER];
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int i = threadIdx.x + j * kPackThreads;
    rr[j] = i < T ? pack_swz(rd_rank[i]) : 0;
    ro[j] = i < T ? rd_off[i] : 0;
    wo[j] = i < T ? wr_off[i] : 0;
  }
  const ll n_blk = n_outer * n_slices;
  // Software pipeline: the loads of the next tile are in flight while this tile is written out.
  auto load = [&](ll blk, cf32* v) {
    const ll s = blk / n_outer, o = blk - s * n_outer;
    const cf32* sb = src + slice_offset(so, g0, s) + src_base[o];
#pragma unroll
    for (int j = 0; j < PER; ++j)
      if (threadIdx.x + j * kPackThreads < T) v[j] = sb[ro[j]];
  };
  cf32 v[PER], nv[PER];
  ll blk = blockIdx.x;
  if (blk < n_blk) load(blk, v);
  for (; blk < n_blk; blk += gridDim.x) {
#pragma unroll
    for (int j = 0; j < PER; ++j)
      if (threadIdx.x + j * kPackThreads < T) {
        t_re[rr[j]] = v[j].re;
        t_im[rr[j]] = v[j].im;
      }
    __syncthreads();
    const ll next = blk + gridDim.x;
    if (next < n_blk) load(next, nv);
    const ll s = blk / n_outer, o = blk - s * n_outer;
    PT* db = dst + s * dst_slice_stride + dst_base[o];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int i = threadIdx.x + j * kPackThreads;
      if (i < T) {
        const int e = pack_swz(i);
        put_split(db, plane, wo[j], t_re[e]);
        put_split(db + pieces_of<PT>() * plane, plane, wo[j], im_sign * t_im[e]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < PER; ++j) v[j] = nv[j];
  }
}

// C[e] = sum over splits s = 0, 1, ... of part[s][e], added in that order in FP64 and rounded once.
static __global__ void k_splitk_reduce(const cf32* __restrict__ part, cf32* __restrict__ C, ll count, int splits) {
  for (ll e = (ll)blockIdx.x * blockDim.x + threadIdx.x; e < count; e += (ll)gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int s = 0; s < splits; ++s) {
      const cf32 v = part[(ll)s * count + e];
      re += v.re;
      im += v.im;
    }
    C[e] = cf32{(float)re, (float)im};
  }
}

// Gather one operand of a pairwise step into K-major fp32 planes:
//   dst[(p*Z + z)*Rpad*Kpad + r*Kpad + c] = (p == 0 ? re : im) of src(z, r, c), zero in the padding,
// where src(z, r, c) = src[sliceoff(z / bt) + tabB[z % bt] + tabR[r] + tabC[c]].
// This is the permute of the reference step (src/tensor.rs:453-492) fused with the planar split.
// A 32 x 32 (r, c) tile goes through shared memory: it is read along whichever index the source
// walks with unit stride (r_major) and written along c, so both sides stay coalesced.
template <typename PT>  // plane element: float (split-TF32), __nv_bfloat16 (split-BF16) or bf16p3 (three pieces)
static __global__ void __launch_bounds__(256) k_pack_planar(const cf32* __restrict__ src, PT* __restrict__ dst,
                                                     const ll* __restrict__ tabB, const ll* __restrict__ tabR,
                                                     const ll* __restrict__ tabC, ll bt, ll R, ll K, ll Rpad, ll Kpad,
                                                     ll Z, SliceOff so, ll g0, int r_major, int conj) {
  const float im_sign = conj ? -1.f : 1.f;
  __shared__ cf32 tile[32][33];
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;  // 32 x 8
  const ll tiles_c = (Kpad + 31) / 32, tiles_r = Rpad / 32, per_z = tiles_c * tiles_r;
  const ll plane = Z * Rpad * Kpad;
  for (ll t = blockIdx.x; t < Z * per_z; t += gridDim.x) {
    const ll zz = t / per_z, rem = t - zz * per_z;
    const ll r0 = (rem / tiles_c) * 32, c0 = (rem % tiles_c) * 32;
    const ll s = zz / bt, b = zz - s * bt;
    const cf32* base = src + slice_offset(so, g0, s) + tabB[b];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int u = ty + 8 * j;
      const ll r = r0 + (r_major ? tx : u), c = c0 + (r_major ? u : tx);
      cf32 v{0.f, 0.f};
      if (r < R && c < K) v = base[tabR[r] + tabC[c]];
      if (r_major) tile[tx][u] = v;
      else tile[u][tx] = v;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int u = ty + 8 * j;
      const ll r = r0 + u, c = c0 + tx;
      if (c < Kpad) {
        const ll o = (zz * Rpad + r) * Kpad + c;
        put_split(dst, plane, o, tile[u][tx].re);
        put_split(dst + pieces_of<PT>() * plane, plane, o, im_sign * tile[u][tx].im);
      }
    }
    __syncthreads();
  }
}

// A real float32 operand packed as a complex one of half the K (Kc = ceil(K / 2)): element (z, r, c) is
// src(z, r, c) + i src(z, r, c + Kc), zero past K, conjugated for the B operand; then the same tile
// transposition and planar split as k_pack_planar.  With both operands packed this way the complex
// product's real part is the real product over the full K.
template <typename PT>
static __global__ void __launch_bounds__(256) k_pack_planar_real(const float* __restrict__ src, PT* __restrict__ dst,
                                                          const ll* __restrict__ tabB, const ll* __restrict__ tabR,
                                                          const ll* __restrict__ tabC, ll bt, ll R, ll Kc, ll K,
                                                          ll Rpad, ll Kpad, ll Z, SliceOff so, ll g0, int r_major,
                                                          int conj) {
  const float im_sign = conj ? -1.f : 1.f;
  __shared__ cf32 tile[32][33];
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;  // 32 x 8
  const ll tiles_c = (Kpad + 31) / 32, tiles_r = Rpad / 32, per_z = tiles_c * tiles_r;
  const ll plane = Z * Rpad * Kpad;
  for (ll t = blockIdx.x; t < Z * per_z; t += gridDim.x) {
    const ll zz = t / per_z, rem = t - zz * per_z;
    const ll r0 = (rem / tiles_c) * 32, c0 = (rem % tiles_c) * 32;
    const ll s = zz / bt, b = zz - s * bt;
    const float* base = src + slice_offset(so, g0, s) + tabB[b];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int u = ty + 8 * j;
      const ll r = r0 + (r_major ? tx : u), c = c0 + (r_major ? u : tx);
      cf32 v{0.f, 0.f};
      if (r < R && c < Kc) {
        v.re = base[tabR[r] + tabC[c]];
        if (c + Kc < K) v.im = base[tabR[r] + tabC[c + Kc]];
      }
      if (r_major) tile[tx][u] = v;
      else tile[u][tx] = v;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int u = ty + 8 * j;
      const ll r = r0 + u, c = c0 + tx;
      if (c < Kpad) {
        const ll o = (zz * Rpad + r) * Kpad + c;
        put_split(dst, plane, o, tile[u][tx].re);
        put_split(dst + pieces_of<PT>() * plane, plane, o, im_sign * tile[u][tx].im);
      }
    }
    __syncthreads();
  }
}

}  // namespace tc
}  // namespace ab2

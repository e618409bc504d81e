// Tensor-pipe peak probe: the dense MMA rate of this GPU for the operand kinds the GEMMs use, and the rate of the
// split-TF32 GEMM's own MMA stream over operands laid out as its ring (kind 2: every operand 1.0; kind 3: random
// TF32 hi / lo values with random signs, as the GEMM's packed operands).  The tensor pipe's power depends on how
// many operand bits change from one MMA to the next, so under the power cap the two kinds can settle at
// different clocks when run for seconds.
//
// Every SM runs one CTA whose single issuing thread streams `iters` tcgen05.mma instructions (M = 128,
// N = 128 or 256, K = 8 for kind::tf32 / 16 for kind::f16 with BF16 operands) over operands that stay
// resident in shared memory, accumulating into TMEM.  There is no TMA traffic and no epilogue, so the
// rate is the tensor pipe's own, limited only by how fast it can read its operands from shared memory:
// an M = 128, N = 128 TF32 MMA reads 8 KB for 131072 MACs, an N = 256 one 12 KB for twice the MACs.
// The host times the launch with CUDA events; flops = 2 * 128 * N * K * iters * CTAs.  The only wait (the
// final commit) is bounded and reports expiry in the caller's status word.
#include <cuda_runtime.h>

#include <string>

#include "../../include/arctn_b200.h"
#include "tc_gemm.cuh"

namespace ab2 {
void set_last_error(const std::string& m);  // capi.cu
}

namespace {

using namespace ab2;

__host__ __device__ constexpr uint32_t peak_idesc(bool bf16, int n) {
  return (1u << 4) | ((bf16 ? 1u : 2u) << 7) | ((bf16 ? 1u : 2u) << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

template <bool kBF16, int N>
__global__ void __launch_bounds__(128, 1) k_tc_peak(long long iters, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  constexpr int kRows = 128 + N;  // A rows then B rows, 64 bytes each (64-byte swizzle atoms)
  uint32_t* words = (uint32_t*)smem;
  // Operand values: 1.0 (TF32) or a pair of BF16 1.0; the sums stay finite for every allowed iters.
  const uint32_t one = kBF16 ? 0x3F803F80u : 0x3F800000u;
  for (int i = threadIdx.x; i < kRows * 16; i += blockDim.x) words[i] = one;
  uint64_t* bar = (uint64_t*)(smem + kRows * 64);
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(bar + 1);
  const int warp = threadIdx.x / 32;
  if (threadIdx.x == 0) {
    tc::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // operand writes visible to the tensor core
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32((const void*)tmem_slot)),
                 "r"((uint32_t)N));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  if (threadIdx.x == 32) {
    const uint32_t a0 = tc::smem_u32(smem), b0 = a0 + 128 * 64;
    const uint32_t idesc = peak_idesc(kBF16, N);
    for (long long i = 0; i < iters; ++i) {
      const uint32_t o = (uint32_t)(i & 1) * 32;  // the two 32-byte K halves of the 64-byte rows
      tc::umma<kBF16>(tmem, tc::sw64_desc(a0 + o), tc::sw64_desc(b0 + o), idesc, i > 0 ? 1u : 0u);
    }
    tc::umma_commit(bar);
    tc::mbar_wait(bar, 0, err, 9);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)N));
  }
}

// The split-TF32 GEMM's own MMA stream without TMA or epilogue: per iteration (one 8-wide K step) the 12 MMAs of
// the 4M product in the kernel's order, over A and B planes laid out as the GEMM's operand ring -- three
// 64 KB stages of 8 planes, a new stage every two iterations -- into two accumulators (Cr, Ci).  Its rate is
// the ceiling the GEMM's MMA phase can reach with operands streaming through shared memory.
// A 32-bit integer mix (the MurmurHash3 finaliser), for the random operands.
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x85EBCA6Bu;
  x ^= x >> 13;
  x *= 0xC2B2AE35u;
  x ^= x >> 16;
  return x;
}

template <bool kRandom>
__global__ void __launch_bounds__(128, 1) k_tc_peak_stream(long long iters, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint32_t* words = (uint32_t*)smem;
  for (int i = threadIdx.x; i < tc::STAGES * tc::STAGE_BYTES / 4; i += blockDim.x) {
    if constexpr (kRandom) {
      // plane (i * 4 / PLANE_BYTES) % 8: even planes hold hi parts in +-[0.5, 1), odd planes lo parts about 2^-11
      // of that; both carry a random 10-bit TF32 mantissa and a random sign
      const uint32_t h = mix32((uint32_t)i * 0x9E3779B9u + blockIdx.x * 0x632BE5ABu + 1u);
      const bool lo = ((i * 4 / tc::PLANE_BYTES) & 1) != 0;
      words[i] = (h & 0x80000000u) | (lo ? 0x39800000u : 0x3F000000u) | (h & 0x007FE000u);
    } else {
      words[i] = 0x3F800000u;
    }
  }
  uint64_t* bar = (uint64_t*)(smem + tc::STAGES * tc::STAGE_BYTES);
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(bar + 1);
  const int warp = threadIdx.x / 32;
  if (threadIdx.x == 0) {
    tc::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32((const void*)tmem_slot)),
                 "r"(256u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  if (threadIdx.x == 32) {
    const uint32_t base = tc::smem_u32(smem), P = tc::PLANE_BYTES;
    const uint32_t cr = tmem, ci = tmem + 128;
    const uint32_t pos = tc::idesc_tf32(false), neg = tc::idesc_tf32(true);
    for (long long i = 0; i < iters; ++i) {
      const uint32_t o = (uint32_t)(i & 1) * 32;
      const uint32_t a0 = base + (uint32_t)((i / 2) % tc::STAGES) * tc::STAGE_BYTES, b0 = a0 + tc::PLANES * P;
      const uint32_t hAr = a0 + o, lAr = hAr + P, hAi = hAr + 2 * P, lAi = hAr + 3 * P;
      const uint32_t hBr = b0 + o, lBr = hBr + P, hBi = hBr + 2 * P, lBi = hBr + 3 * P;
      const uint32_t acc = i > 0 ? 1u : 0u;
      tc::umma<false>(cr, tc::sw64_desc(hAr), tc::sw64_desc(hBr), pos, acc);
      tc::umma<false>(ci, tc::sw64_desc(hAr), tc::sw64_desc(hBi), pos, acc);
      tc::umma<false>(cr, tc::sw64_desc(hAi), tc::sw64_desc(hBi), neg, 1);
      tc::umma<false>(ci, tc::sw64_desc(hAi), tc::sw64_desc(hBr), pos, 1);
      tc::umma<false>(cr, tc::sw64_desc(lAr), tc::sw64_desc(hBr), pos, 1);
      tc::umma<false>(ci, tc::sw64_desc(lAr), tc::sw64_desc(hBi), pos, 1);
      tc::umma<false>(cr, tc::sw64_desc(lAi), tc::sw64_desc(hBi), neg, 1);
      tc::umma<false>(ci, tc::sw64_desc(lAi), tc::sw64_desc(hBr), pos, 1);
      tc::umma<false>(cr, tc::sw64_desc(hAr), tc::sw64_desc(lBr), pos, 1);
      tc::umma<false>(ci, tc::sw64_desc(hAr), tc::sw64_desc(lBi), pos, 1);
      tc::umma<false>(cr, tc::sw64_desc(hAi), tc::sw64_desc(lBi), neg, 1);
      tc::umma<false>(ci, tc::sw64_desc(hAi), tc::sw64_desc(lBr), pos, 1);
    }
    tc::umma_commit(bar);
    tc::mbar_wait(bar, 0, err, 9);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u));
  }
}

// The three-piece split-BF16 GEMM's MMA stream (FMT_BF16X6) on random operands: per iteration (one 16-wide K step)
// the 24 kind::f16 MMAs of its 4M product in the kernel's order -- products (h,h), (h,m), (m,h), (h,l), (l,h),
// (m,m) of each real product -- over planes laid out as its two-stage ring of 96 KB stages (re h, m, l, im h,
// m, l for A, then B), a new stage every two iterations.  Pieces are random BF16 values with random signs:
// h in +-[0.5, 1), m about 2^-8 and l about 2^-16 of that.
__global__ void __launch_bounds__(128, 1) k_tc_peak_six(long long iters, int* err) {
  using FM = tc::Fmt<tc::FMT_BF16X6>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint32_t* words = (uint32_t*)smem;
  for (int i = threadIdx.x; i < FM::kStages * FM::kStageBytes / 4; i += blockDim.x) {
    const uint32_t h = mix32((uint32_t)i * 0x9E3779B9u + blockIdx.x * 0x632BE5ABu + 7u);
    const int piece = ((i * 4 % FM::kStageBytes) / tc::PLANE_BYTES) % 3;  // h, m, l
    const uint32_t base = piece == 0 ? 0x3F00u : piece == 1 ? 0x3B00u : 0x3700u;
    const uint32_t lo16 = (h & 0x8000u) | base | (h & 0x7Fu), hi16 = ((h >> 16) & 0x8000u) | base | ((h >> 16) & 0x7Fu);
    words[i] = hi16 << 16 | lo16;
  }
  uint64_t* bar = (uint64_t*)(smem + FM::kStages * FM::kStageBytes);
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(bar + 1);
  const int warp = threadIdx.x / 32;
  if (threadIdx.x == 0) {
    tc::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32((const void*)tmem_slot)),
                 "r"(256u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  if (threadIdx.x == 32) {
    const uint32_t base = tc::smem_u32(smem), P = tc::PLANE_BYTES;
    const uint32_t cr = tmem, ci = tmem + 128;
    const uint32_t pos = tc::idesc_bf16(false), neg = tc::idesc_bf16(true);
    constexpr int px[6] = {0, 0, 1, 0, 2, 1}, py[6] = {0, 1, 0, 2, 0, 1};
    for (long long i = 0; i < iters; ++i) {
      const uint32_t o = (uint32_t)(i & 1) * 32;
      const uint32_t a0 = base + (uint32_t)((i / 2) % FM::kStages) * FM::kStageBytes, b0 = a0 + FM::kPlanes * P;
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const uint32_t Ar = a0 + px[q] * P + o, Ai = Ar + 3 * P;
        const uint32_t Br = b0 + py[q] * P + o, Bi = Br + 3 * P;
        const uint32_t acc = (i > 0 || q > 0) ? 1u : 0u;
        tc::umma<true>(cr, tc::sw64_desc(Ar), tc::sw64_desc(Br), pos, acc);
        tc::umma<true>(ci, tc::sw64_desc(Ar), tc::sw64_desc(Bi), pos, acc);
        tc::umma<true>(cr, tc::sw64_desc(Ai), tc::sw64_desc(Bi), neg, 1);
        tc::umma<true>(ci, tc::sw64_desc(Ai), tc::sw64_desc(Br), pos, 1);
      }
    }
    tc::umma_commit(bar);
    tc::mbar_wait(bar, 0, err, 9);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u));
  }
}

// A 3M (Gauss) split-TF32 complex product's MMA stream on random operands, as a measurement of what that form
// would sustain: per iteration (one 8-wide K step) 9 MMAs -- the split products (h,h), (l,h), (h,l) of
// T1 = Ar.Br, T2 = Ai.Bi and T3 = (Ar + Ai).(Br + Bi), into three accumulators -- over six planes per operand
// (hi and lo of Ar, Ai and Ar + Ai) in a two-stage ring of 96 KB stages.  Re = T1 - T2 and Im = T3 - T1 - T2
// would be formed when draining; the probe only streams the MMAs.
__global__ void __launch_bounds__(128, 1) k_tc_peak_3m(long long iters, int* err) {
  constexpr int kPlanes = 6, kStageBytes = 2 * kPlanes * tc::PLANE_BYTES, kStages = 2;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint32_t* words = (uint32_t*)smem;
  for (int i = threadIdx.x; i < kStages * kStageBytes / 4; i += blockDim.x) {
    const uint32_t h = mix32((uint32_t)i * 0x9E3779B9u + blockIdx.x * 0x632BE5ABu + 11u);
    const bool lo = ((i * 4 / tc::PLANE_BYTES) & 1) != 0;
    words[i] = (h & 0x80000000u) | (lo ? 0x39800000u : 0x3F000000u) | (h & 0x007FE000u);
  }
  uint64_t* bar = (uint64_t*)(smem + kStages * kStageBytes);
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(bar + 1);
  const int warp = threadIdx.x / 32;
  if (threadIdx.x == 0) {
    tc::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32((const void*)tmem_slot)),
                 "r"(512u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  if (threadIdx.x == 32) {
    const uint32_t base = tc::smem_u32(smem), P = tc::PLANE_BYTES;
    const uint32_t t1 = tmem, t2 = tmem + 128, t3 = tmem + 256;
    const uint32_t pos = tc::idesc_tf32(false);
    for (long long i = 0; i < iters; ++i) {
      const uint32_t o = (uint32_t)(i & 1) * 32;
      const uint32_t a0 = base + (uint32_t)((i / 2) % kStages) * kStageBytes + o, b0 = a0 + kPlanes * P;
      const uint32_t acc = i > 0 ? 1u : 0u;
      // operand planes: 0/1 hi/lo of the real part, 2/3 of the imaginary part, 4/5 of their sum
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        const uint32_t d = t == 0 ? t1 : t == 1 ? t2 : t3, ah = a0 + 2 * t * P, bh = b0 + 2 * t * P;
        tc::umma<false>(d, tc::sw64_desc(ah), tc::sw64_desc(bh), pos, acc);
        tc::umma<false>(d, tc::sw64_desc(ah + P), tc::sw64_desc(bh), pos, 1);
        tc::umma<false>(d, tc::sw64_desc(ah), tc::sw64_desc(bh + P), pos, 1);
      }
    }
    tc::umma_commit(bar);
    tc::mbar_wait(bar, 0, err, 9);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u));
  }
}

cudaError_t launch_peak_3m(int ctas, long long iters, int* err, cudaStream_t st) {
  constexpr int smem = 2 * 2 * 6 * tc::PLANE_BYTES + 64 + 1024;
  cudaError_t e = cudaFuncSetAttribute(k_tc_peak_3m, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_tc_peak_3m<<<ctas, 128, smem, st>>>(iters, err);
  return cudaGetLastError();
}

cudaError_t launch_peak_six(int ctas, long long iters, int* err, cudaStream_t st) {
  constexpr int smem = tc::Fmt<tc::FMT_BF16X6>::kStages * tc::Fmt<tc::FMT_BF16X6>::kStageBytes + 64 + 1024;
  cudaError_t e = cudaFuncSetAttribute(k_tc_peak_six, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_tc_peak_six<<<ctas, 128, smem, st>>>(iters, err);
  return cudaGetLastError();
}

template <bool kRandom>
cudaError_t launch_peak_stream(int ctas, long long iters, int* err, cudaStream_t st) {
  constexpr int smem = tc::STAGES * tc::STAGE_BYTES + 64 + 1024;
  cudaError_t e = cudaFuncSetAttribute(k_tc_peak_stream<kRandom>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_tc_peak_stream<kRandom><<<ctas, 128, smem, st>>>(iters, err);
  return cudaGetLastError();
}

template <bool kBF16, int N>
cudaError_t launch_peak(int ctas, long long iters, int* err, cudaStream_t st) {
  constexpr int smem = (128 + N) * 64 + 64 + 1024;
  cudaError_t e = cudaFuncSetAttribute(k_tc_peak<kBF16, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_tc_peak<kBF16, N><<<ctas, 128, smem, st>>>(iters, err);
  return cudaGetLastError();
}

}  // namespace

extern "C" int arctn_b200_tc_peak(int kind, int n, uint64_t iters, void* status, void* cuda_stream,
                                  double* tflops_out) {
  auto fail = [](const std::string& m, int code) {
    ab2::set_last_error(m);
    return code;
  };
  if (kind < 0 || kind > 5)
    return fail("kind must be 0 (tf32), 1 (bf16), 2 (split-TF32 GEMM stream), 3 (the stream on random operands), "
                "4 (the three-piece split-BF16 GEMM stream on random operands) or 5 (a 3M split-TF32 stream on "
                "random operands)", ARCTN_B200_ERR_INVALID);
  if (n != 128 && n != 256) return fail("n must be 128 or 256", ARCTN_B200_ERR_INVALID);
  if (kind >= 2 && n != 128) return fail("kinds 2 to 5 run the GEMMs' N = 128 MMAs", ARCTN_B200_ERR_INVALID);
  if (iters < 2 || iters > (1ull << 22)) return fail("iters must lie in [2, 2^22]", ARCTN_B200_ERR_INVALID);
  if (!status || !tflops_out) return fail("status and tflops_out must not be null", ARCTN_B200_ERR_INVALID);
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return fail("no usable current device", ARCTN_B200_ERR_CUDA);
  cudaStream_t st = (cudaStream_t)cuda_stream;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    return fail("cudaEventCreate failed", ARCTN_B200_ERR_CUDA);
  cudaError_t e = cudaEventRecord(e0, st);
  const long long it = (long long)iters;
  int* err = (int*)status;
  if (e == cudaSuccess) {
    if (kind == 2) e = launch_peak_stream<false>(sms, it, err, st);
    else if (kind == 3) e = launch_peak_stream<true>(sms, it, err, st);
    else if (kind == 4) e = launch_peak_six(sms, it, err, st);
    else if (kind == 5) e = launch_peak_3m(sms, it, err, st);
    else if (kind == 0) e = n == 128 ? launch_peak<false, 128>(sms, it, err, st) : launch_peak<false, 256>(sms, it, err, st);
    else e = n == 128 ? launch_peak<true, 128>(sms, it, err, st) : launch_peak<true, 256>(sms, it, err, st);
  }
  if (e == cudaSuccess) e = cudaEventRecord(e1, st);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return fail(std::string("tensor-core peak probe: ") + cudaGetErrorString(e), ARCTN_B200_ERR_CUDA);
  // kinds 2, 3: 12 TF32 MMAs (K = 8) an iteration; kind 4: 24 BF16 MMAs (K = 16); kind 5: 9 TF32 MMAs
  const double k = (kind == 1 || kind == 4) ? 16.0 : 8.0;
  const double per_iter = kind == 5 ? 9.0 : kind == 4 ? 24.0 : kind >= 2 ? 12.0 : 1.0;
  *tflops_out = 2.0 * 128.0 * n * k * per_iter * (double)iters * sms / (ms * 1e-3) / 1e12;
  ab2::set_last_error("");
  return ARCTN_B200_OK;
}

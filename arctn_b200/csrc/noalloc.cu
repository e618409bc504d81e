// Batched complex64 GEMM on the split-TF32 tensor-core path that allocates no
// device memory.
//
// Some callers cannot call cudaMalloc: code that runs while a framework holds
// the whole device memory pool (allocators that pre-reserve all HBM, such as
// XLA's preallocation), code inside a region where an allocation would
// synchronise the device or break a stream capture, and plugins whose host
// process forbids foreign allocations.  For them this file offers one entry
// point whose scratch -- the planar operand copies the tensor-core kernel
// reads and its status word -- lives in a file-scope __device__ array of
// kScratchBytes that every GPU loading the library holds until the process
// exits.  The caller still provides A, B and C.
//
// The first call on a device looks up the device address of the array with
// cudaGetSymbolAddress (host code cannot use the array's name as a device
// pointer); make that first call before any stream capture.  Every call on a
// device shares the one array and leaves its contents behind, so calls whose
// work overlaps on the GPU (different streams, no ordering) race: order them.
//
// The array's first 256 bytes hold the kernel's status word (the code of a
// bounded wait that expired, 0 otherwise), cleared by every call and read back
// by arctn_b200_cgemm_noalloc_status; the operand planes follow it.
#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/arctn_b200.h"
#include "tc_gemm.cuh"

namespace {

using ab2::ll;

constexpr size_t kScratchBytes = 64u << 20;  // 64 MiB per device
constexpr size_t kStatusBytes = 256;          // status word at the start, then the operand planes
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};
bool g_attr_set[kMaxDevices] = {};

// src[b*bs + r*rs + c*cs] -> K-major TF32-pair planes [re_hi|re_lo|im_hi|im_lo][b][Rpad][Kpad], zero padding.
__global__ void __launch_bounds__(256) k_pack_strided(const ab2::cf32* __restrict__ src, float* __restrict__ dst,
                                                      ll Z, ll R, ll K, ll Rpad, ll Kpad, ll bs, ll rs, ll cs,
                                                      int r_major) {
  __shared__ ab2::cf32 tile[32][33];
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;
  const ll tiles_c = (Kpad + 31) / 32, tiles_r = Rpad / 32, per_z = tiles_c * tiles_r;
  const ll plane = Z * Rpad * Kpad;
  for (ll t = blockIdx.x; t < Z * per_z; t += gridDim.x) {
    const ll z = t / per_z, rem = t - z * per_z;
    const ll r0 = (rem / tiles_c) * 32, c0 = (rem % tiles_c) * 32;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int u = ty + 8 * j;
      const ll r = r0 + (r_major ? tx : u), c = c0 + (r_major ? u : tx);
      ab2::cf32 v{0.f, 0.f};
      if (r < R && c < K) v = src[z * bs + r * rs + c * cs];
      if (r_major) tile[tx][u] = v;
      else tile[u][tx] = v;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int u = ty + 8 * j;
      const ll r = r0 + u, c = c0 + tx;
      if (c < Kpad) {
        const ll o = (z * Rpad + r) * Kpad + c;
        ab2::tc::put_split(dst, plane, o, tile[u][tx].re);
        ab2::tc::put_split(dst + 2 * plane, plane, o, tile[u][tx].im);
      }
    }
    __syncthreads();
  }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

bool plane_map(CUtensorMap* m, void* base, ll kpad, ll rows, ll zplanes) {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiled)p;
  });
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)kpad, (cuuint64_t)rows, (cuuint64_t)zplanes};
  cuuint64_t strides[2] = {(cuuint64_t)(kpad * 4), (cuuint64_t)(kpad * rows * 4)};
  cuuint32_t box[3] = {(cuuint32_t)ab2::tc::BK, (cuuint32_t)ab2::tc::BM, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

}  // namespace

namespace ab2 {
void set_last_error(const std::string& m);  // capi.cu: the library's arctn_b200_last_error() channel
}

namespace {
int fail_with(const std::string& m, int code) {
  ab2::set_last_error(m);
  return code;
}
}  // namespace

extern "C" int arctn_b200_cgemm_tf32x3_noalloc(const void* a, const void* b, void* c, uint64_t bt, uint64_t m,
                                               uint64_t k, uint64_t n, void* cuda_stream) {
  using namespace ab2;
  if (!a || !b || !c) return fail_with("A, B and C must be device pointers", ARCTN_B200_ERR_INVALID);
  if (bt == 0 || m == 0 || k == 0 || n == 0) return fail_with("bt, m, k and n must be positive", ARCTN_B200_ERR_INVALID);
  const unsigned __int128 kpad = (k + tc::BK - 1) / tc::BK * tc::BK, rpa = (m + tc::BM - 1) / tc::BM * tc::BM,
                          rpb = (n + tc::BN - 1) / tc::BN * tc::BN;
  const unsigned __int128 a_bytes = ab2::tc::PLANES * (unsigned __int128)bt * rpa * kpad * 4;
  const unsigned __int128 b_bytes = ab2::tc::PLANES * (unsigned __int128)bt * rpb * kpad * 4;
  const unsigned __int128 need = kStatusBytes + ((a_bytes + 255) / 256 * 256) + ((b_bytes + 255) / 256 * 256);
  if (need > kScratchBytes)
    return fail_with("problem needs " + std::to_string((unsigned long long)need) + " scratch bytes; the fixed maximum is " +
                         std::to_string(kScratchBytes) + " (reduce bt, m, n or k)",
                     ARCTN_B200_ERR_UNSUPPORTED);
  if (bt > 65535) return fail_with("bt exceeds 65535", ARCTN_B200_ERR_UNSUPPORTED);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev >= kMaxDevices) return fail_with("no usable current device", ARCTN_B200_ERR_CUDA);
  unsigned char* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {  // set-up, once per device, with that device current
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return fail_with(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e), ARCTN_B200_ERR_CUDA);
      g_scratch_ptr[dev] = p;
    }
    if (!g_attr_set[dev]) {
      cudaError_t e = cudaFuncSetAttribute(tc::k_tc_cgemm_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES);
      if (e != cudaSuccess) return fail_with(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e), ARCTN_B200_ERR_CUDA);
      cudaFuncAttributes fa{};
      e = cudaFuncGetAttributes(&fa, tc::k_tc_cgemm_tf32x3);
      if (e != cudaSuccess) return fail_with(std::string("cudaFuncGetAttributes: ") + cudaGetErrorString(e), ARCTN_B200_ERR_CUDA);
      if (fa.numRegs != tc::kLaunchRegs)
        return fail_with("tensor-core GEMM register count differs from its setmaxnreg split", ARCTN_B200_ERR_UNSUPPORTED);
      g_attr_set[dev] = true;
    }
    scratch = (unsigned char*)g_scratch_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)cuda_stream;
  int* err = (int*)scratch;
  float* pa = (float*)(scratch + kStatusBytes);
  float* pb = (float*)(scratch + kStatusBytes + (size_t)((a_bytes + 255) / 256 * 256));
  // The status word must start at zero; the planes are fully rewritten (padding included) by the packs.
  if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) return fail_with("cudaMemsetAsync failed", ARCTN_B200_ERR_CUDA);
  const ll Kp = (ll)kpad, Ra = (ll)rpa, Rb = (ll)rpb, Z = (ll)bt;
  auto tiles = [](ll z, ll r, ll kp) { return (int)std::min<ll>(z * (r / 32) * ((kp + 31) / 32), 148 * 16); };
  // A (bt x m x k, row-major): rows m, k contiguous.  B (bt x k x n): rows n are contiguous, k strided.
  k_pack_strided<<<tiles(Z, Ra, Kp), 256, 0, st>>>((const cf32*)a, pa, Z, (ll)m, (ll)k, Ra, Kp, (ll)(m * k), (ll)k, 1, 0);
  k_pack_strided<<<tiles(Z, Rb, Kp), 256, 0, st>>>((const cf32*)b, pb, Z, (ll)n, (ll)k, Rb, Kp, (ll)(k * n), 1, (ll)n, 1);
  CUtensorMap ma, mb;
  if (!plane_map(&ma, pa, Kp, Ra, ab2::tc::PLANES * Z) || !plane_map(&mb, pb, Kp, Rb, ab2::tc::PLANES * Z))
    return fail_with("cuTensorMapEncodeTiled failed", ARCTN_B200_ERR_CUDA);
  tc::TcArgs args;
  args.C = (cf32*)c;
  args.m = (ll)m;
  args.n = (ll)n;
  args.k_tiles = (int)(Kp / tc::BK);
  args.za = (int)Z;
  args.zb = (int)Z;
  args.bt = (int)Z;
  args.a_var = 0;
  args.b_var = 0;
  args.err = err;
  args.m_tiles = (int)(Ra / tc::BM);
  args.m_fast = Ra <= Rb ? 1 : 0;
  args.zc = (int)Z;
  args.tiles = (int)((Ra / tc::BM) * (Rb / tc::BN));
  args.n_items = args.tiles * (int)Z;
  int n_sm = 0;
  if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n_sm <= 0)
    return fail_with("cudaDeviceGetAttribute failed", ARCTN_B200_ERR_CUDA);
  tc::k_tc_cgemm_tf32x3<<<(unsigned)std::min(args.n_items, n_sm), tc::kThreads, tc::SMEM_BYTES, st>>>(ma, mb, args);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_with(std::string("launch: ") + cudaGetErrorString(e), ARCTN_B200_ERR_CUDA);
  ab2::set_last_error("");
  return ARCTN_B200_OK;
}

// Waits for cuda_stream, then copies the status word of the last call on the current device into *code
// (0: every bounded wait of the kernel completed; nonzero: the code of the wait that expired, and C is
// incomplete).  One device-to-host copy of 4 bytes into the caller's host memory; nothing is allocated.
extern "C" int arctn_b200_cgemm_noalloc_status(void* cuda_stream, int* code) {
  if (!code) return fail_with("code must point to host memory", ARCTN_B200_ERR_INVALID);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev >= kMaxDevices) return fail_with("no usable current device", ARCTN_B200_ERR_CUDA);
  void* p = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    p = g_scratch_ptr[dev];
  }
  if (!p) {  // no call on this device yet: nothing can have failed
    *code = 0;
    ab2::set_last_error("");
    return ARCTN_B200_OK;
  }
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)cuda_stream);
  if (e != cudaSuccess) return fail_with(std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e), ARCTN_B200_ERR_CUDA);
  int v = 0;
  e = cudaMemcpy(&v, p, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail_with(std::string("cudaMemcpy: ") + cudaGetErrorString(e), ARCTN_B200_ERR_CUDA);
  *code = v;
  ab2::set_last_error("");
  return ARCTN_B200_OK;
}

// SIMT kernels of the B200 executor (sm_100a).
//
// Every kernel reads its operands through offset tables built on the host: a
// pairwise step C[s,b,i,j] = sum_l A[s,b,i,l] * B[s,b,l,j] reads
//   A[sliceoff_A(s) + aB[b] + aM[i] + aK[l]]   and   B[sliceoff_B(s) + bB[b] + bK[l] + bN[j]]
// so the reference's permute (src/tensor.rs:453-492) and slice selection
// (src/tensor.rs:636-669, src/slice.rs:1005-1012) are folded into the GEMM's
// loads instead of being materialised in HBM.  `s` runs over the slices of one
// group; slices are an extra batch dimension of every step.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ab2 {

typedef long long ll;

// ---------------------------------------------------------------- scalar types
struct __align__(8) cf32 { float re, im; };
struct __align__(16) cf64 { double re, im; };

template <class T> struct Num;
template <> struct Num<float> {
  using acc = float; using wide = double;
  __device__ static float zero() { return 0.f; }
  __device__ static void fma(float& c, float a, float b) { c = fmaf(a, b, c); }
  __device__ static double widen(float v) { return (double)v; }
  __device__ static float narrow(double v) { return (float)v; }
  __device__ static float add(float a, float b) { return a + b; }
  __device__ static double mag(float v) { return fabs((double)v); }
  __device__ static float scale(float v, double s) { return v * (float)s; }
};
template <> struct Num<double> {
  using acc = double; using wide = double;
  __device__ static double zero() { return 0.0; }
  __device__ static void fma(double& c, double a, double b) { c = fma_rn(a, b, c); }
  __device__ static double fma_rn(double a, double b, double c) { return ::fma(a, b, c); }
  __device__ static double widen(double v) { return v; }
  __device__ static double narrow(double v) { return v; }
  __device__ static double add(double a, double b) { return a + b; }
  __device__ static double mag(double v) { return fabs(v); }
  __device__ static double scale(double v, double s) { return v * s; }
};
template <> struct Num<cf32> {
  using acc = cf32; using wide = cf64;
  __device__ static cf32 zero() { return {0.f, 0.f}; }
  __device__ static void fma(cf32& c, cf32 a, cf32 b) {
    c.re = fmaf(a.re, b.re, c.re);
    c.re = fmaf(-a.im, b.im, c.re);
    c.im = fmaf(a.re, b.im, c.im);
    c.im = fmaf(a.im, b.re, c.im);
  }
  __device__ static cf64 widen(cf32 v) { return {(double)v.re, (double)v.im}; }
  __device__ static cf32 narrow(cf64 v) { return {(float)v.re, (float)v.im}; }
  __device__ static cf32 add(cf32 a, cf32 b) { return {a.re + b.re, a.im + b.im}; }
  __device__ static double mag(cf32 v) { return hypot((double)v.re, (double)v.im); }
  __device__ static cf32 scale(cf32 v, double s) { float f = (float)s; return {v.re * f, v.im * f}; }
};
template <> struct Num<cf64> {
  using acc = cf64; using wide = cf64;
  __device__ static cf64 zero() { return {0.0, 0.0}; }
  __device__ static void fma(cf64& c, cf64 a, cf64 b) {
    c.re = ::fma(a.re, b.re, c.re);
    c.re = ::fma(-a.im, b.im, c.re);
    c.im = ::fma(a.re, b.im, c.im);
    c.im = ::fma(a.im, b.re, c.im);
  }
  __device__ static cf64 widen(cf64 v) { return v; }
  __device__ static cf64 narrow(cf64 v) { return v; }
  __device__ static cf64 add(cf64 a, cf64 b) { return {a.re + b.re, a.im + b.im}; }
  __device__ static double mag(cf64 v) { return hypot(v.re, v.im); }
  __device__ static cf64 scale(cf64 v, double s) { return {v.re * s, v.im * s}; }
};

// Complex conjugate when `c` is set; identity for real types.
__device__ __forceinline__ float cj(float v, int) { return v; }
__device__ __forceinline__ double cj(double v, int) { return v; }
__device__ __forceinline__ cf32 cj(cf32 v, int c) { return c ? cf32{v.re, -v.im} : v; }
__device__ __forceinline__ cf64 cj(cf64 v, int c) { return c ? cf64{v.re, -v.im} : v; }

__device__ inline double wadd(double a, double b) { return a + b; }
__device__ inline cf64 wadd(cf64 a, cf64 b) { return {a.re + b.re, a.im + b.im}; }
__device__ inline double wzero(double*) { return 0.0; }
__device__ inline cf64 wzero(cf64*) { return {0.0, 0.0}; }

// ---------------------------------------------------------------- slice offsets
// Element offset of slice `s` (local index inside a group) of one operand:
//   s * local_stride + sum_t ((g0 + s) / div_t % mod_t) * stride_t
// The first term addresses per-slice intermediates laid out [S][numel]; the
// terms decode the global slice number into sliced-leg values for an input
// tensor (last sliced leg fastest, src/slice.rs:881-888).
constexpr int kMaxSliceTerms = 12;
struct SliceTerm { ll div, mod, stride; };
struct SliceOff {
  ll local_stride;
  int n;
  SliceTerm t[kMaxSliceTerms];
};

__device__ __forceinline__ ll slice_offset(const SliceOff& so, ll g0, ll s) {
  ll off = s * so.local_stride;
  const ll g = g0 + s;
  for (int i = 0; i < so.n; ++i) off += ((g / so.t[i].div) % so.t[i].mod) * so.t[i].stride;
  return off;
}

// ---------------------------------------------------------------- gather-reduce
// out[s*n_out + e] = sum_{r < n_red} in[sliceoff(s) + offE[e] + offR[r]]
// Used for input traces / diagonals (src/tensor.rs:503-590), dangling-leg sums
// (src/tensor.rs:593-633) and the final sum + permute (src/compiled.rs:211-218).
template <class T, class TO>
struct OutCast;
template <class T> struct OutCast<T, T> { __device__ static T cast(T v) { return v; } };
template <> struct OutCast<float, double> { __device__ static double cast(float v) { return v; } };
template <> struct OutCast<cf32, cf64> { __device__ static cf64 cast(cf32 v) { return {(double)v.re, (double)v.im}; } };

//
// Every SIMT kernel below is a thin __global__ wrapper over a __device__ body that takes its block index
// and block count (vb, nvb) as arguments: a launch passes (blockIdx.x, gridDim.x); the batch interpreter
// (interp.cuh) runs the same bodies as tasks of one persistent launch.  An output element's arithmetic
// never depends on (vb, nvb), so both forms give the same bits.
template <class T, class TO>
__device__ __forceinline__ void gather_reduce_body(const T* in, TO* out, const ll* offE, const ll* offR, ll n_out,
                                                   ll n_red, ll S, const SliceOff& so, ll g0, ll vb, ll nvb) {
  const ll total = S * n_out;
  for (ll idx = vb * blockDim.x + threadIdx.x; idx < total; idx += nvb * blockDim.x) {
    const ll s = idx / n_out, e = idx - s * n_out;
    const T* base = in + slice_offset(so, g0, s) + offE[e];
    T acc = base[offR[0]];
    for (ll r = 1; r < n_red; ++r) acc = Num<T>::add(acc, base[offR[r]]);
    out[idx] = OutCast<T, TO>::cast(acc);
  }
}
template <class T, class TO>
__global__ void k_gather_reduce(const T* __restrict__ in, TO* __restrict__ out, const ll* __restrict__ offE,
                                const ll* __restrict__ offR, ll n_out, ll n_red, ll S, SliceOff so, ll g0) {
  gather_reduce_body<T, TO>(in, out, offE, offR, n_out, n_red, S, so, g0, blockIdx.x, gridDim.x);
}

// out[offE[e] + offR[r]] = in[e] for every (e, r): the adjoint of a trace (every diagonal element
// receives the traced gradient) or of a diagonal extraction (the diagonal receives it).  The
// (e, r) -> position map is injective, so plain stores suffice after the output is zeroed.
template <class T>
__device__ __forceinline__ void scatter_body(const T* in, T* out, const ll* offE, const ll* offR, ll n_in, ll n_red,
                                             ll vb, ll nvb) {
  const ll total = n_in * n_red;
  for (ll idx = vb * blockDim.x + threadIdx.x; idx < total; idx += nvb * blockDim.x) {
    const ll e = idx / n_red, r = idx - e * n_red;
    out[offE[e] + offR[r]] = in[e];
  }
}
template <class T>
__global__ void k_scatter(const T* __restrict__ in, T* __restrict__ out, const ll* __restrict__ offE,
                          const ll* __restrict__ offR, ll n_in, ll n_red) {
  scatter_body<T>(in, out, offE, offR, n_in, n_red, blockIdx.x, gridDim.x);
}

// Gradient of a sliced input: acc[sliceoff(s) + offE[e]] += G[s][e] in the wide type.  One thread per
// element e walks the group's slices in order, so slices that share a sub-block (they differ only in
// sliced legs the input does not hold) add up deterministically without atomics; distinct (slice
// digits, e) pairs reach distinct targets because the input's index map is injective.
template <class T>
__device__ __forceinline__ void grad_accum_body(const T* G, typename Num<T>::wide* acc, const ll* offE, ll n_e, ll S,
                                                const SliceOff& so, ll g0, ll vb, ll nvb) {
  using W = typename Num<T>::wide;
  for (ll e = vb * blockDim.x + threadIdx.x; e < n_e; e += nvb * blockDim.x) {
    const ll t = offE[e];
    for (ll s = 0; s < S; ++s) {
      W* dst = acc + slice_offset(so, g0, s) + t;
      *dst = Num<W>::add(*dst, Num<T>::widen(G[s * n_e + e]));
    }
  }
}
template <class T>
__global__ void k_grad_accum(const T* __restrict__ G, typename Num<T>::wide* __restrict__ acc,
                             const ll* __restrict__ offE, ll n_e, ll S, SliceOff so, ll g0) {
  grad_accum_body<T>(G, acc, offE, n_e, S, so, g0, blockIdx.x, gridDim.x);
}

template <class T>
__device__ __forceinline__ void narrow_body(const typename Num<T>::wide* in, T* out, ll n, ll vb, ll nvb) {
  for (ll i = vb * blockDim.x + threadIdx.x; i < n; i += nvb * blockDim.x) out[i] = Num<T>::narrow(in[i]);
}
template <class T>
__global__ void k_narrow(const typename Num<T>::wide* __restrict__ in, T* __restrict__ out, ll n) {
  narrow_body<T>(in, out, n, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------- GEMM tables
struct GemmArgs {
  const void* A;
  const void* B;
  void* C;
  ll bt, m, k, n, S, g0;
  const ll* aB; const ll* aM; const ll* aK;
  const ll* bB; const ll* bK; const ll* bN;
  SliceOff sa, sb;
  int conj_a = 0, conj_b = 0;  // read an operand conjugated (adjoint steps)
};

// Thin steps: one thread per output element, k-loop through the tables.  sh_tab holds 2 * k entries
// when k <= 1024.  The bodies copy the scalar arguments to locals first: the interpreter passes `g` from
// global memory, where every access would otherwise be reloaded after each store.
template <class T>
__device__ __forceinline__ void gemm_small_body(const GemmArgs& g, ll* sh_tab, ll vb, ll nvb) {
  using A = typename Num<T>::acc;
  const T* Ap = (const T*)g.A;
  const T* Bp = (const T*)g.B;
  T* Cp = (T*)g.C;
  const ll m = g.m, k = g.k, n = g.n, g0 = g.g0;
  const ll *gaB = g.aB, *gaM = g.aM, *gaK = g.aK, *gbB = g.bB, *gbK = g.bK, *gbN = g.bN;
  const int ca = g.conj_a, cb = g.conj_b;
  const ll mn = m * n, per_s = g.bt * mn, total = g.S * per_s;
  const bool tab_in_smem = k <= 1024;
  if (tab_in_smem) {
    for (ll l = threadIdx.x; l < k; l += blockDim.x) { sh_tab[l] = gaK[l]; sh_tab[k + l] = gbK[l]; }
    __syncthreads();
  }
  const ll* aK = tab_in_smem ? sh_tab : gaK;
  const ll* bK = tab_in_smem ? sh_tab + k : gbK;
  for (ll idx = vb * blockDim.x + threadIdx.x; idx < total; idx += nvb * blockDim.x) {
    const ll s = idx / per_s;
    ll r = idx - s * per_s;
    const ll b = r / mn;
    r -= b * mn;
    const ll i = r / n, j = r - i * n;
    const T* a = Ap + slice_offset(g.sa, g0, s) + gaB[b] + gaM[i];
    const T* bb = Bp + slice_offset(g.sb, g0, s) + gbB[b] + gbN[j];
    A acc = Num<T>::zero();
    for (ll l = 0; l < k; ++l) Num<T>::fma(acc, cj(a[aK[l]], ca), cj(bb[bK[l]], cb));
    Cp[idx] = acc;
  }
}
template <class T>
__global__ void __launch_bounds__(256) k_gemm_small(GemmArgs g) {
  extern __shared__ ll sh_tab[];  // aK[0..k) then bK[0..k) when they fit
  gemm_small_body<T>(g, sh_tab, blockIdx.x, gridDim.x);
}

// Independent one-slice thin steps of one level of the step DAG, run as one launch: each block finds its
// problem by its first block, then loops exactly as k_gemm_small does (one thread per output element, k
// ascending), so every element gets the same bits as in its own launch.
constexpr int kMaxGroup = 64;
struct SmallProb {
  const void* A;
  const void* B;
  void* C;
  const ll* aB; const ll* aM; const ll* aK;
  const ll* bB; const ll* bK; const ll* bN;
  ll bt, m, k, n;
  int conj_a, conj_b;
  int block0;  // first block of this problem in the grouped grid
};
struct SmallGroup {
  int n;
  SmallProb p[kMaxGroup];
};
template <class T>
__global__ void __launch_bounds__(256) k_gemm_small_grouped(const __grid_constant__ SmallGroup g) {
  using A = typename Num<T>::acc;
  int lo = 0, hi = g.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (g.p[mid].block0 <= (int)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const SmallProb& q = g.p[lo];
  const ll nblk = (lo + 1 < g.n ? g.p[lo + 1].block0 : (int)gridDim.x) - q.block0;
  const ll blk = (ll)blockIdx.x - q.block0;
  const T* Ap = (const T*)q.A;
  const T* Bp = (const T*)q.B;
  T* Cp = (T*)q.C;
  const ll mn = q.m * q.n, total = q.bt * mn;
  extern __shared__ ll sh_tab[];  // aK[0..k) then bK[0..k); every grouped problem has k <= 1024
  for (ll l = threadIdx.x; l < q.k; l += blockDim.x) { sh_tab[l] = q.aK[l]; sh_tab[q.k + l] = q.bK[l]; }
  __syncthreads();
  const ll* aK = sh_tab;
  const ll* bK = sh_tab + q.k;
  for (ll idx = blk * blockDim.x + threadIdx.x; idx < total; idx += nblk * blockDim.x) {
    ll r = idx;
    const ll b = r / mn;
    r -= b * mn;
    const ll i = r / q.n, j = r - i * q.n;
    const T* a = Ap + q.aB[b] + q.aM[i];
    const T* bb = Bp + q.bB[b] + q.bN[j];
    A acc = Num<T>::zero();
    for (ll l = 0; l < q.k; ++l) Num<T>::fma(acc, cj(a[aK[l]], q.conj_a), cj(bb[bK[l]], q.conj_b));
    Cp[idx] = acc;
  }
}

// Few outputs with a long contraction (a dot product per slice, k up to 2^19):
// one CTA per output element, the k range strided over 256 threads and
// folded by a fixed shared-memory tree, so the sum order never varies.
template <class T>
__device__ __forceinline__ void gemm_dot_body(const GemmArgs& g, typename Num<T>::acc* red, ll vb, ll nvb) {
  using A = typename Num<T>::acc;
  const T* Ap = (const T*)g.A;
  const T* Bp = (const T*)g.B;
  T* Cp = (T*)g.C;
  const ll m = g.m, k = g.k, n = g.n, g0 = g.g0;
  const ll *gaB = g.aB, *gaM = g.aM, *gaK = g.aK, *gbB = g.bB, *gbK = g.bK, *gbN = g.bN;
  const int ca = g.conj_a, cb = g.conj_b;
  const ll mn = m * n, per_s = g.bt * mn, total = g.S * per_s;
  for (ll idx = vb; idx < total; idx += nvb) {
    const ll s = idx / per_s;
    ll r = idx - s * per_s;
    const ll b = r / mn;
    r -= b * mn;
    const ll i = r / n, j = r - i * n;
    const T* a = Ap + slice_offset(g.sa, g0, s) + gaB[b] + gaM[i];
    const T* bb = Bp + slice_offset(g.sb, g0, s) + gbB[b] + gbN[j];
    A acc = Num<T>::zero();
    for (ll l = threadIdx.x; l < k; l += 256) Num<T>::fma(acc, cj(a[gaK[l]], ca), cj(bb[gbK[l]], cb));
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) red[threadIdx.x] = Num<T>::add(red[threadIdx.x], red[threadIdx.x + w]);
      __syncthreads();
    }
    if (threadIdx.x == 0) Cp[idx] = red[0];
    __syncthreads();
  }
}
template <class T>
__global__ void __launch_bounds__(256) k_gemm_dot(GemmArgs g) {
  __shared__ typename Num<T>::acc red[256];
  gemm_dot_body<T>(g, red, blockIdx.x, gridDim.x);
}

// Long dot products split over CTAs: CTA (output o, part p) reduces k-range [p * chunk, ...) with the
// same fixed tree as k_gemm_dot and stores the widened partial at part[o * parts + p]; k_dot_reduce then
// adds each output's partials in part order in the wide type and rounds once.
template <class T>
__device__ __forceinline__ void gemm_dot_part_body(const GemmArgs& g, ll chunk, int parts, typename Num<T>::wide* part,
                                                   typename Num<T>::acc* red, ll vb, ll nvb) {
  using A = typename Num<T>::acc;
  const T* Ap = (const T*)g.A;
  const T* Bp = (const T*)g.B;
  const ll m = g.m, k = g.k, n = g.n, g0 = g.g0;
  const ll *gaB = g.aB, *gaM = g.aM, *gaK = g.aK, *gbB = g.bB, *gbK = g.bK, *gbN = g.bN;
  const int ca = g.conj_a, cb = g.conj_b;
  const ll mn = m * n, per_s = g.bt * mn, total = g.S * per_s;
  for (ll blk = vb; blk < total * parts; blk += nvb) {
    const ll idx = blk / parts, p = blk - idx * parts;
    const ll s = idx / per_s;
    ll r = idx - s * per_s;
    const ll b = r / mn;
    r -= b * mn;
    const ll i = r / n, j = r - i * n;
    const T* a = Ap + slice_offset(g.sa, g0, s) + gaB[b] + gaM[i];
    const T* bb = Bp + slice_offset(g.sb, g0, s) + gbB[b] + gbN[j];
    const ll l0 = p * chunk, l1 = l0 + chunk < k ? l0 + chunk : k;
    A acc = Num<T>::zero();
    for (ll l = l0 + threadIdx.x; l < l1; l += 256) Num<T>::fma(acc, cj(a[gaK[l]], ca), cj(bb[gbK[l]], cb));
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) red[threadIdx.x] = Num<T>::add(red[threadIdx.x], red[threadIdx.x + w]);
      __syncthreads();
    }
    if (threadIdx.x == 0) part[blk] = Num<T>::widen(red[0]);
    __syncthreads();
  }
}
template <class T>
__global__ void __launch_bounds__(256) k_gemm_dot_part(GemmArgs g, ll chunk, int parts,
                                                       typename Num<T>::wide* __restrict__ part) {
  __shared__ typename Num<T>::acc red[256];
  gemm_dot_part_body<T>(g, chunk, parts, part, red, blockIdx.x, gridDim.x);
}

template <class T>
__device__ __forceinline__ void dot_reduce_body(const typename Num<T>::wide* part, T* C, ll total, int parts, ll vb,
                                                ll nvb) {
  using W = typename Num<T>::wide;
  for (ll o = vb * blockDim.x + threadIdx.x; o < total; o += nvb * blockDim.x) {
    W acc = Num<W>::zero();
    for (int p = 0; p < parts; ++p) acc = Num<W>::add(acc, part[o * parts + p]);
    C[o] = Num<T>::narrow(acc);
  }
}
template <class T>
__global__ void k_dot_reduce(const typename Num<T>::wide* __restrict__ part, T* __restrict__ C, ll total, int parts) {
  dot_reduce_body<T>(part, C, total, parts, blockIdx.x, gridDim.x);
}

// Warp-wide butterfly reduction in a fixed order (xor 16, 8, 4, 2, 1): deterministic, lane 0 holds it.
__device__ __forceinline__ float shfl_xor(float v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
__device__ __forceinline__ double shfl_xor(double v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
__device__ __forceinline__ cf32 shfl_xor(cf32 v, int m) { return {shfl_xor(v.re, m), shfl_xor(v.im, m)}; }
__device__ __forceinline__ cf64 shfl_xor(cf64 v, int m) { return {shfl_xor(v.re, m), shfl_xor(v.im, m)}; }

// Thin steps with a moderate k (k >= 64, an output too small for a tile kernel): one warp per output,
// lanes striding over k, then a fixed butterfly.  Eight outputs per 256-thread CTA.
template <class T>
__device__ __forceinline__ void gemm_warp_body(const GemmArgs& g, ll vb, ll nvb) {
  using A = typename Num<T>::acc;
  const T* Ap = (const T*)g.A;
  const T* Bp = (const T*)g.B;
  T* Cp = (T*)g.C;
  const ll m = g.m, k = g.k, n = g.n, g0 = g.g0;
  const ll *gaB = g.aB, *gaM = g.aM, *gaK = g.aK, *gbB = g.bB, *gbK = g.bK, *gbN = g.bN;
  const int ca = g.conj_a, cb = g.conj_b;
  const int lane = threadIdx.x % 32;
  const ll mn = m * n, per_s = g.bt * mn, total = g.S * per_s;
  const ll warps = nvb * (blockDim.x / 32);
  for (ll idx = vb * (blockDim.x / 32) + threadIdx.x / 32; idx < total; idx += warps) {
    const ll s = idx / per_s;
    ll r = idx - s * per_s;
    const ll b = r / mn;
    r -= b * mn;
    const ll i = r / n, j = r - i * n;
    const T* a = Ap + slice_offset(g.sa, g0, s) + gaB[b] + gaM[i];
    const T* bb = Bp + slice_offset(g.sb, g0, s) + gbB[b] + gbN[j];
    A acc = Num<T>::zero();
    for (ll l = lane; l < k; l += 32) Num<T>::fma(acc, cj(a[gaK[l]], ca), cj(bb[gbK[l]], cb));
#pragma unroll
    for (int w = 16; w > 0; w >>= 1) acc = Num<T>::add(acc, shfl_xor(acc, w));
    if (lane == 0) Cp[idx] = acc;
  }
}
template <class T>
__global__ void __launch_bounds__(256) k_gemm_warp(GemmArgs g) {
  gemm_warp_body<T>(g, blockIdx.x, gridDim.x);
}

// Dense-enough steps on the CUDA cores: TM x TN output tile per CTA, TK-deep
// k-slabs staged through shared memory, (TM/16) x (TN/16) outputs per thread.
// This is the plain-FP32 (or FP64) form of the step GEMM.
template <class T, int TM, int TN, int TK>
__device__ __forceinline__ void gemm_tile_body(const GemmArgs& g, T (*As)[TM + 1], T (*Bs)[TN + 1], ll vb, ll nvb) {
  constexpr int RM = TM / 16, RN = TN / 16;
  const T* Ap = (const T*)g.A;
  const T* Bp = (const T*)g.B;
  T* Cp = (T*)g.C;
  const ll bt = g.bt, g0 = g.g0, m = g.m, k = g.k, n = g.n;
  const ll *gaB = g.aB, *gaM = g.aM, *gaK = g.aK, *gbB = g.bB, *gbK = g.bK, *gbN = g.bN;
  const int ca = g.conj_a, cb = g.conj_b;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const ll tiles_n = (n + TN - 1) / TN, tiles_m = (m + TM - 1) / TM;
  const ll n_tiles = tiles_n * tiles_m * g.S * bt;
  for (ll t = vb; t < n_tiles; t += nvb) {
    ll r = t;
    const ll tn = r % tiles_n; r /= tiles_n;
    const ll tm = r % tiles_m; r /= tiles_m;
    const ll sb = r, s = sb / bt, b = sb - s * bt;
    const ll i0 = tm * TM, j0 = tn * TN;
    const T* abase = Ap + slice_offset(g.sa, g0, s) + gaB[b];
    const T* bbase = Bp + slice_offset(g.sb, g0, s) + gbB[b];
    typename Num<T>::acc acc[RM][RN];
#pragma unroll
    for (int x = 0; x < RM; ++x)
#pragma unroll
      for (int y = 0; y < RN; ++y) acc[x][y] = Num<T>::zero();
    for (ll l0 = 0; l0 < k; l0 += TK) {
      for (int q = threadIdx.x; q < TM * TK; q += 256) {
        const int ii = q / TK, ll_ = q % TK;
        const ll i = i0 + ii, l = l0 + ll_;
        As[ll_][ii] = (i < m && l < k) ? cj(abase[gaM[i] + gaK[l]], ca) : Num<T>::zero();
      }
      for (int q = threadIdx.x; q < TN * TK; q += 256) {
        const int jj = q % TN, ll_ = q / TN;
        const ll j = j0 + jj, l = l0 + ll_;
        Bs[ll_][jj] = (j < n && l < k) ? cj(bbase[gbK[l] + gbN[j]], cb) : Num<T>::zero();
      }
      __syncthreads();
#pragma unroll 4
      for (int l = 0; l < TK; ++l) {
        T av[RM], bv[RN];
#pragma unroll
        for (int x = 0; x < RM; ++x) av[x] = As[l][ty + 16 * x];
#pragma unroll
        for (int y = 0; y < RN; ++y) bv[y] = Bs[l][tx + 16 * y];
#pragma unroll
        for (int x = 0; x < RM; ++x)
#pragma unroll
          for (int y = 0; y < RN; ++y) Num<T>::fma(acc[x][y], av[x], bv[y]);
      }
      __syncthreads();
    }
    T* cbase = Cp + (s * bt + b) * m * n;
#pragma unroll
    for (int x = 0; x < RM; ++x)
#pragma unroll
      for (int y = 0; y < RN; ++y) {
        const ll i = i0 + ty + 16 * x, j = j0 + tx + 16 * y;
        if (i < m && j < n) cbase[i * n + j] = acc[x][y];
      }
  }
}
template <class T, int TM, int TN, int TK>
__global__ void __launch_bounds__(256) k_gemm_tile(GemmArgs g) {
  __shared__ T As[TK][TM + 1];
  __shared__ T Bs[TK][TN + 1];
  gemm_tile_body<T, TM, TN, TK>(g, As, Bs, blockIdx.x, gridDim.x);
}

// Large real FP32 steps: a 128 x 128 output tile per CTA, 8 x 8 outputs per thread (rows ty + 16 x,
// columns tx + 16 y), K in slabs of 16 through shared memory.  Every slab, a thread loads the same eight
// rows of A at one K column and one column of B at eight K rows, so those row and column offsets stay in
// registers; four FMAs per shared-memory load instead of k_gemm_tile's two.  Each output accumulates its K
// terms in increasing order with one fmaf each, slabs zero-padded to 16, exactly as k_gemm_tile does, so
// the two give the same bits.
constexpr int kTile128 = 128;
__device__ __forceinline__ void gemm_tile128_body(const GemmArgs& g, float (*As)[kTile128 + 1],
                                                  float (*Bs)[kTile128 + 1], ll vb, ll nvb) {
  constexpr int TM = kTile128, TN = kTile128, TK = 16;
  const float* Ap = (const float*)g.A;
  const float* Bp = (const float*)g.B;
  float* Cp = (float*)g.C;
  const ll bt = g.bt, g0 = g.g0, m = g.m, k = g.k, n = g.n;
  const ll *gaB = g.aB, *gaM = g.aM, *gaK = g.aK, *gbB = g.bB, *gbK = g.bK, *gbN = g.bN;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int a_l = threadIdx.x % TK, a_i = threadIdx.x / TK;  // A: rows a_i + 16 x, K column a_l
  const int b_j = threadIdx.x % TN, b_l = threadIdx.x / TN;  // B: column b_j, K rows b_l + 2 x
  const ll tiles_n = (n + TN - 1) / TN, tiles_m = (m + TM - 1) / TM;
  const ll n_tiles = tiles_n * tiles_m * g.S * bt;
  for (ll t = vb; t < n_tiles; t += nvb) {
    ll r = t;
    const ll tn = r % tiles_n; r /= tiles_n;
    const ll tm = r % tiles_m; r /= tiles_m;
    const ll sb = r, s = sb / bt, b = sb - s * bt;
    const ll i0 = tm * TM, j0 = tn * TN;
    const float* abase = Ap + slice_offset(g.sa, g0, s) + gaB[b];
    const float* bbase = Bp + slice_offset(g.sb, g0, s) + gbB[b];
    ll aoff[8];
    unsigned amask = 0;
#pragma unroll
    for (int x = 0; x < 8; ++x) {
      const ll i = i0 + a_i + 16 * x;
      aoff[x] = i < m ? gaM[i] : 0;
      amask |= (i < m ? 1u : 0u) << x;
    }
    const ll jb = j0 + b_j;
    const bool bok = jb < n;
    const ll boff = bok ? gbN[jb] : 0;
    float acc[8][8];
#pragma unroll
    for (int x = 0; x < 8; ++x)
#pragma unroll
      for (int y = 0; y < 8; ++y) acc[x][y] = 0.f;
    for (ll l0 = 0; l0 < k; l0 += TK) {
      const ll la = l0 + a_l;
      const ll ka = la < k ? gaK[la] : 0;
#pragma unroll
      for (int x = 0; x < 8; ++x) As[a_l][a_i + 16 * x] = (la < k && ((amask >> x) & 1u)) ? abase[aoff[x] + ka] : 0.f;
#pragma unroll
      for (int x = 0; x < 8; ++x) {
        const ll lb = l0 + b_l + 2 * x;
        Bs[b_l + 2 * x][b_j] = (bok && lb < k) ? bbase[gbK[lb] + boff] : 0.f;
      }
      __syncthreads();
#pragma unroll 4
      for (int l = 0; l < TK; ++l) {
        float av[8], bv[8];
#pragma unroll
        for (int x = 0; x < 8; ++x) av[x] = As[l][ty + 16 * x];
#pragma unroll
        for (int y = 0; y < 8; ++y) bv[y] = Bs[l][tx + 16 * y];
#pragma unroll
        for (int x = 0; x < 8; ++x)
#pragma unroll
          for (int y = 0; y < 8; ++y) acc[x][y] = fmaf(av[x], bv[y], acc[x][y]);
      }
      __syncthreads();
    }
    float* cbase = Cp + (s * bt + b) * m * n;
#pragma unroll
    for (int x = 0; x < 8; ++x)
#pragma unroll
      for (int y = 0; y < 8; ++y) {
        const ll i = i0 + ty + 16 * x, j = j0 + tx + 16 * y;
        if (i < m && j < n) cbase[i * n + j] = acc[x][y];
      }
  }
}
static __global__ void __launch_bounds__(256, 2) k_gemm_tile128(GemmArgs g) {
  __shared__ float As[16][kTile128 + 1];
  __shared__ float Bs[16][kTile128 + 1];
  gemm_tile128_body(g, As, Bs, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------- cross-slice sum
// FP64 accumulation of per-slice results into chunk partials, in slice order
// within each chunk (src/slice.rs:1020-1064).  A segment is one (block, chunk)
// intersected with the current group: partial[seg.part] += sum_{s in [lo,hi)} F[s].
struct Segment { ll part, lo, hi; };  // lo/hi are local slice indices in the group

template <class T>
__device__ __forceinline__ void slice_accumulate_body(const T* F, typename Num<T>::wide* P, const Segment* segs,
                                                      ll n_segs, ll n_e, ll vb, ll nvb) {
  using W = typename Num<T>::wide;
  const ll total = n_segs * n_e;
  for (ll idx = vb * blockDim.x + threadIdx.x; idx < total; idx += nvb * blockDim.x) {
    const ll sg = idx / n_e, e = idx - sg * n_e;
    const Segment seg = segs[sg];
    W acc = P[seg.part * n_e + e];
    for (ll s = seg.lo; s < seg.hi; ++s) acc = wadd(acc, Num<T>::widen(F[s * n_e + e]));
    P[seg.part * n_e + e] = acc;
  }
}
template <class T>
__global__ void k_slice_accumulate(const T* __restrict__ F, typename Num<T>::wide* __restrict__ P,
                                   const Segment* __restrict__ segs, ll n_segs, ll n_e) {
  slice_accumulate_body<T>(F, P, segs, n_segs, n_e, blockIdx.x, gridDim.x);
}

// out[blockbase[blk] + scatter[e]] = sum_c P[blk][c][e], chunks merged in order.
template <class T, class TO>
__device__ __forceinline__ void slice_output_body(const typename Num<T>::wide* P, TO* out, const ll* block_base,
                                                  const ll* scatter, ll n_blocks, ll n_chunks, ll n_e, ll vb,
                                                  ll nvb) {
  using W = typename Num<T>::wide;
  const ll total = n_blocks * n_e;
  for (ll idx = vb * blockDim.x + threadIdx.x; idx < total; idx += nvb * blockDim.x) {
    const ll blk = idx / n_e, e = idx - blk * n_e;
    const W* p = P + blk * n_chunks * n_e + e;
    W acc = p[0];
    for (ll c = 1; c < n_chunks; ++c) acc = wadd(acc, p[c * n_e]);
    TO v;
    if constexpr (sizeof(TO) == sizeof(W)) v = *reinterpret_cast<TO*>(&acc);
    else v = Num<T>::narrow(acc);
    out[block_base[blk] + scatter[e]] = v;
  }
}
template <class T, class TO>
__global__ void k_slice_output(const typename Num<T>::wide* __restrict__ P, TO* __restrict__ out,
                               const ll* __restrict__ block_base, const ll* __restrict__ scatter, ll n_blocks,
                               ll n_chunks, ll n_e) {
  slice_output_body<T, TO>(P, out, block_base, scatter, n_blocks, n_chunks, n_e, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------- stripped execution
// max |c| over a step result (src/compiled.rs:412-421), reduced into *mx as
// the bit pattern of a non-negative double (monotone under unsigned compare).
template <class T>
__global__ void k_maxabs(const T* __restrict__ c, ll n, unsigned long long* mx) {
  double m = 0.0;
  for (ll i = (ll)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (ll)gridDim.x * blockDim.x) {
    double v = Num<T>::mag(c[i]);
    if (!(v <= m)) m = v;  // propagates NaN as a large value
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(mx, (unsigned long long)__double_as_longlong(m));
}

// Divide by the max and accumulate log10(max) (src/compiled.rs:422-429).
template <class T>
__global__ void k_strip_scale(T* __restrict__ c, ll n, const unsigned long long* mx, double* exponent, int last_block_adds) {
  const double f = __longlong_as_double((long long)*mx);
  if (!(f > 0.0) || isinf(f) || isnan(f)) return;
  const double inv = 1.0 / f;
  for (ll i = (ll)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (ll)gridDim.x * blockDim.x) c[i] = Num<T>::scale(c[i], inv);
  if (last_block_adds && blockIdx.x == 0 && threadIdx.x == 0) *exponent += log10(f);
}

// ---------------------------------------------------------------- batch interpreter descriptors
// One step of one program of a batch, as the persistent interpreter (interp.cuh) runs it: the kind's
// body with every pointer resolved, split into `nvb` tasks (virtual blocks of 256 threads).  The steps
// listed in succ[succ0 .. succ0 + nsucc) depend on it.
enum IKind : int {
  I_GATHER, I_SCATTER, I_GRAD_ACCUM, I_NARROW, I_GEMM_SMALL, I_GEMM_DOT, I_DOT_PART, I_DOT_REDUCE, I_GEMM_WARP,
  I_TILE64, I_TILE32, I_ACCUM, I_OUTPUT, I_MEMSET, I_TILE128
};
struct IOp {
  int kind;      // IKind
  int dtype;     // 0 f32, 1 f64, 2 c64, 3 c128 (DType order)
  int nvb;       // tasks of this op
  int out_wide;  // gather / slice output: store the FP64 (wide) type
  int succ0, nsucc;
  int parts;     // split dot product: number of K parts
  int pad_;
  ll chunk;      // split dot product: K per part
  const void* a;  // non-GEMM kinds: source
  void* c;        // non-GEMM kinds: destination
  void* d;        // split dot product: the partials
  const ll* t0;
  const ll* t1;
  ll n0, n1, n2, n3;  // per kind: gather (n_out, n_red, S, g0), scatter (n_in, n_red), grad_accum (n_e, -, S, g0),
                      // narrow (n), dot_reduce (total), accumulate (n_segs, n_e), output (n_blocks, n_chunks,
                      // n_e), memset (bytes)
  GemmArgs g;         // GEMM kinds; g.sa is also the slice offset of gather and grad_accum
};

}  // namespace ab2

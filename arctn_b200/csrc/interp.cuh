// Persistent batch interpreter (sm_100a): one launch runs every SIMT step of many programs.
//
// Dataflow over a ready queue.  The host gives every step (one op of one program, split into tasks =
// virtual blocks) the number of same-launch steps it waits for, and seeds the queue with the tasks of
// the steps that wait for none.  Each CTA of a persistent grid pops the next queue entry with one atomic,
// runs the step's body for that virtual block (the same __device__ body a standalone launch runs, so the
// bits are the same) and counts the task done.  The CTA that finishes a step's last task decrements the
// wait count of each dependent step and appends the tasks of those that reach zero.  Only ready tasks
// are ever queued, so a CTA waits only for an entry that a running task is about to append: the grid
// always makes progress, whatever the number of resident CTAs.  Every wait is bounded; an expired wait
// records kInterpErrCode in the error word, after which the remaining tasks skip their bodies and the
// launch drains.
#pragma once

#include <type_traits>

#include "kernels.cuh"

namespace ab2 {

constexpr int kInterpThreads = 256;
constexpr int kInterpErrCode = 16;
constexpr unsigned long long kInterpWaitNs = 2000000000ull;  // 2 s
// Dynamic shared memory of the interpreter: the largest body's need (64 x 64 complex128 tile, two
// 16 x 65 slabs); covers gemm_small's 2 x 1024 K tables and the dot product's 256-entry tree.
constexpr size_t kInterpSmem = 2 * 16 * 65 * sizeof(cf64);
static_assert(kInterpSmem >= 2 * 1024 * sizeof(ll), "gemm_small K tables");

__device__ __forceinline__ unsigned long long interp_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned long long interp_ld_acquire64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Queue entries: (step + 1, virtual block) packed in 64 bits, 0 while unwritten.
__device__ __forceinline__ unsigned long long interp_entry(int step, int vb) {
  return (unsigned long long)(unsigned)(step + 1) | ((unsigned long long)(unsigned)vb << 32);
}

// Waits until queue entry *e is written; 0 once the error word is set or kInterpWaitNs has passed.
__device__ __forceinline__ unsigned long long interp_pop_wait(const unsigned long long* e, int* err) {
  unsigned long long v = interp_ld_acquire64(e);
  if (v) return v;
  const unsigned long long t0 = interp_now();
  for (unsigned i = 1;; ++i) {
    v = interp_ld_acquire64(e);
    if (v) return v;
    if ((i & 63) == 0) {
      if (*(volatile int*)err != 0) return 0;
      if (interp_now() - t0 > kInterpWaitNs) {
        atomicCAS(err, 0, kInterpErrCode);
        return 0;
      }
    }
    __nanosleep(32);
  }
}

// The tile bodies and each dtype's dispatch are separate (not inlined) functions, so that each gets its
// own register allocation within the launch bound instead of the union of all of them.
template <class T, int TM>
__device__ __noinline__ void interp_tile(const IOp& op, unsigned char* smem, ll vb) {
  gemm_tile_body<T, TM, TM, 16>(op.g, reinterpret_cast<T(*)[TM + 1]>(smem),
                                reinterpret_cast<T(*)[TM + 1]>(smem + 16 * (TM + 1) * sizeof(T)), vb, op.nvb);
}

__device__ __noinline__ void interp_tile128(const IOp& op, unsigned char* smem, ll vb) {
  gemm_tile128_body(op.g, reinterpret_cast<float(*)[kTile128 + 1]>(smem),
                    reinterpret_cast<float(*)[kTile128 + 1]>(smem + 16 * (kTile128 + 1) * sizeof(float)), vb, op.nvb);
}

template <class T>
__device__ __noinline__ void interp_body(const IOp& op, unsigned char* smem, ll vb) {
  using W = typename Num<T>::wide;
  using A = typename Num<T>::acc;
  const ll nvb = op.nvb;
  switch (op.kind) {
    case I_GATHER:
      if (op.out_wide)
        gather_reduce_body<T, W>((const T*)op.a, (W*)op.c, op.t0, op.t1, op.n0, op.n1, op.n2, op.g.sa, op.n3, vb, nvb);
      else
        gather_reduce_body<T, T>((const T*)op.a, (T*)op.c, op.t0, op.t1, op.n0, op.n1, op.n2, op.g.sa, op.n3, vb, nvb);
      break;
    case I_SCATTER: scatter_body<T>((const T*)op.a, (T*)op.c, op.t0, op.t1, op.n0, op.n1, vb, nvb); break;
    case I_GRAD_ACCUM: grad_accum_body<T>((const T*)op.a, (W*)op.c, op.t0, op.n0, op.n2, op.g.sa, op.n3, vb, nvb); break;
    case I_NARROW: narrow_body<T>((const W*)op.a, (T*)op.c, op.n0, vb, nvb); break;
    case I_GEMM_SMALL: gemm_small_body<T>(op.g, (ll*)smem, vb, nvb); break;
    case I_GEMM_DOT: gemm_dot_body<T>(op.g, (A*)smem, vb, nvb); break;
    case I_DOT_PART: gemm_dot_part_body<T>(op.g, op.chunk, op.parts, (W*)op.d, (A*)smem, vb, nvb); break;
    case I_DOT_REDUCE: dot_reduce_body<T>((const W*)op.a, (T*)op.c, op.n0, op.parts, vb, nvb); break;
    case I_GEMM_WARP: gemm_warp_body<T>(op.g, vb, nvb); break;
    case I_TILE64: interp_tile<T, 64>(op, smem, vb); break;
    case I_TILE32: interp_tile<T, 32>(op, smem, vb); break;
    case I_TILE128:  // float32 only (the planner picks it for no other dtype)
      if constexpr (std::is_same<T, float>::value) interp_tile128(op, smem, vb);
      break;
    case I_ACCUM: slice_accumulate_body<T>((const T*)op.a, (W*)op.c, (const Segment*)op.t0, op.n0, op.n1, vb, nvb); break;
    case I_OUTPUT:
      if (op.out_wide) slice_output_body<T, W>((const W*)op.a, (W*)op.c, op.t0, op.t1, op.n0, op.n1, op.n2, vb, nvb);
      else slice_output_body<T, T>((const W*)op.a, (T*)op.c, op.t0, op.t1, op.n0, op.n1, op.n2, vb, nvb);
      break;
    case I_MEMSET: {  // 16-byte stores from a 16-byte aligned start, then the tail bytes; else bytes
      unsigned char* p = (unsigned char*)op.c;
      const ll n16 = ((uintptr_t)p & 15) == 0 ? op.n0 / 16 : 0;
      for (ll i = vb * blockDim.x + threadIdx.x; i < n16; i += nvb * blockDim.x) ((uint4*)p)[i] = make_uint4(0, 0, 0, 0);
      for (ll i = n16 * 16 + vb * blockDim.x + threadIdx.x; i < op.n0; i += nvb * blockDim.x) p[i] = 0;
      break;
    }
    default: break;
  }
}

// Runs the n_tasks tasks of one launch.  queue holds n_tasks entries, the first *tail of them (the
// tasks of the steps that wait for nothing) written by the host and the rest zero; head counts pops;
// wait[s] is the number of unfinished steps step s waits for, done[s] its finished tasks (zero).
__global__ void __launch_bounds__(kInterpThreads, 2) k_interp(const IOp* __restrict__ ops,
                                                              const int* __restrict__ succ,
                                                              unsigned long long* queue, int n_tasks, int* head,
                                                              int* tail, int* wait, int* done, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned long long s_entry;
  __shared__ int s_last;
  for (;;) {
    if (threadIdx.x == 0) {
      const int i = atomicAdd(head, 1);
      unsigned long long e = 0;
      if (i < n_tasks) {
        e = interp_pop_wait(queue + i, err);
        __threadfence();  // the body's loads come after the producers' stores
      }
      s_entry = e;
    }
    __syncthreads();
    const unsigned long long e = s_entry;
    if (e == 0) return;  // queue exhausted, or an expired wait
    const int step = (int)(e & 0xffffffffu) - 1, vb = (int)(e >> 32);
    const IOp& op = ops[step];
    const int skip = __syncthreads_or(threadIdx.x == 0 && *(volatile int*)err != 0);
    if (!skip) {
      switch (op.dtype) {
        case 0: interp_body<float>(op, smem, vb); break;
        case 1: interp_body<double>(op, smem, vb); break;
        case 2: interp_body<cf32>(op, smem, vb); break;
        case 3: interp_body<cf64>(op, smem, vb); break;
        default: break;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      s_last = atomicAdd(done + step, 1) == op.nvb - 1;
    }
    __syncthreads();
    if (s_last) {  // this CTA finished the step: release the dependents that wait for nothing else
      for (int q = threadIdx.x; q < op.nsucc; q += blockDim.x) {
        const int d = succ[op.succ0 + q];
        __threadfence();
        if (atomicSub(wait + d, 1) == 1) {
          __threadfence();
          const int nv = ops[d].nvb;
          const int base = atomicAdd(tail, nv);
          for (int v = 0; v < nv; ++v) *(volatile unsigned long long*)(queue + base + v) = interp_entry(d, v);
        }
      }
    }
  }
}

// status[j] = *errp[j] for every program j of the batch (their device error words after the run).
__global__ void k_collect_status(const int* const* __restrict__ errp, int* status, int n) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) status[j] = *errp[j];
}

}  // namespace ab2

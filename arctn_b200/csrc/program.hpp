// Device program: a compiled plan bound to slices, a dtype and a GPU.
//
// Built once on the host (all validation, slice decoding, offset tables and
// the workspace layout), then executed any number of times as a fixed
// sequence of kernel launches on the caller's stream, optionally replayed
// from a captured CUDA graph.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <set>
#include <tuple>

#include "host.hpp"
#include "kernels.cuh"

namespace ab2 {

enum : int { DT_F32 = 0, DT_F64 = 1, DT_C64 = 2, DT_C128 = 3 };
enum : int { PREC_FP32 = 0, PREC_TF32X3 = 1, PREC_BF16X3 = 2, PREC_BF16X6 = 3 };

// GEMM kernel variants a tuning table can pin per GEMM shape (the values of ARCTN_B200_GEMM_*).
enum : int {
  GV_AUTO = 0, GV_SMALL = 1, GV_TILE64 = 2, GV_TILE32 = 3, GV_WARP = 4, GV_TILE128 = 5, GV_DOT = 6,
  GV_TC_MFAST = 7, GV_TC_NFAST = 8, GV_TC_SPLITK = 9, GV_TC_STREAM = 10, GV_TC_DEEP = 11, GV_TC_PAIR = 12,
  GV_TC_PAIR_STREAM = 13, GV_COUNT = 14
};
// A GEMM's shape key: element type, precision, phase (1: slice-invariant, run once; 2: run per slice group),
// which operands vary per slice, and gemm_dims (bt, m, k, n) of one slice.
struct GemmKey {
  int dtype = 0, precision = 0, phase = 1, a_var = 0, b_var = 0;
  u64 bt = 1, m = 1, k = 1, n = 1;
  bool operator<(const GemmKey& o) const {
    return std::tie(dtype, precision, phase, a_var, b_var, bt, m, k, n) <
           std::tie(o.dtype, o.precision, o.phase, o.a_var, o.b_var, o.bt, o.m, o.k, o.n);
  }
};

size_t dtype_bytes(int dt);
const char* gemm_variant_name(int v);  // "simt_tile64", "tc_mfast", ...
inline bool dtype_complex(int dt) { return dt == DT_C64 || dt == DT_C128; }

constexpr u64 kDefaultBudget = 8ull << 30;  // workspace budget when the caller gives none

struct ProgramOptions {
  int dtype = DT_C64;
  int precision = PREC_FP32;
  int device = 0;
  bool use_graph = true;
  u64 max_slices_per_group = 0;
  u64 workspace_budget = 0;
  u64 slice_begin = 0, slice_end = 0;  // both 0: every slice
  bool gradient = false;               // also build the adjoint (reverse) sweep
  u64 tc_k_chunk = 0;                  // tf32x3: K per CTA before a split-K reduce (multiple of 16); 0: auto
  std::map<GemmKey, int> tuning;       // GEMM shape -> GV_* variant (an autotuner's table); others: heuristics
};

// Where an operand lives at run time.
struct Ref {
  enum Kind : int { NONE = 0, INPUT = 1, WS = 2, OUTPUT = 3, GRAD_OUT = 4, GRADS = 5 } kind = NONE;
  u64 index = 0;  // input / gradient index, or byte offset into the workspace
};

struct Op {
  enum Kind : int {
    GATHER = 0, GEMM_SMALL = 1, GEMM_TILE64 = 2, GEMM_TILE32 = 3, ACCUM = 4, OUTPUT = 5, MEMSET = 6, MAXABS = 7,
    STRIP = 8, GEMM_TC = 9, GEMM_DOT = 10, PACK = 11, SCATTER = 12, PACK_TILED = 13, GEMM_WARP = 14, GRAD_ACCUM = 15, NARROW = 16,
    GEMM_TILE128 = 17
  } kind;
  Ref a, b, c;
  u64 tab[6] = {0, 0, 0, 0, 0, 0};  // byte offsets of offset tables in the program's table buffer
  ll bt = 1, m = 1, k = 1, n = 1, S = 1, g0 = 0;
  SliceOff sa{}, sb{};
  ll n_out = 0, n_red = 0;  // GATHER
  ll n_segs = 0, n_e = 0, n_blocks = 0, n_chunks = 0;  // ACCUM / OUTPUT
  u64 bytes = 0;            // MEMSET
  bool out_f64 = false;     // GATHER / OUTPUT writing FP64
  // PACK: rows x cols gathered into [re|im][z][rpad][kpad]; GEMM_TC: padded operand geometry.
  ll rows = 0, cols = 0, rpad = 0, kpad = 0, rpad_b = 0;
  bool a_var = false, b_var = false;
  bool conj_a = false, conj_b = false;  // GEMM operands read conjugated (adjoint); PACK uses conj_a
  ll tile_T = 0, n_outer = 0;           // PACK_TILED: tile size and number of outer leg combinations
  int splits = 1;                       // GEMM_TC: K splits (partials in `d`, summed in order into `c`)
  int kt_chunk = 0;
  int raster = -1;                      // GEMM_TC tile order: 1 m-tiles fastest, 0 n-tiles fastest, -1 smaller side fastest
  bool stream = false;                  // GEMM_TC: the streaming-epilogue kernel (two-stage ring, double staging)
  bool deep = false;                    // GEMM_TC: the deep-ring kernel (six stages of 8 of K)
  bool pair = false;                    // GEMM_TC: the CTA-pair kernel (clusters of 2, 256 x 128 tiles)
  int chunk_mul = 1;                    // GEMM_TC: TMEM accumulation chunk in units of the format's 32 of K
  // GEMM kinds: the shape key, the variant that runs (never GV_AUTO) and whether a tuning table chose it.
  GemmKey key;
  int variant = GV_AUTO;
  bool tuned = false;
  int gemm = -1;                        // the GEMM (numbered in emit order) this op runs or serves; -1: none
  Ref d;                                // GEMM_TC: FP32 split-K partial buffer
  bool bwd = false;                     // part of the adjoint sweep (skipped by a plain execute)
  bool bf16 = false;                    // PACK / PACK_TILED / GEMM_TC / their MEMSET: split-BF16 planes
  bool six = false;                     // ... with three BF16 pieces per value (6 planes per operand)
  // PACK / GEMM_TC of a real float32 step on the complex tensor-core GEMM: K folds in half into the real and
  // imaginary parts (A' = A[:, c] + i A[:, c + Kc], B' = conj(B[c, :] + i B[c + Kc, :]), Re(A'.B') = A.B);
  // PACK: `cols` = Kc, `kfull` = K.
  bool real = false;
  ll kfull = 0;
  // GEMM_TC whose epilogue writes the next GEMM's packed operand instead of `c`: the pack buffer, the
  // offset tables over the output's rows, columns and batch, the tile's 32-float chunks and their lane
  // pattern, and the packed size of one slice.
  Ref pk;
  u64 pk_tab[5] = {0, 0, 0, 0, 0};
  int pk_qbeg[5] = {0, 0, 0, 0, 0};     // chunk ranges per 32-row group of the tile
  ll pk_slice = 0;
  bool pk_vec = false;                  // every packed chunk start is 16-byte aligned (vector stores)
  int pk_rows = 0;                      // rows a packed chunk spans (1 + its largest row offset)
};

class Program {
 public:
  Program(const Network& net, const SsaPath& path, const std::vector<Leg>& sliced, const ProgramOptions& opt);
  ~Program();
  Program(const Program&) = delete;
  Program& operator=(const Program&) = delete;

  u64 workspace_size() const { return ws_total_; }
  u64 n_slices() const { return n_total_; }
  u64 slices_per_group() const { return S_; }
  double flops() const { return flops_; }
  u64 launches() const;
  const Plan& plan() const { return plan_; }

  void execute(const void* const* inputs, void* output, bool f64_out, void* ws, u64 ws_bytes, cudaStream_t st);
  void execute_stripped(const void* const* inputs, void* output, void* ws, u64 ws_bytes, cudaStream_t st,
                        double* exponent);
  // Op-by-op run with an event between launches; per launch: ms, kind, algorithmic work.  Gradient
  // programs run forward + reverse and need grad_out / grads bound.
  void profile(const void* const* inputs, void* output, void* ws, u64 ws_bytes, cudaStream_t st, float* ms,
               int* kind, double* work, const void* grad_out = nullptr, void* const* grads = nullptr);
  // Gradient programs: part 0 = forward (keeps intermediates in ws) + reverse sweep, 1 = forward only,
  // 2 = reverse sweep only (needs the ws of a preceding part-1 run and the same inputs).
  void execute_gradient(int part, const void* const* inputs, const void* grad_out, void* const* grads, void* output,
                        void* ws, u64 ws_bytes, cudaStream_t st);
  bool has_gradient() const { return opt_.gradient; }
  // Steps whose results the adjoint sweep recomputes instead of keeping (workspace over budget).
  u64 recomputed_steps() const { return drop_.size(); }
  u64 forward_launches() const;
  u64 backward_launches() const;

  // Hooks for ProgramBatch.  part: -1 plain execute (a gradient program's forward), 0 forward +
  // reverse, 1 forward keeping intermediates, 2 reverse.  check_run validates the bindings of one run;
  // enqueue_part launches its ops on `st` without a graph and without locking (the caller holds mutex()).
  void check_run(int part, const void* const* inputs, const void* grad_out, void* const* grads,
                 const void* output) const;
  void enqueue_part(int part, const void* const* inputs, const void* grad_out, void* const* grads, void* output,
                    void* ws, cudaStream_t st);
  std::mutex& mutex() { return mu_; }
  // Uploads the offset tables if the constructor could not (no GPU at build time); needs mutex() held
  // and the program's device current, outside any stream capture.
  void ensure_tables();
  int device() const { return opt_.device; }
  int dtype() const { return opt_.dtype; }
  u64 error_offset() const { return err_off_; }
  u64 n_inputs() const { return plan_.n_inputs; }
  // JSON description of the launch sequence and workspace layout (host-only; no GPU needed).
  std::string describe() const;
  // K per TMEM accumulation chain of the split-TF32 tensor-core GEMMs (32, 64 or 128): changes launch
  // parameters only, so the next graph execute re-captures.
  void set_tc_chain(int k_per_chain);
  // Every GEMM op in launch order: its shape key, the variant it runs and whether the tuning table chose it.
  struct GemmChoice { GemmKey key; int variant; bool tuned; size_t op; };
  std::vector<GemmChoice> gemm_choices() const;

  // Hooks for the batch interpreter (interp.cuh).  Ops of the main sequence by index: whether `part`
  // runs op i, its dependencies (earlier ops touching its memory), whether the interpreter can run it
  // (every SIMT kind; not the tensor-core GEMM and its packs), its interpreter descriptors (two for a
  // split dot product: partials, then their sum) with pointers resolved against one run's bindings
  // (null bindings give the shapes and task counts only), and a standalone launch of it on `st`.
  size_t n_ops() const { return ops_.size(); }
  bool in_part(size_t i, int part) const;
  const std::vector<int>& op_deps(size_t i) const { return deps_[i]; }
  bool interp_supported(size_t i) const;
  void interp_descs(size_t i, const void* const* inputs, const void* grad_out, void* const* grads, void* output,
                    char* ws, std::vector<IOp>& out) const;
  void launch_one(size_t i, const void* const* inputs, const void* grad_out, void* const* grads, void* output,
                  char* ws, cudaStream_t st);

 private:
  // Workspace buffer with an op-index lifetime; region-2 sizes scale with the
  // group size unless `fixed` (operands shared by every slice of a group).
  struct Buf { u64 bytes, first, last; bool region2; u64 offset; bool fixed = false; };

  void build(const Network& net, const SsaPath& path, const std::vector<Leg>& sliced);
  void enqueue(const std::vector<Op>& ops, const void* const* inputs, void* output, char* ws, cudaStream_t st);
  void launch_op(const Op& op, const void* const* inputs, void* output, char* ws, cudaStream_t st);

  ProgramOptions opt_;
  Plan plan_;
  u64 n_total_ = 1, n_int_ = 1, n_blocks_ = 1, n_chunks_ = 1, S_ = 1, n_groups_ = 1;
  u64 range_begin_ = 0, range_end_ = 1;
  bool sliced_ = false;
  double flops_ = 0;
  std::vector<Op> ops_;          // full launch sequence for one execute (all groups)
  std::vector<Op> strip_ops_;    // unsliced stripped variant
  std::vector<char> host_tab_;   // offset tables, uploaded once
  char* dev_tab_ = nullptr;
  u64 ws_total_ = 0;
  u64 strip_mx_off_ = 0, strip_exp_off_ = 0;
  u64 err_off_ = 0;  // device error word (bounded-wait expiry codes), cleared by every execute

 public:
  // Synchronises `st` and returns the device error word of the last execute on `ws`.
  int device_status(void* ws, cudaStream_t st);

 private:

  size_t bwd_begin_ = 0;             // gradient programs: first op of the reverse sweep in ops_
  std::set<size_t> drop_;            // gradient programs: steps recomputed by the reverse sweep
  const void* grad_out_ = nullptr;   // bound during execute_gradient
  void* const* grads_ = nullptr;

  std::mutex mu_;
  bool out_f64_flag_ = false;

  // Graph capture as a dependency DAG over kLanes streams (plain executes of non-gradient programs).  Op j
  // depends on the last earlier op that touched any byte of its memory footprint (workspace ranges, the
  // output, gradient buffers), which orders it after every earlier op touching that memory.  Ops are
  // assigned to lanes at build time: an op continues the lane of its latest dependency where it can;
  // waits_ lists its dependencies on other lanes (an event each).
  static constexpr int kLanes = 8;
  struct Foot { int space; u64 lo, hi; };  // space 0: workspace bytes, 1: output, 2 + i: gradient i
  std::vector<std::vector<Foot>> foot_;
  std::vector<std::vector<int>> deps_;   // per op
  // Launch units in launch order: one op, or up to kMaxGroup independent one-slice thin GEMMs of one DAG
  // level run as a single grouped launch.  waits_ / lane_ / need_ev_ are per unit.
  std::vector<std::vector<int>> units_;
  std::vector<int> unit_of_;             // op -> unit
  std::vector<std::vector<int>> waits_;  // per unit: units on other lanes it waits for
  std::vector<int> lane_;
  std::vector<char> need_ev_;
  std::vector<cudaStream_t> side_;   // lanes 1 .. kLanes - 1 (lane 0 is the caller's stream)
  std::vector<cudaEvent_t> ev_;      // per op with need_ev_, recorded after it
  std::vector<cudaEvent_t> join_ev_;
  cudaEvent_t fork_ev_ = nullptr;
  void plan_dag();
  void ensure_lanes();
  void launch_group(const std::vector<int>& members, const void* const* inputs, void* output, char* ws,
                    cudaStream_t st);
  void enqueue_dag(const void* const* inputs, void* output, char* ws, cudaStream_t st);
  cudaGraphExec_t gexec_ = nullptr;
  std::vector<const void*> gkey_;
};

}  // namespace ab2

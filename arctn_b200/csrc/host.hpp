// Host-side model of ArcTN's contraction path: networks, SSA paths, metrics,
// the compiled plan, and the public planners the executor needs to produce a
// plan (greedy path, slice selection).  Pure C++17, no CUDA.
#pragma once

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

namespace ab2 {

using Leg = uint32_t;
using u64 = uint64_t;
using i64 = int64_t;

// Error carrying an ABI status code.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
enum : int { OK = 0, E_INVALID = 1, E_CUDA = 2, E_UNSUPPORTED = 3, E_TIMEOUT = 4, E_WORKSPACE = 5 };
[[noreturn]] inline void fail(const std::string& m) { throw Error(E_INVALID, m); }

using SsaPath = std::vector<std::pair<u64, u64>>;

// TensorNetwork (src/network.rs:134-143).  Leg dimensions live in an ordered
// map so every iteration over legs is deterministic.
struct Network {
  std::vector<std::vector<Leg>> inputs;
  std::vector<Leg> output;
  std::map<Leg, u64> size;

  u64 dim(Leg l) const {
    auto it = size.find(l);
    if (it == size.end()) fail("leg " + std::to_string(l) + " has no size_dict dimension");
    return it->second;
  }
  double log2_dim(Leg l) const;
  size_t n_tensors() const { return inputs.size(); }
  // src/network.rs:171-229
  void validate() const;
};

// Element count with zero-axis and overflow rejection (src/tensor.rs:11-22).
u64 checked_numel(const std::vector<u64>& shape);
// Scalar-independent GEMM geometry checks (src/contract.rs:49-100).
void check_gemm_geometry(u64 bt, u64 m, u64 k, u64 n);

struct PathStats {
  double log10_flops, log2_max_size, log2_max_contraction_size, log2_total_size, log2_read_write, log2_peak_size;
};
// simulate_path_full (src/path.rs:239-434); optionally returns each step's result legs.
PathStats simulate_path(const Network& net, const SsaPath& path, std::vector<std::vector<Leg>>* step_legs = nullptr);

// greedy (src/paths/greedy.rs:307-320): costmod 1, zero temperature, one branch.
SsaPath greedy_path(const Network& net);
// find_slices_to_size (src/slice.rs:209-215); false where the reference returns None.  allow_output: output
// legs may be chosen too (find_slices_until_for_target_with_output_slicing, src/slice.rs:254-289).
bool find_slices_to_size(const Network& net, const SsaPath& path, u64 target, std::vector<Leg>& legs_out,
                         bool allow_output = false);
// src/slice.rs:893-905
u64 slice_parallel_chunks(u64 n_slices, u64 out_numel);
// src/slice.rs:152-176: uniqueness, presence and no repetition inside one input.
void validate_slice_legs(const Network& net, const std::vector<Leg>& sliced);
// Every intermediate of `path` holds at most `target` elements (src/slice.rs:102-111).
bool path_fits_target_size(const Network& net, const SsaPath& path, u64 target);
// Per-slice metrics: the path on the network with every sliced leg set to 1 (src/execution_plan.rs:879-890).
PathStats sliced_path_stats(const Network& net, const SsaPath& path, const std::vector<Leg>& sliced);
// The same audit with the sliced legs removed first (src/slice.rs:114-130).
bool slice_result_fits_target_size(const Network& net, const SsaPath& path, const std::vector<Leg>& sliced,
                                   u64 target);

// ---------------------------------------------------------------- compiled plan
// CompiledInputPrep (src/compiled.rs:33-75)
struct InputPrep {
  std::vector<u64> input_shape;
  std::vector<u64> traces;  // flattened (ax_i, ax_j, is_diag) triples
  std::vector<Leg> legs;
  std::vector<u64> shape;
  bool identity() const { return traces.empty(); }
};

// CompiledPairContraction (src/compiled.rs:77-172)
struct PairStep {
  u64 left_slot, right_slot, result_slot;
  std::vector<Leg> left_legs, right_legs, result_legs;
  std::vector<u64> left_shape, right_shape, result_shape;
  std::vector<u64> sum_a, sum_b, a_perm, b_perm;
  u64 bt, m, k, n;
  // Number of legs in each GEMM group (batch, free_a, con, free_b).
  size_t n_batch, n_free_a, n_con, n_free_b;
};

// CompiledFinalize (src/compiled.rs:174-219)
struct Finalize {
  u64 slot;
  std::vector<Leg> input_legs;
  std::vector<u64> input_shape, sum, perm, output_shape;
  bool identity() const;
};

struct Plan {
  u64 n_inputs = 0;
  std::vector<InputPrep> preps;
  std::vector<PairStep> steps;
  Finalize fin;
  double log10_flops = 0, log2_peak_size = 0;
};

// CompiledContraction::compile (src/compiled.rs:254-366)
Plan compile_plan(const Network& net, const SsaPath& path);

// Per-input trace/diagonal plan (src/compiled.rs:445-478) for arbitrary leg
// lists; `external(l)` decides diagonal (kept) versus trace (removed).
template <class F>
std::vector<u64> plan_traces(std::vector<Leg>& legs, F&& external) {
  std::vector<u64> ops;
  for (;;) {
    size_t fi = 0, fj = 0;
    bool hit = false;
    for (size_t i = 0; i < legs.size() && !hit; ++i)
      for (size_t j = i + 1; j < legs.size(); ++j)
        if (legs[i] == legs[j]) { fi = i; fj = j; hit = true; break; }
    if (!hit) return ops;
    Leg l = legs[fi];
    size_t cnt = 0;
    for (Leg x : legs) cnt += (x == l);
    if (cnt > 2) fail("leg " + std::to_string(l) + " appears more than twice in one tensor");
    bool diag = external(l);
    ops.push_back(fi);
    ops.push_back(fj);
    ops.push_back(diag ? 1 : 0);
    legs.erase(legs.begin() + fj);
    if (!diag) legs.erase(legs.begin() + fi);
  }
}

inline std::vector<u64> row_major_strides(const std::vector<u64>& shape) {
  std::vector<u64> s(shape.size(), 1);
  for (size_t i = shape.size(); i-- > 1;) s[i - 1] = s[i] * shape[i];
  return s;
}

}  // namespace ab2

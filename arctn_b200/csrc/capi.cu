// extern "C" boundary of the executor (declared in include/arctn_b200.h).
//
// Stage-level calls (one prep, one pair step, finalize) are served by small
// cached programs over a one- or two-tensor network that reproduces exactly
// that stage: a pair step is the contraction of its two operand leg lists
// with the step's result legs as output, which classifies every leg the same
// way plan_pairwise does (src/compiled.rs:481-602).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>

#include "../../include/arctn_b200.h"
#include "batch.hpp"
#include "program.hpp"

using namespace ab2;

static thread_local std::string g_last_error;

namespace ab2 {
// Lets other translation units of the library report through arctn_b200_last_error().
void set_last_error(const std::string& m) { g_last_error = m; }
}  // namespace ab2

struct arctn_b200_plan {
  Network net;
  SsaPath path;
  Plan plan;
  std::mutex mu;
  std::map<std::tuple<int, u64, int, int, int>, std::unique_ptr<Program>> stages;
};

struct arctn_b200_program {
  std::unique_ptr<Program> p;
};
struct arctn_b200_batch {
  std::unique_ptr<ProgramBatch> b;
};

namespace {

template <class F>
int guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return ARCTN_B200_OK;
  } catch (Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return ARCTN_B200_ERR_INVALID;
  } catch (std::exception& e) {
    g_last_error = e.what();
    return ARCTN_B200_ERR_INVALID;
  }
}

// Host-side fault injection for tests of the error paths.  A test arms a countdown per site; the armed call
// fails at its entry, before any CUDA work, with the status and message of a failed CUDA allocation.  Nothing
// reaches the GPU.  Site 0: program and batch execute / gradient calls; site 1: program and batch creation.
std::atomic<int> g_inject[2];

void maybe_inject(int site) {
  int c = g_inject[site].load();
  while (c > 0) {
    if (g_inject[site].compare_exchange_weak(c, c - 1)) {
      if (c == 1)
        throw Error(E_CUDA, "cudaErrorMemoryAllocation: out of memory (injected by arctn_b200_debug_inject_failure, "
                            "site " + std::to_string(site) + ")");
      return;
    }
  }
}

Network to_network(const arctn_b200_network* n) {
  if (!n) fail("network is null");
  Network net;
  if (n->n_inputs && (!n->input_offsets)) fail("input_offsets is null");
  for (u64 i = 0; i < n->n_inputs; ++i) {
    u64 a = n->input_offsets[i], b = n->input_offsets[i + 1];
    if (b < a) fail("input_offsets must be non-decreasing");
    if (b > a && !n->input_legs) fail("input_legs is null");
    net.inputs.emplace_back(n->input_legs + a, n->input_legs + b);
  }
  if (n->n_output && !n->output) fail("output is null");
  net.output.assign(n->output, n->output + n->n_output);
  if (n->n_sizes && (!n->size_legs || !n->size_dims)) fail("size_dict arrays are null");
  for (u64 j = 0; j < n->n_sizes; ++j) {
    if (!net.size.emplace(n->size_legs[j], n->size_dims[j]).second)
      fail("size_dict lists leg " + std::to_string(n->size_legs[j]) + " twice");
  }
  return net;
}

SsaPath to_path(u64 n_steps, const u64* ssa) {
  if (n_steps && !ssa) fail("ssa_path is null");
  SsaPath p;
  for (u64 s = 0; s < n_steps; ++s) p.push_back({ssa[2 * s], ssa[2 * s + 1]});
  return p;
}

ProgramOptions to_options(const arctn_b200_program_options* o) {
  ProgramOptions po;
  if (o) {
    po.dtype = o->dtype;
    po.precision = o->precision;
    po.device = o->device;
    po.use_graph = o->use_graph != 0;
    po.max_slices_per_group = o->max_slices_per_group;
    po.workspace_budget = o->workspace_budget;
    po.slice_begin = o->slice_begin;
    po.slice_end = o->slice_end;
    po.gradient = o->gradient != 0;
    po.tc_k_chunk = o->tc_k_chunk;
  }
  return po;
}

// Stage kinds for the cache key.
enum { STAGE_PREP = 0, STAGE_STEP = 1, STAGE_FIN = 2 };

Program& stage_program(arctn_b200_plan* pl, int kind, u64 idx, int dtype, int precision) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) throw Error(E_CUDA, "cudaGetDevice failed");
  auto key = std::make_tuple(kind, idx, dtype, precision, dev);
  std::lock_guard<std::mutex> lk(pl->mu);
  auto it = pl->stages.find(key);
  if (it != pl->stages.end()) return *it->second;
  Network n;
  SsaPath path;
  if (kind == STAGE_PREP) {
    if (idx >= pl->plan.n_inputs) fail("input index out of range");
    n.inputs = {pl->net.inputs[idx]};
    n.output = pl->plan.preps[idx].legs;
  } else if (kind == STAGE_STEP) {
    if (idx >= pl->plan.steps.size()) fail("step index out of range");
    const PairStep& st = pl->plan.steps[idx];
    n.inputs = {st.left_legs, st.right_legs};
    n.output = st.result_legs;
    path = {{0, 1}};
  } else {
    n.inputs = {pl->plan.fin.input_legs};
    n.output = pl->net.output;
  }
  for (auto& t : n.inputs)
    for (Leg l : t) n.size[l] = pl->net.dim(l);
  ProgramOptions po;
  po.dtype = dtype;
  po.precision = precision;
  po.device = dev;
  po.use_graph = false;
  auto prog = std::make_unique<Program>(n, path, std::vector<Leg>{}, po);
  Program& ref = *prog;
  pl->stages.emplace(key, std::move(prog));
  return ref;
}

}  // namespace

extern "C" {

uint32_t arctn_b200_abi_version(void) { return ARCTN_B200_ABI_VERSION; }

int arctn_b200_debug_inject_failure(int site, int countdown) {
  return guarded([&] {
    if (site < 0 || site > 1) fail("site must be 0 (execute / gradient) or 1 (create)");
    if (countdown < 0) fail("countdown must be >= 0");
    g_inject[site].store(countdown);
  });
}
const char* arctn_b200_last_error(void) { return g_last_error.c_str(); }

int arctn_b200_simulate_path(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path, double stats_out[6]) {
  return guarded([&] {
    PathStats s = simulate_path(to_network(net), to_path(n_steps, ssa_path));
    double v[6] = {s.log10_flops, s.log2_max_size, s.log2_max_contraction_size, s.log2_total_size, s.log2_read_write, s.log2_peak_size};
    for (int i = 0; i < 6; ++i) stats_out[i] = v[i];
  });
}

int arctn_b200_greedy(const arctn_b200_network* net, uint64_t* ssa_out, uint64_t* n_steps_out) {
  return guarded([&] {
    SsaPath p = greedy_path(to_network(net));
    for (size_t s = 0; s < p.size(); ++s) { ssa_out[2 * s] = p[s].first; ssa_out[2 * s + 1] = p[s].second; }
    *n_steps_out = p.size();
  });
}

int arctn_b200_find_slices_to_size(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                                   uint64_t target_size, uint32_t* legs_out, uint64_t* n_legs_out, int* found) {
  return guarded([&] {
    std::vector<Leg> legs;
    bool ok = find_slices_to_size(to_network(net), to_path(n_steps, ssa_path), target_size, legs);
    *found = ok ? 1 : 0;
    *n_legs_out = legs.size();
    for (size_t i = 0; i < legs.size(); ++i) legs_out[i] = legs[i];
  });
}

int arctn_b200_find_slices_with_output(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                                       uint64_t target_size, int allow_output_slicing, uint32_t* legs_out,
                                       uint64_t* n_legs_out, int* found) {
  return guarded([&] {
    std::vector<Leg> legs;
    bool ok = find_slices_to_size(to_network(net), to_path(n_steps, ssa_path), target_size, legs,
                                  allow_output_slicing != 0);
    *found = ok ? 1 : 0;
    *n_legs_out = legs.size();
    for (size_t i = 0; i < legs.size(); ++i) legs_out[i] = legs[i];
  });
}

int arctn_b200_slice_plan_check(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                                uint64_t n_sliced, const uint32_t* sliced_legs, uint64_t target_size,
                                double per_slice_stats_out[6], int* fits_out) {
  return guarded([&] {
    if (n_sliced && !sliced_legs) fail("sliced_legs is null");
    const Network n = to_network(net);
    const SsaPath p = to_path(n_steps, ssa_path);
    const std::vector<Leg> sl(sliced_legs, sliced_legs + n_sliced);
    const PathStats s = sliced_path_stats(n, p, sl);
    if (per_slice_stats_out) {
      const double v[6] = {s.log10_flops, s.log2_max_size, s.log2_max_contraction_size, s.log2_total_size,
                           s.log2_read_write, s.log2_peak_size};
      for (int i = 0; i < 6; ++i) per_slice_stats_out[i] = v[i];
    }
    if (fits_out) *fits_out = target_size ? (slice_result_fits_target_size(n, p, sl, target_size) ? 1 : 0) : 1;
  });
}

uint64_t arctn_b200_slice_parallel_chunks(uint64_t n_slices, uint64_t out_numel) {
  return slice_parallel_chunks(n_slices, out_numel);
}

int arctn_b200_plan_compile(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                            arctn_b200_plan** plan_out) {
  return guarded([&] {
    if (!plan_out) fail("plan_out is null");
    auto pl = std::make_unique<arctn_b200_plan>();
    pl->net = to_network(net);
    pl->path = to_path(n_steps, ssa_path);
    pl->plan = compile_plan(pl->net, pl->path);
    *plan_out = pl.release();
  });
}

void arctn_b200_plan_destroy(arctn_b200_plan* plan) { delete plan; }

uint64_t arctn_b200_plan_n_inputs(const arctn_b200_plan* p) { return p ? p->plan.n_inputs : 0; }
uint64_t arctn_b200_plan_n_steps(const arctn_b200_plan* p) { return p ? p->plan.steps.size() : 0; }
double arctn_b200_plan_log10_flops(const arctn_b200_plan* p) { return p ? p->plan.log10_flops : 0.0; }
double arctn_b200_plan_log2_peak_size(const arctn_b200_plan* p) { return p ? p->plan.log2_peak_size : 0.0; }

int arctn_b200_plan_step_info(const arctn_b200_plan* p, uint64_t step, arctn_b200_step_info* o) {
  return guarded([&] {
    if (!p || !o) fail("null argument");
    if (step >= p->plan.steps.size()) fail("step index out of range");
    const PairStep& s = p->plan.steps[step];
    o->left_slot = s.left_slot;
    o->right_slot = s.right_slot;
    o->result_slot = s.result_slot;
    o->n_left = s.left_legs.size();
    o->n_right = s.right_legs.size();
    o->n_result = s.result_legs.size();
    o->left_legs = s.left_legs.data();
    o->right_legs = s.right_legs.data();
    o->result_legs = s.result_legs.data();
    o->left_shape = s.left_shape.data();
    o->right_shape = s.right_shape.data();
    o->result_shape = s.result_shape.data();
    o->n_sum_a = s.sum_a.size();
    o->n_sum_b = s.sum_b.size();
    o->sum_a = s.sum_a.data();
    o->sum_b = s.sum_b.data();
    o->a_perm = s.a_perm.data();
    o->b_perm = s.b_perm.data();
    o->bt = s.bt;
    o->m = s.m;
    o->k = s.k;
    o->n = s.n;
  });
}

int arctn_b200_plan_prep_info(const arctn_b200_plan* p, uint64_t input, arctn_b200_prep_info* o) {
  return guarded([&] {
    if (!p || !o) fail("null argument");
    if (input >= p->plan.preps.size()) fail("input index out of range");
    const InputPrep& r = p->plan.preps[input];
    o->n_input_shape = r.input_shape.size();
    o->input_shape = r.input_shape.data();
    o->n_traces = r.traces.size() / 3;
    o->traces = r.traces.data();
    o->n_legs = r.legs.size();
    o->legs = r.legs.data();
    o->shape = r.shape.data();
  });
}

int arctn_b200_plan_finalize_info(const arctn_b200_plan* p, arctn_b200_finalize_info* o) {
  return guarded([&] {
    if (!p || !o) fail("null argument");
    const Finalize& f = p->plan.fin;
    o->slot = f.slot;
    o->n_input = f.input_legs.size();
    o->input_legs = f.input_legs.data();
    o->input_shape = f.input_shape.data();
    o->n_sum = f.sum.size();
    o->sum = f.sum.data();
    o->n_output = f.perm.size();
    o->perm = f.perm.data();
    o->output_shape = f.output_shape.data();
  });
}

static uint64_t stage_ws(const arctn_b200_plan* p, int kind, u64 idx, int dtype, int precision) {
  uint64_t out = 0;
  int rc = guarded([&] {
    if (!p) fail("plan is null");
    out = stage_program(const_cast<arctn_b200_plan*>(p), kind, idx, dtype, precision).workspace_size();
  });
  return rc == ARCTN_B200_OK ? out : UINT64_MAX;
}

uint64_t arctn_b200_plan_prep_workspace_size(const arctn_b200_plan* p, int dtype, uint64_t input) {
  return stage_ws(p, STAGE_PREP, input, dtype, ARCTN_B200_PREC_FP32);
}
uint64_t arctn_b200_plan_step_workspace_size(const arctn_b200_plan* p, int dtype, int precision, uint64_t step) {
  return stage_ws(p, STAGE_STEP, step, dtype, precision);
}
uint64_t arctn_b200_plan_finalize_workspace_size(const arctn_b200_plan* p, int dtype) {
  return stage_ws(p, STAGE_FIN, 0, dtype, ARCTN_B200_PREC_FP32);
}

static int run_stage(const arctn_b200_plan* p, int kind, u64 idx, int dtype, int precision, const void* const* ins,
                     void* out, void* ws, u64 ws_bytes, void* stream) {
  return guarded([&] {
    if (!p) fail("plan is null");
    Program& prog = stage_program(const_cast<arctn_b200_plan*>(p), kind, idx, dtype, precision);
    prog.execute(ins, out, false, ws, ws_bytes, (cudaStream_t)stream);
  });
}

int arctn_b200_plan_prep_execute(const arctn_b200_plan* p, int dtype, uint64_t input, const void* in, void* out,
                                 void* workspace, uint64_t workspace_bytes, void* cuda_stream) {
  const void* ins[1] = {in};
  return run_stage(p, STAGE_PREP, input, dtype, ARCTN_B200_PREC_FP32, ins, out, workspace, workspace_bytes, cuda_stream);
}

int arctn_b200_plan_step_execute(const arctn_b200_plan* p, int dtype, int precision, uint64_t step, const void* left,
                                 const void* right, void* out, void* workspace, uint64_t workspace_bytes,
                                 void* cuda_stream) {
  const void* ins[2] = {left, right};
  return run_stage(p, STAGE_STEP, step, dtype, precision, ins, out, workspace, workspace_bytes, cuda_stream);
}

int arctn_b200_plan_finalize_execute(const arctn_b200_plan* p, int dtype, const void* in, void* out, void* workspace,
                                     uint64_t workspace_bytes, void* cuda_stream) {
  const void* ins[1] = {in};
  return run_stage(p, STAGE_FIN, 0, dtype, ARCTN_B200_PREC_FP32, ins, out, workspace, workspace_bytes, cuda_stream);
}

int arctn_b200_program_create(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                              uint64_t n_sliced, const uint32_t* sliced_legs, const arctn_b200_program_options* options,
                              arctn_b200_program** program_out) {
  return guarded([&] {
    maybe_inject(1);
    if (!program_out) fail("program_out is null");
    if (n_sliced && !sliced_legs) fail("sliced_legs is null");
    std::vector<Leg> sl(sliced_legs, sliced_legs + n_sliced);
    auto h = std::make_unique<arctn_b200_program>();
    h->p = std::make_unique<Program>(to_network(net), to_path(n_steps, ssa_path), sl, to_options(options));
    *program_out = h.release();
  });
}

int arctn_b200_program_create_tuned(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                                    uint64_t n_sliced, const uint32_t* sliced_legs,
                                    const arctn_b200_program_options* options, const arctn_b200_gemm_choice* table,
                                    uint64_t n_table, arctn_b200_program** program_out) {
  return guarded([&] {
    maybe_inject(1);
    if (!program_out) fail("program_out is null");
    if (n_sliced && !sliced_legs) fail("sliced_legs is null");
    if (n_table && !table) fail("table is null");
    std::vector<Leg> sl(sliced_legs, sliced_legs + n_sliced);
    ProgramOptions po = to_options(options);
    for (u64 i = 0; i < n_table; ++i) {
      const arctn_b200_gemm_choice& e = table[i];
      if (e.variant < ARCTN_B200_GEMM_AUTO || e.variant > ARCTN_B200_GEMM_TC_PAIR_STREAM)
        fail("tuning entry " + std::to_string(i) + ": unknown variant " + std::to_string(e.variant));
      if (e.phase != 1 && e.phase != 2) fail("tuning entry " + std::to_string(i) + ": phase must be 1 or 2");
      GemmKey k{e.dtype, e.precision, e.phase, e.a_var ? 1 : 0, e.b_var ? 1 : 0, e.bt, e.m, e.k, e.n};
      po.tuning[k] = e.variant;
    }
    auto h = std::make_unique<arctn_b200_program>();
    h->p = std::make_unique<Program>(to_network(net), to_path(n_steps, ssa_path), sl, po);
    *program_out = h.release();
  });
}

int arctn_b200_program_set_tc_chain(arctn_b200_program* p, uint64_t k_per_chain) {
  return guarded([&] {
    if (!p) fail("null argument");
    p->p->set_tc_chain((int)std::min<uint64_t>(k_per_chain, 1u << 20));
  });
}

int arctn_b200_program_gemms(const arctn_b200_program* p, arctn_b200_gemm_choice* out, int* tuned_out, uint64_t cap,
                             uint64_t* n_out) {
  return guarded([&] {
    if (!p || !n_out) fail("null argument");
    const auto v = p->p->gemm_choices();
    *n_out = v.size();
    if (cap && !out) fail("out is null");
    for (size_t i = 0; i < v.size() && i < cap; ++i) {
      const GemmKey& k = v[i].key;
      out[i] = arctn_b200_gemm_choice{k.dtype, k.precision, k.phase, k.a_var, k.b_var, v[i].variant,
                                      k.bt, k.m, k.k, k.n};
      if (tuned_out) tuned_out[i] = v[i].tuned ? 1 : 0;
    }
  });
}

void arctn_b200_program_destroy(arctn_b200_program* program) { delete program; }

uint64_t arctn_b200_program_workspace_size(const arctn_b200_program* p) { return p ? p->p->workspace_size() : 0; }
uint64_t arctn_b200_program_n_slices(const arctn_b200_program* p) { return p ? p->p->n_slices() : 0; }
uint64_t arctn_b200_program_slices_per_group(const arctn_b200_program* p) { return p ? p->p->slices_per_group() : 0; }
double arctn_b200_program_flops(const arctn_b200_program* p) { return p ? p->p->flops() : 0.0; }
uint64_t arctn_b200_program_launches(const arctn_b200_program* p) { return p ? p->p->launches() : 0; }
uint64_t arctn_b200_program_recomputed_steps(const arctn_b200_program* p) {
  return p ? p->p->recomputed_steps() : 0;
}

int arctn_b200_program_execute(arctn_b200_program* p, const void* const* inputs, void* output, void* workspace,
                               uint64_t workspace_bytes, void* cuda_stream) {
  return guarded([&] {
    maybe_inject(0);
    if (!p || !inputs) fail("null argument");
    p->p->execute(inputs, output, false, workspace, workspace_bytes, (cudaStream_t)cuda_stream);
  });
}

int arctn_b200_program_execute_f64out(arctn_b200_program* p, const void* const* inputs, void* output_f64,
                                      void* workspace, uint64_t workspace_bytes, void* cuda_stream) {
  return guarded([&] {
    maybe_inject(0);
    if (!p || !inputs) fail("null argument");
    p->p->execute(inputs, output_f64, true, workspace, workspace_bytes, (cudaStream_t)cuda_stream);
  });
}

int arctn_b200_program_execute_stripped(arctn_b200_program* p, const void* const* inputs, void* output,
                                        void* workspace, uint64_t workspace_bytes, void* cuda_stream,
                                        double* log10_exponent) {
  return guarded([&] {
    maybe_inject(0);
    if (!p || !inputs || !log10_exponent) fail("null argument");
    p->p->execute_stripped(inputs, output, workspace, workspace_bytes, (cudaStream_t)cuda_stream, log10_exponent);
  });
}

int arctn_b200_program_gradient(arctn_b200_program* p, int part, const void* const* inputs, const void* grad_output,
                                void* const* grad_inputs, void* output, void* workspace, uint64_t workspace_bytes,
                                void* cuda_stream) {
  return guarded([&] {
    maybe_inject(0);
    if (!p || !inputs) fail("null argument");
    if (part < 0 || part > 2) fail("part must be 0, 1 or 2");
    p->p->execute_gradient(part, inputs, grad_output, grad_inputs, output, workspace, workspace_bytes,
                           (cudaStream_t)cuda_stream);
  });
}

int arctn_b200_program_describe(const arctn_b200_program* p, char* buf, uint64_t buf_bytes, uint64_t* needed) {
  return guarded([&] {
    if (!p) fail("program is null");
    const std::string d = p->p->describe();
    if (needed) *needed = d.size() + 1;
    if (buf && buf_bytes) {
      const size_t n = std::min<size_t>(d.size(), buf_bytes - 1);
      std::memcpy(buf, d.data(), n);
      buf[n] = 0;
    }
  });
}

int arctn_b200_batch_create_mode(arctn_b200_program* const* programs, uint64_t n_programs, int max_lanes, int mode,
                                 arctn_b200_batch** batch_out) {
  return guarded([&] {
    maybe_inject(1);
    if (!programs || !batch_out) fail("null argument");
    std::vector<Program*> ps;
    for (uint64_t j = 0; j < n_programs; ++j) {
      if (!programs[j]) fail("program " + std::to_string(j) + " is null");
      ps.push_back(programs[j]->p.get());
    }
    auto h = std::make_unique<arctn_b200_batch>();
    h->b = std::make_unique<ProgramBatch>(std::move(ps), max_lanes, mode);
    *batch_out = h.release();
  });
}

int arctn_b200_batch_create(arctn_b200_program* const* programs, uint64_t n_programs, int max_lanes,
                            arctn_b200_batch** batch_out) {
  return arctn_b200_batch_create_mode(programs, n_programs, max_lanes, ARCTN_B200_BATCH_PERSISTENT, batch_out);
}

int arctn_b200_batch_wait_selftest(void* cuda_stream, int* code) {
  return guarded([&] {
    if (!code) fail("null argument");
    *code = interp_wait_selftest((cudaStream_t)cuda_stream);
  });
}

int arctn_b200_batch_describe(const arctn_b200_batch* batch, int detail, char* buf, uint64_t buf_bytes,
                              uint64_t* needed) {
  return guarded([&] {
    if (!batch) fail("batch is null");
    const std::string d = batch->b->describe(detail);
    if (needed) *needed = d.size() + 1;
    if (buf && buf_bytes) {
      const size_t n = std::min<size_t>(d.size(), (size_t)buf_bytes - 1);
      std::memcpy(buf, d.data(), n);
      buf[n] = 0;
    }
  });
}

void arctn_b200_batch_destroy(arctn_b200_batch* batch) { delete batch; }
uint64_t arctn_b200_batch_workspace_size(const arctn_b200_batch* b) { return b ? b->b->workspace_size() : 0; }
uint64_t arctn_b200_batch_lanes(const arctn_b200_batch* b) { return b ? b->b->n_lanes() : 0; }

int arctn_b200_batch_execute(arctn_b200_batch* batch, const void* const* const* inputs, void* const* outputs,
                             void* workspace, uint64_t workspace_bytes, void* cuda_stream) {
  return guarded([&] {
    maybe_inject(0);
    if (!batch) fail("batch is null");
    batch->b->run(-1, inputs, nullptr, nullptr, outputs, workspace, workspace_bytes, (cudaStream_t)cuda_stream);
  });
}

int arctn_b200_batch_gradient(arctn_b200_batch* batch, const void* const* const* inputs,
                              const void* const* grad_outputs, void* const* const* grads, void* const* outputs,
                              void* workspace, uint64_t workspace_bytes, void* cuda_stream) {
  return guarded([&] {
    maybe_inject(0);
    if (!batch) fail("batch is null");
    batch->b->run(0, inputs, grad_outputs, grads, outputs, workspace, workspace_bytes, (cudaStream_t)cuda_stream);
  });
}

int arctn_b200_batch_device_status(arctn_b200_batch* batch, void* workspace, void* cuda_stream, int* code) {
  int c = 0;
  int rc = guarded([&] {
    if (!batch || !workspace || !code) fail("null argument");
    c = batch->b->device_status(workspace, (cudaStream_t)cuda_stream);
    *code = c;
  });
  if (rc == ARCTN_B200_OK && c != 0) {
    g_last_error = "a bounded device-side wait expired (code " + std::to_string(c) + ")";
    return ARCTN_B200_ERR_DEVICE_TIMEOUT;
  }
  return rc;
}

int arctn_b200_program_device_status(arctn_b200_program* p, void* workspace, void* cuda_stream, int* code) {
  int c = 0;
  int rc = guarded([&] {
    if (!p || !workspace || !code) fail("null argument");
    c = p->p->device_status(workspace, (cudaStream_t)cuda_stream);
    *code = c;
  });
  if (rc == ARCTN_B200_OK && c != 0) {
    g_last_error = "a bounded device-side wait expired (code " + std::to_string(c) + ")";
    return ARCTN_B200_ERR_DEVICE_TIMEOUT;
  }
  return rc;
}

int arctn_b200_program_profile(arctn_b200_program* p, const void* const* inputs, void* output, void* workspace,
                               uint64_t workspace_bytes, void* cuda_stream, float* ms_out, int* kind_out,
                               double* work_out) {
  return guarded([&] {
    if (!p || !inputs || !ms_out || !kind_out || !work_out) fail("null argument");
    p->p->profile(inputs, output, workspace, workspace_bytes, (cudaStream_t)cuda_stream, ms_out, kind_out, work_out);
  });
}

int arctn_b200_program_profile_gradient(arctn_b200_program* p, const void* const* inputs, const void* grad_output,
                                        void* const* grads, void* output, void* workspace, uint64_t workspace_bytes,
                                        void* cuda_stream, float* ms_out, int* kind_out, double* work_out) {
  return guarded([&] {
    if (!p || !inputs || !ms_out || !kind_out || !work_out) fail("null argument");
    if (!p->p->has_gradient()) fail("the program was built without gradient support");
    p->p->profile(inputs, output, workspace, workspace_bytes, (cudaStream_t)cuda_stream, ms_out, kind_out, work_out,
                  grad_output, grads);
  });
}

int arctn_b200_contract_sliced_host(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                                    uint64_t n_sliced, const uint32_t* sliced_legs,
                                    const arctn_b200_program_options* options, const void* const* host_inputs,
                                    void* host_output) {
  return guarded([&] {
    Network n = to_network(net);
    std::vector<Leg> sl(sliced_legs, sliced_legs + n_sliced);
    ProgramOptions po = to_options(options);
    po.use_graph = false;
    Program prog(n, to_path(n_steps, ssa_path), sl, po);
    const size_t eb = dtype_bytes(po.dtype);
    std::vector<void*> dev(n.n_tensors(), nullptr);
    void* d_out = nullptr;
    void* d_ws = nullptr;
    auto cleanup = [&] {
      for (void* d : dev) if (d) cudaFree(d);
      if (d_out) cudaFree(d_out);
      if (d_ws) cudaFree(d_ws);
    };
    try {
      for (size_t i = 0; i < n.n_tensors(); ++i) {
        std::vector<u64> shape;
        for (Leg l : n.inputs[i]) shape.push_back(n.dim(l));
        size_t bytes = checked_numel(shape) * eb;
        if (cudaMalloc(&dev[i], bytes) != cudaSuccess) throw Error(E_CUDA, "cudaMalloc failed for an input");
        if (cudaMemcpy(dev[i], host_inputs[i], bytes, cudaMemcpyHostToDevice) != cudaSuccess) throw Error(E_CUDA, "input copy failed");
      }
      std::vector<u64> oshape;
      for (Leg l : n.output) oshape.push_back(n.dim(l));
      size_t obytes = checked_numel(oshape) * eb;
      if (cudaMalloc(&d_out, obytes) != cudaSuccess) throw Error(E_CUDA, "cudaMalloc failed for the output");
      if (prog.workspace_size() && cudaMalloc(&d_ws, prog.workspace_size()) != cudaSuccess) throw Error(E_CUDA, "cudaMalloc failed for the workspace");
      prog.execute(dev.data(), d_out, false, d_ws, prog.workspace_size(), nullptr);
      if (cudaMemcpy(host_output, d_out, obytes, cudaMemcpyDeviceToHost) != cudaSuccess) throw Error(E_CUDA, "output copy failed");
    } catch (...) {
      cleanup();
      throw;
    }
    cleanup();
  });
}

}  // extern "C"

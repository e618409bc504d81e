// ProgramBatch: independent programs as one graph launch (see batch.hpp).
#include "batch.hpp"

#include <algorithm>
#include <map>
#include <numeric>
#include <set>
#include <string>
#include <tuple>

#include "interp.cuh"

namespace ab2 {

namespace {

#define BCK(x)                                                                                    \
  do {                                                                                            \
    cudaError_t e_ = (x);                                                                         \
    if (e_ != cudaSuccess) throw Error(E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr u64 kLaneAlign = 256;
// Nominal costs for the lane assignment only: a sustained complex GEMM rate and a per-launch cost.
constexpr double kNominalFlops = 1.0e14;
constexpr double kNominalLaunch = 4.0e-6;
// Programs up to this many flops per forward pass run inside the interpreter (when all their steps can).
constexpr double kInterpMaxFlops = 5.0e8;

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DevGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

u64 align_lane(u64 b) { return (b + kLaneAlign - 1) / kLaneAlign * kLaneAlign; }

}  // namespace

ProgramBatch::ProgramBatch(std::vector<Program*> programs, int max_lanes, int mode)
    : progs_(std::move(programs)), mode_(mode) {
  if (progs_.empty()) throw Error(E_INVALID, "a batch needs at least one program");
  if (max_lanes < 1 || max_lanes > 128) throw Error(E_INVALID, "max_lanes must be in [1, 128]");
  if (mode != LANES && mode != PERSISTENT && mode != STAGED)
    throw Error(E_INVALID, "batch mode must be 0 (lanes), 1 (persistent) or 2 (staged)");
  for (size_t j = 0; j < progs_.size(); ++j) {
    if (!progs_[j]) throw Error(E_INVALID, "program " + std::to_string(j) + " is null");
    if (progs_[j]->device() != progs_[0]->device())
      throw Error(E_INVALID, "every program of a batch must be bound to the same device");
  }
  device_ = progs_[0]->device();
  // Longest processing time first onto the least loaded lane.
  std::vector<double> cost(progs_.size());
  for (size_t j = 0; j < progs_.size(); ++j)
    cost[j] = progs_[j]->flops() / kNominalFlops + (double)progs_[j]->launches() * kNominalLaunch;
  std::vector<size_t> order(progs_.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
  const size_t n_lanes = std::min<size_t>((size_t)max_lanes, progs_.size());
  lanes_.assign(n_lanes, {});
  lane_of_.assign(progs_.size(), 0);
  std::vector<double> load(n_lanes, 0.0);
  for (size_t j : order) {
    const size_t l = std::min_element(load.begin(), load.end()) - load.begin();
    lanes_[l].push_back(j);
    lane_of_[j] = (int)l;
    load[l] += cost[j];
  }
  // The interpreter takes the programs made of SIMT steps only whose work is small; the others (tensor-core
  // steps, or large SIMT GEMMs that run best as full-occupancy launches) run launch by launch on the lane
  // streams at the same time, again longest first onto the least-loaded lane.
  interp_.assign(progs_.size(), 0);
  side_lanes_.assign(n_lanes, {});
  if (mode_ != LANES) {
    std::vector<double> side_load(n_lanes, 0.0);
    for (size_t j : order) {
      const Program* P = progs_[j];
      bool ok = mode_ == STAGED;
      if (!ok) {
        ok = P->flops() <= kInterpMaxFlops;
        for (size_t i = 0; ok && i < P->n_ops(); ++i) ok = P->interp_supported(i);
      }
      interp_[j] = ok;
      if (!ok) {
        const size_t l = std::min_element(side_load.begin(), side_load.end()) - side_load.begin();
        side_lanes_[l].push_back(j);
        side_load[l] += cost[j];
      }
    }
  }
  prog_off_.assign(progs_.size(), 0);
  u64 off = 0;
  if (mode_ != LANES) {  // one region per program: the interpreter interleaves them all
    for (size_t j = 0; j < progs_.size(); ++j) {
      prog_off_[j] = off;
      off += align_lane(progs_[j]->workspace_size());
    }
  } else {
    for (auto& lane : lanes_) {
      u64 need = 0;
      for (size_t j : lane) need = std::max<u64>(need, progs_[j]->workspace_size());
      for (size_t j : lane) prog_off_[j] = off;
      off += align_lane(need);
    }
  }
  status_off_ = off;
  u64 words = progs_.size() + 1, queue = 0;  // program error words, the interpreter's error word
  if (mode_ != LANES) {
    bool all_grad = true;
    for (Program* p : progs_) all_grad = all_grad && p->has_gradient();
    plan_slot(0);
    if (all_grad) plan_slot(1);
    for (const Slot& sl : slot_)
      if (sl.valid) {
        words = std::max<u64>(words, progs_.size() + sl.ctr0.size());
        queue = std::max<u64>(queue, sl.n_tasks);
      }
  }
  queue_off_ = off + align_lane(words * sizeof(int));
  ws_total_ = queue_off_ + align_lane(queue * sizeof(unsigned long long));
}

ProgramBatch::~ProgramBatch() {
  DevGuard g(device_);
  for (auto& ge : gexec_)
    if (ge) cudaGraphExecDestroy(ge);
  for (auto s : streams_) cudaStreamDestroy(s);
  for (auto e : join_) cudaEventDestroy(e);
  if (fork_) cudaEventDestroy(fork_);
  for (Slot& sl : slot_) {
    if (sl.d_ops) cudaFree(sl.d_ops);
    if (sl.d_succ) cudaFree(sl.d_succ);
    if (sl.d_ctr0) cudaFree(sl.d_ctr0);
    if (sl.d_queue0) cudaFree(sl.d_queue0);
    if (sl.d_errp) cudaFree(sl.d_errp);
    if (sl.used) cudaEventDestroy(sl.used);
  }
}

void ProgramBatch::ensure_streams() {
  if (fork_) return;
  BCK(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
  for (size_t l = 0; l < lanes_.size(); ++l) {
    cudaStream_t s;
    BCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    streams_.push_back(s);
    cudaEvent_t e;
    BCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    join_.push_back(e);
  }
  int occ = 0, sms = 0;
  BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_interp, kInterpThreads, kInterpSmem));
  BCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
  // With lane programs running alongside, one CTA an SM leaves the rest of every SM to their kernels.
  bool side = false;
  for (const auto& l : side_lanes_) side = side || !l.empty();
  grid_ = (side ? 1 : std::max(1, occ)) * std::max(1, sms);
}

// Stages and queue order.  An op the interpreter cannot run (tensor-core GEMM, pack) at stage t is
// launched before interpreter launch t; an interpreter op runs in launch t.  So an interpreter op's stage
// is the largest stage among its dependencies, and an external op's stage is one past that of its
// interpreter dependencies (its external dependencies of the same stage run before it on its lane).
// Interpreter ops are queued by (stage, level within the stage's DAG, program, op): a topological order
// in which the programs' ready steps interleave.
void ProgramBatch::plan_slot(int s) {
  Slot& sl = slot_[s];
  sl = Slot{};
  sl.part = s == 0 ? -1 : 0;
  struct Entry { int stage, level, prog, op; };
  std::vector<Entry> entries;
  std::vector<std::vector<int>> stage(progs_.size()), level(progs_.size());
  int n_stages = 1;
  std::vector<std::vector<std::vector<int>>> deps(progs_.size());  // per program and op, within the part
  for (size_t j = 0; j < progs_.size(); ++j) {
    if (!interp_[j]) continue;
    const Program* P = progs_[j];
    const size_t n = P->n_ops();
    stage[j].assign(n, -1);
    level[j].assign(n, 0);
    // A dependency outside the part (a sliced gradient program's reverse step, for part -1) is replaced by
    // its own dependencies: they touched the same memory last before it.
    deps[j].assign(n, {});
    for (size_t i = 0; i < n; ++i) {
      std::set<int> d;
      for (int x : P->op_deps(i)) {
        if (P->in_part((size_t)x, sl.part)) d.insert(x);
        else d.insert(deps[j][(size_t)x].begin(), deps[j][(size_t)x].end());
      }
      deps[j][i].assign(d.begin(), d.end());
    }
    for (size_t i = 0; i < n; ++i) {
      if (!P->in_part(i, sl.part)) continue;
      const bool ext = !P->interp_supported(i);
      int st = 0, lv = 0;
      for (int d : deps[j][i]) {
        const bool dext = !P->interp_supported((size_t)d);
        st = std::max(st, stage[j][(size_t)d] + (ext && !dext ? 1 : 0));
      }
      if (!ext)
        for (int d : deps[j][i])
          if (P->interp_supported((size_t)d) && stage[j][(size_t)d] == st) lv = std::max(lv, level[j][(size_t)d] + 1);
      stage[j][i] = st;
      level[j][i] = lv;
      n_stages = std::max(n_stages, st + 1);
      if (ext) {
        if ((int)sl.ext.size() <= st) sl.ext.resize((size_t)st + 1);
        sl.ext[(size_t)st].push_back({(int)j, (int)i});
      } else {
        entries.push_back(Entry{st, lv, (int)j, (int)i});
      }
    }
  }
  sl.n_stages = n_stages;
  sl.ext.resize((size_t)n_stages);
  std::stable_sort(entries.begin(), entries.end(), [](const Entry& x, const Entry& y) {
    return std::tie(x.stage, x.level, x.prog, x.op) < std::tie(y.stage, y.level, y.prog, y.op);
  });
  std::vector<std::map<int, int>> last(progs_.size());  // op -> its last interpreter step
  std::vector<IOp> tmp;
  for (const Entry& e : entries) {
    tmp.clear();
    progs_[(size_t)e.prog]->interp_descs((size_t)e.op, nullptr, nullptr, nullptr, nullptr, nullptr, tmp);
    for (size_t k = 0; k < tmp.size(); ++k) {
      const int idx = (int)sl.iops.size();
      std::vector<int> wait;
      if (k == 0) {
        std::set<int> seen;
        for (int dd : deps[(size_t)e.prog][(size_t)e.op]) {
          if (!progs_[(size_t)e.prog]->interp_supported((size_t)dd) || stage[(size_t)e.prog][(size_t)dd] != e.stage)
            continue;  // an earlier launch (stage boundary) orders it
          if (seen.insert(last[(size_t)e.prog].at(dd)).second) wait.push_back(last[(size_t)e.prog].at(dd));
        }
      } else {
        wait.push_back(idx - 1);  // the sum waits for its partials
      }
      sl.iops.push_back(tmp[k]);
      sl.deps.push_back(wait);
      sl.src.push_back({e.prog, e.op});
      sl.sub.push_back((int)k);
      sl.stage.push_back(e.stage);
      sl.level.push_back(e.level);
    }
    last[(size_t)e.prog][e.op] = (int)sl.iops.size() - 1;
  }
  // Dependents (CSR through IOp::succ0 / nsucc), launch-time counters and the seeded queue.
  const size_t N = sl.iops.size(), T = (size_t)n_stages;
  std::vector<std::vector<int>> succ(N);
  for (size_t q = 0; q < N; ++q)
    for (int d : sl.deps[q]) succ[(size_t)d].push_back((int)q);
  for (size_t q = 0; q < N; ++q) {
    sl.iops[q].succ0 = (int)sl.succ.size();
    sl.iops[q].nsucc = (int)succ[q].size();
    sl.succ.insert(sl.succ.end(), succ[q].begin(), succ[q].end());
  }
  sl.ctr0.assign(1 + 2 * T + 2 * N, 0);  // [error word][heads][tails][wait counts][done counts]
  sl.stage_begin.assign(T + 1, 0);
  size_t q = 0;
  for (size_t t = 0; t < T; ++t) {
    sl.stage_begin[t] = (int)sl.n_tasks;
    const size_t q0 = q;
    u64 roots = 0;
    for (; q < N && sl.stage[q] == (int)t; ++q) {
      sl.ctr0[1 + 2 * T + q] = (int)sl.deps[q].size();
      sl.n_tasks += (u64)sl.iops[q].nvb;
      if (sl.deps[q].empty()) roots += (u64)sl.iops[q].nvb;
    }
    sl.queue0.resize(sl.n_tasks, 0ull);
    u64 w = sl.stage_begin[t];
    for (size_t r = q0; r < q; ++r)
      if (sl.deps[r].empty())
        for (int vb = 0; vb < sl.iops[r].nvb; ++vb)
          sl.queue0[w++] = (unsigned long long)(unsigned)(r + 1) | ((unsigned long long)(unsigned)vb << 32);
    sl.ctr0[1 + T + t] = (int)roots;
  }
  sl.stage_begin[T] = (int)sl.n_tasks;
  if (sl.n_tasks > 0x7FFFFFFFull || N > 0x7FFFFFFEull)
    throw Error(E_UNSUPPORTED, "batch interpreter queue exceeds 2^31 tasks");
  sl.valid = true;
}

// Descriptors with this run's pointers, uploaded to the slot's device tables.  The tables are rewritten
// only after every earlier launch that reads them has finished.
void ProgramBatch::bind_slot(int s, const void* const* const* inputs, const void* const* grad_outs,
                             void* const* const* grads, void* const* outputs, char* ws) {
  Slot& sl = slot_[s];
  std::vector<IOp> tmp;
  for (size_t q = 0; q < sl.iops.size();) {
    const int j = sl.src[q].first, i = sl.src[q].second;
    tmp.clear();
    progs_[(size_t)j]->interp_descs((size_t)i, inputs[j], sl.part == 0 ? grad_outs[j] : nullptr,
                                    sl.part == 0 ? grads[j] : nullptr, outputs[j], ws + prog_off_[(size_t)j], tmp);
    for (size_t k = 0; k < tmp.size(); ++k, ++q) {
      IOp d = tmp[k];
      d.succ0 = sl.iops[q].succ0;
      d.nsucc = sl.iops[q].nsucc;
      sl.iops[q] = d;
    }
  }
  std::vector<int*> errp(progs_.size());
  for (size_t j = 0; j < progs_.size(); ++j) errp[j] = (int*)(ws + prog_off_[j] + progs_[j]->error_offset());
  if (!sl.d_ops) {
    BCK(cudaMalloc(&sl.d_ops, std::max<size_t>(1, sl.iops.size()) * sizeof(IOp)));
    BCK(cudaMalloc(&sl.d_succ, std::max<size_t>(1, sl.succ.size()) * sizeof(int)));
    BCK(cudaMalloc(&sl.d_ctr0, sl.ctr0.size() * sizeof(int)));
    BCK(cudaMalloc(&sl.d_queue0, std::max<size_t>(1, sl.queue0.size()) * sizeof(unsigned long long)));
    BCK(cudaMalloc(&sl.d_errp, progs_.size() * sizeof(int*)));
    BCK(cudaEventCreateWithFlags(&sl.used, cudaEventDisableTiming));
    BCK(cudaMemcpy(sl.d_succ, sl.succ.data(), sl.succ.size() * sizeof(int), cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(sl.d_ctr0, sl.ctr0.data(), sl.ctr0.size() * sizeof(int), cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(sl.d_queue0, sl.queue0.data(), sl.queue0.size() * sizeof(unsigned long long),
                   cudaMemcpyHostToDevice));
  }
  if (sl.launched) BCK(cudaEventSynchronize(sl.used));
  BCK(cudaMemcpy(sl.d_ops, sl.iops.data(), sl.iops.size() * sizeof(IOp), cudaMemcpyHostToDevice));
  BCK(cudaMemcpy(sl.d_errp, errp.data(), errp.size() * sizeof(int*), cudaMemcpyHostToDevice));
}

void ProgramBatch::enqueue_persistent(int s, const void* const* const* inputs, const void* const* grad_outs,
                                      void* const* const* grads, void* const* outputs, char* ws, cudaStream_t st) {
  Slot& sl = slot_[s];
  const size_t n = progs_.size(), T = (size_t)sl.n_stages, N = sl.iops.size();
  int* status = (int*)(ws + status_off_);
  int* err = status + n;
  int* heads = err + 1;
  int* tails = heads + T;
  int* wait = tails + T;
  int* done = wait + N;
  unsigned long long* queue = (unsigned long long*)(ws + queue_off_);
  // The lane programs, on the lane streams alongside the interpreter.
  std::vector<char> side(lanes_.size(), 0);
  BCK(cudaEventRecord(fork_, st));
  for (size_t l = 0; l < side_lanes_.size(); ++l) {
    if (side_lanes_[l].empty()) continue;
    side[l] = 1;
    BCK(cudaStreamWaitEvent(streams_[l], fork_, 0));
    for (size_t j : side_lanes_[l])
      progs_[j]->enqueue_part(sl.part, inputs[j], sl.part == 0 ? grad_outs[j] : nullptr,
                              sl.part == 0 ? grads[j] : nullptr, outputs[j], ws + prog_off_[j], streams_[l]);
  }
  BCK(cudaMemcpyAsync(err, sl.d_ctr0, sl.ctr0.size() * sizeof(int), cudaMemcpyDeviceToDevice, st));
  if (sl.n_tasks)
    BCK(cudaMemcpyAsync(queue, sl.d_queue0, sl.n_tasks * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st));
  std::vector<char> used(lanes_.size());
  for (int t = 0; t < sl.n_stages; ++t) {
    if (!sl.ext[(size_t)t].empty()) {
      BCK(cudaEventRecord(fork_, st));
      std::fill(used.begin(), used.end(), 0);
      for (const auto& e : sl.ext[(size_t)t]) {
        const size_t j = (size_t)e.first;
        const int l = lane_of_[j];
        if (!used[(size_t)l]) {
          BCK(cudaStreamWaitEvent(streams_[(size_t)l], fork_, 0));
          used[(size_t)l] = 1;
        }
        progs_[j]->launch_one((size_t)e.second, inputs[j], sl.part == 0 ? grad_outs[j] : nullptr,
                              sl.part == 0 ? grads[j] : nullptr, outputs[j], ws + prog_off_[j], streams_[(size_t)l]);
      }
      for (size_t l = 0; l < lanes_.size(); ++l)
        if (used[l]) {
          BCK(cudaEventRecord(join_[l], streams_[l]));
          BCK(cudaStreamWaitEvent(st, join_[l], 0));
        }
    }
    const int b = sl.stage_begin[(size_t)t], e = sl.stage_begin[(size_t)t + 1];
    if (e > b) {
      k_interp<<<std::min(grid_, e - b), kInterpThreads, kInterpSmem, st>>>(sl.d_ops, sl.d_succ, queue + b, e - b,
                                                                           heads + t, tails + t, wait, done, err);
      BCK(cudaGetLastError());
    }
  }
  for (size_t l = 0; l < side.size(); ++l)
    if (side[l]) {
      BCK(cudaEventRecord(join_[l], streams_[l]));
      BCK(cudaStreamWaitEvent(st, join_[l], 0));
    }
  k_collect_status<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(sl.d_errp, status, (int)n);
  BCK(cudaGetLastError());
}

void ProgramBatch::enqueue(int part, const void* const* const* inputs, const void* const* grad_outs,
                           void* const* const* grads, void* const* outputs, char* ws, cudaStream_t st) {
  BCK(cudaMemsetAsync(ws + status_off_ + progs_.size() * sizeof(int), 0, sizeof(int), st));  // interpreter word
  BCK(cudaEventRecord(fork_, st));
  for (size_t l = 0; l < lanes_.size(); ++l) {
    BCK(cudaStreamWaitEvent(streams_[l], fork_, 0));
    for (size_t j : lanes_[l]) {
      progs_[j]->enqueue_part(part, inputs[j], part == 0 ? grad_outs[j] : nullptr, part == 0 ? grads[j] : nullptr,
                              outputs[j], ws + prog_off_[j], streams_[l]);
      BCK(cudaMemcpyAsync(ws + status_off_ + j * sizeof(int), ws + prog_off_[j] + progs_[j]->error_offset(),
                          sizeof(int), cudaMemcpyDeviceToDevice, streams_[l]));
    }
    BCK(cudaEventRecord(join_[l], streams_[l]));
    BCK(cudaStreamWaitEvent(st, join_[l], 0));
  }
}

void ProgramBatch::run(int part, const void* const* const* inputs, const void* const* grad_outs,
                       void* const* const* grads, void* const* outputs, void* ws, u64 ws_bytes, cudaStream_t st) {
  if (part != -1 && part != 0) throw Error(E_INVALID, "a batch runs part -1 (execute) or 0 (forward + reverse)");
  if (!inputs || !outputs) throw Error(E_INVALID, "inputs / outputs arrays are null");
  if (part == 0 && (!grad_outs || !grads)) throw Error(E_INVALID, "grad_outputs / grads arrays are null");
  if (ws_bytes < ws_total_)
    throw Error(E_WORKSPACE, "workspace of " + std::to_string(ws_bytes) + " bytes is smaller than the required " +
                                 std::to_string(ws_total_));
  if (ws_total_ && !ws) throw Error(E_INVALID, "workspace pointer is null");
  for (size_t j = 0; j < progs_.size(); ++j)
    progs_[j]->check_run(part, inputs[j], part == 0 ? grad_outs[j] : nullptr, part == 0 ? grads[j] : nullptr,
                         outputs[j]);
  DevGuard g(device_);
  std::lock_guard<std::mutex> lk(mu_);
  ensure_streams();
  // Lock every program (address order) so no other call interleaves with the captured sequence.
  std::vector<Program*> locked(progs_);
  std::sort(locked.begin(), locked.end());
  locked.erase(std::unique(locked.begin(), locked.end()), locked.end());
  std::vector<std::unique_lock<std::mutex>> locks;
  for (Program* p : locked) locks.emplace_back(p->mutex());
  for (Program* p : locked) p->ensure_tables();

  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (st) BCK(cudaStreamIsCapturing(st, &cs));
  if (!st || cs != cudaStreamCaptureStatusNone) {  // legacy stream, or inside the caller's capture
    enqueue(part, inputs, grad_outs, grads, outputs, (char*)ws, st);
    return;
  }
  const int slot = part == 0 ? 1 : 0;
  const bool interp = mode_ != LANES && slot_[slot].valid;
  std::vector<const void*> key;
  key.push_back(ws);
  for (size_t j = 0; j < progs_.size(); ++j) {
    const u64 n = progs_[j]->n_inputs();
    key.insert(key.end(), inputs[j], inputs[j] + n);
    key.push_back(outputs[j]);
    if (part == 0) {
      key.push_back(grad_outs[j]);
      key.insert(key.end(), grads[j], grads[j] + n);
    }
  }
  if (!gexec_[slot] || key != gkey_[slot]) {
    if (interp) bind_slot(slot, inputs, grad_outs, grads, outputs, (char*)ws);
    cudaGraph_t graph = nullptr;
    BCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      if (interp) enqueue_persistent(slot, inputs, grad_outs, grads, outputs, (char*)ws, st);
      else enqueue(part, inputs, grad_outs, grads, outputs, (char*)ws, st);
    } catch (...) {
      cudaStreamEndCapture(st, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    BCK(cudaStreamEndCapture(st, &graph));
    bool updated = false;
    if (gexec_[slot]) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(gexec_[slot], graph, &info) == cudaSuccess) updated = true;
      else {
        cudaGetLastError();
        cudaGraphExecDestroy(gexec_[slot]);
        gexec_[slot] = nullptr;
      }
    }
    if (!updated) {
      const cudaError_t e = cudaGraphInstantiate(&gexec_[slot], graph, 0);
      if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        gexec_[slot] = nullptr;
        throw Error(E_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      }
    }
    cudaGraphDestroy(graph);
    gkey_[slot] = key;
  }
  BCK(cudaGraphLaunch(gexec_[slot], st));
  if (interp) {
    BCK(cudaEventRecord(slot_[slot].used, st));
    slot_[slot].launched = true;
  }
}

int ProgramBatch::device_status(void* ws, cudaStream_t st) {
  DevGuard g(device_);
  std::vector<int> codes(progs_.size() + 1, 0);
  BCK(cudaMemcpyAsync(codes.data(), (char*)ws + status_off_, codes.size() * sizeof(int), cudaMemcpyDeviceToHost,
                      st));
  BCK(cudaStreamSynchronize(st));
  for (int c : codes)
    if (c) return c;
  return 0;
}

std::string ProgramBatch::describe(int detail) const {
  std::string s = "{\"mode\":\"" + std::string(mode_ == PERSISTENT ? "persistent" : mode_ == STAGED ? "staged" : "lanes") +
                  "\",\"programs\":" + std::to_string(progs_.size()) + ",\"lanes\":" + std::to_string(lanes_.size()) +
                  ",\"workspace_bytes\":" + std::to_string(ws_total_) + ",\"interpreted\":[";
  bool fi = true;
  for (size_t j = 0; j < interp_.size(); ++j)
    if (interp_[j]) {
      s += (fi ? "" : ",") + std::to_string(j);
      fi = false;
    }
  s += "],\"program_offsets\":[";
  for (size_t j = 0; j < prog_off_.size(); ++j) s += (j ? "," : "") + std::to_string(prog_off_[j]);
  s += "],\"parts\":[";
  bool first = true;
  for (const Slot& sl : slot_) {
    if (!sl.valid) continue;
    s += std::string(first ? "" : ",") + "{\"part\":" + std::to_string(sl.part) +
         ",\"stages\":" + std::to_string(sl.n_stages) + ",\"steps\":" + std::to_string(sl.iops.size()) +
         ",\"tasks\":" + std::to_string(sl.n_tasks) + ",\"stage_tasks\":[";
    first = false;
    for (int t = 0; t < sl.n_stages; ++t)
      s += (t ? "," : "") + std::to_string(sl.stage_begin[(size_t)t + 1] - sl.stage_begin[(size_t)t]);
    s += "],\"stage_launches\":[";
    for (int t = 0; t < sl.n_stages; ++t) s += (t ? "," : "") + std::to_string(sl.ext[(size_t)t].size());
    s += "]";
    if (detail) {
      s += ",\"step_list\":[";  // [program, op, sub, stage, level, tasks, [deps]]
      for (size_t q = 0; q < sl.iops.size(); ++q) {
        const IOp& d = sl.iops[q];
        s += std::string(q ? "," : "") + "[" + std::to_string(sl.src[q].first) + "," +
             std::to_string(sl.src[q].second) + "," + std::to_string(sl.sub[q]) + "," + std::to_string(sl.stage[q]) +
             "," + std::to_string(sl.level[q]) + "," + std::to_string(d.nvb) + ",[";
        for (size_t k = 0; k < sl.deps[q].size(); ++k) s += (k ? "," : "") + std::to_string(sl.deps[q][k]);
        s += "]]";
      }
      s += "],\"staged_launches\":[";  // [stage, program, op]
      bool f2 = true;
      for (int t = 0; t < sl.n_stages; ++t)
        for (const auto& e : sl.ext[(size_t)t]) {
          s += std::string(f2 ? "" : ",") + "[" + std::to_string(t) + "," + std::to_string(e.first) + "," +
               std::to_string(e.second) + "]";
          f2 = false;
        }
      s += "]";
    }
    s += "}";
  }
  return s + "]}";
}

int interp_wait_selftest(cudaStream_t st) {
  // Two queue entries of which only the first is ever written: the pop of the second must wait, expire,
  // record kInterpErrCode and end the launch.
  static_assert(sizeof(IOp) <= 1024, "one descriptor fits its slot of the scratch buffer");
  char* buf = nullptr;
  BCK(cudaMalloc(&buf, 4096));
  int code = -1;
  try {
    IOp op{};
    op.kind = I_MEMSET;
    op.nvb = 1;
    op.c = buf + 3584;
    op.n0 = 16;
    const unsigned long long entries[2] = {1ull, 0ull};  // (step 0, block 0); never written
    const int ctr[5] = {0, 0, 1, 0, 0};                  // error word, head, tail, wait[0], done[0]
    int* c = (int*)(buf + 2048);
    unsigned long long* queue = (unsigned long long*)(buf + 3072);
    BCK(cudaMemcpyAsync(buf, &op, sizeof(IOp), cudaMemcpyHostToDevice, st));
    BCK(cudaMemcpyAsync(c, ctr, sizeof(ctr), cudaMemcpyHostToDevice, st));
    BCK(cudaMemcpyAsync(queue, entries, sizeof(entries), cudaMemcpyHostToDevice, st));
    k_interp<<<1, kInterpThreads, kInterpSmem, st>>>((const IOp*)buf, (const int*)(buf + 1024), queue, 2, c + 1,
                                                     c + 2, c + 3, c + 4, c);
    BCK(cudaGetLastError());
    BCK(cudaMemcpyAsync(&code, c, sizeof(int), cudaMemcpyDeviceToHost, st));
    BCK(cudaStreamSynchronize(st));
  } catch (...) {
    cudaFree(buf);
    throw;
  }
  BCK(cudaFree(buf));
  return code;
}

}  // namespace ab2

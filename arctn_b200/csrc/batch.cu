// ProgramBatch: independent programs as one graph launch (see batch.hpp).
#include "batch.hpp"

#include <algorithm>
#include <numeric>
#include <string>

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

}  // namespace

ProgramBatch::ProgramBatch(std::vector<Program*> programs, int max_lanes) : progs_(std::move(programs)) {
  if (progs_.empty()) throw Error(E_INVALID, "a batch needs at least one program");
  if (max_lanes < 1 || max_lanes > 128) throw Error(E_INVALID, "max_lanes must be in [1, 128]");
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
  std::vector<double> load(n_lanes, 0.0);
  for (size_t j : order) {
    const size_t l = std::min_element(load.begin(), load.end()) - load.begin();
    lanes_[l].push_back(j);
    load[l] += cost[j];
  }
  prog_off_.assign(progs_.size(), 0);
  u64 off = 0;
  for (auto& lane : lanes_) {
    u64 need = 0;
    for (size_t j : lane) need = std::max<u64>(need, progs_[j]->workspace_size());
    lane_off_.push_back(off);
    for (size_t j : lane) prog_off_[j] = off;
    off += (need + kLaneAlign - 1) / kLaneAlign * kLaneAlign;
  }
  status_off_ = off;  // one int per program: its device error word, copied out after it runs
  ws_total_ = off + (progs_.size() * sizeof(int) + kLaneAlign - 1) / kLaneAlign * kLaneAlign;
  DevGuard g(device_);
  BCK(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
  for (size_t l = 0; l < n_lanes; ++l) {
    cudaStream_t s;
    BCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    streams_.push_back(s);
    cudaEvent_t e;
    BCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    join_.push_back(e);
  }
}

ProgramBatch::~ProgramBatch() {
  DevGuard g(device_);
  for (auto& ge : gexec_)
    if (ge) cudaGraphExecDestroy(ge);
  for (auto s : streams_) cudaStreamDestroy(s);
  for (auto e : join_) cudaEventDestroy(e);
  if (fork_) cudaEventDestroy(fork_);
}

void ProgramBatch::enqueue(int part, const void* const* const* inputs, const void* const* grad_outs,
                           void* const* const* grads, void* const* outputs, char* ws, cudaStream_t st) {
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
  const int slot = part == 0 ? 1 : 0;
  if (!gexec_[slot] || key != gkey_[slot]) {
    cudaGraph_t graph = nullptr;
    BCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue(part, inputs, grad_outs, grads, outputs, (char*)ws, st);
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
}

int ProgramBatch::device_status(void* ws, cudaStream_t st) {
  DevGuard g(device_);
  std::vector<int> codes(progs_.size(), 0);
  BCK(cudaMemcpyAsync(codes.data(), (char*)ws + status_off_, codes.size() * sizeof(int), cudaMemcpyDeviceToHost,
                      st));
  BCK(cudaStreamSynchronize(st));
  for (int c : codes)
    if (c) return c;
  return 0;
}

}  // namespace ab2

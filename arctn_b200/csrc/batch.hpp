// Many independent programs (uneven networks, mixed dtypes) run as one CUDA graph launch.
//
// The programs are spread over up to `max_lanes` streams by longest-processing-time first (estimated
// time = flops at a nominal rate + launches x a nominal launch cost).  Each lane runs its programs one
// after another in one workspace region sized for the largest of them; the lanes fork from the
// caller's stream and join back into it, so small networks overlap on the GPU.  The fork/join launch
// sequence is captured once per set of bound pointers and replayed as a graph.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "program.hpp"

namespace ab2 {

class ProgramBatch {
 public:
  ProgramBatch(std::vector<Program*> programs, int max_lanes);
  ~ProgramBatch();
  ProgramBatch(const ProgramBatch&) = delete;
  ProgramBatch& operator=(const ProgramBatch&) = delete;

  u64 workspace_size() const { return ws_total_; }
  u64 n_lanes() const { return lanes_.size(); }
  u64 size() const { return progs_.size(); }
  // part -1: every program's forward (plain execute); part 0: forward + reverse of gradient programs.
  // inputs[j] / grads[j] are program j's arrays of device pointers, outputs[j] / grad_outs[j] its tensors.
  void run(int part, const void* const* const* inputs, const void* const* grad_outs, void* const* const* grads,
           void* const* outputs, void* ws, u64 ws_bytes, cudaStream_t st);
  // Synchronises `st`; the first nonzero device error word among the programs of the last run, or 0.
  int device_status(void* ws, cudaStream_t st);

 private:
  void enqueue(int part, const void* const* const* inputs, const void* const* grad_outs,
               void* const* const* grads, void* const* outputs, char* ws, cudaStream_t st);

  std::vector<Program*> progs_;
  std::vector<std::vector<size_t>> lanes_;  // program indices per lane, in launch order
  std::vector<u64> lane_off_;               // byte offset of each lane's workspace region
  std::vector<u64> prog_off_;               // byte offset of each program's workspace (its lane's)
  u64 status_off_ = 0;                      // per-program error words, after the lane regions
  u64 ws_total_ = 0;
  int device_ = 0;
  std::vector<cudaStream_t> streams_;
  cudaEvent_t fork_ = nullptr;
  std::vector<cudaEvent_t> join_;
  cudaGraphExec_t gexec_[2] = {nullptr, nullptr};  // [plain execute, gradient]
  std::vector<const void*> gkey_[2];
  std::mutex mu_;
};

}  // namespace ab2

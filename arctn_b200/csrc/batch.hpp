// ProgramBatch: many independent programs (uneven networks, mixed dtypes) as one CUDA graph launch.
//
// Two modes.
//  - PERSISTENT (the default): the small programs made of SIMT steps only run inside one persistent
//    interpreter launch (interp.cuh) that follows the steps' dependencies on the device; the others
//    (tensor-core steps, large SIMT GEMMs) run launch by launch on the lane streams alongside it.  The
//    interpreter's plan also handles steps it cannot run, in stages (stage t: those launches, then one
//    interpreter launch).  Each program gets its own workspace region.
//  - STAGED: as PERSISTENT, with every program inside the interpreter (tensor-core steps staged).
//  - LANES: the programs are spread over up to `max_lanes` streams by longest-processing-time first
//    (estimated time = flops at a nominal rate + launches x a nominal launch cost); each lane runs its
//    programs one after another, launch by launch, in one workspace region sized for the largest of them.
// Either way the sequence forks from the caller's stream, joins back into it and is captured once per
// set of bound pointers and replayed as a graph.  On the legacy stream or inside the caller's own
// capture both modes launch the lane form directly.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "program.hpp"

namespace ab2 {

class ProgramBatch {
 public:
  enum : int { LANES = 0, PERSISTENT = 1, STAGED = 2 };
  ProgramBatch(std::vector<Program*> programs, int max_lanes, int mode = PERSISTENT);
  ~ProgramBatch();
  ProgramBatch(const ProgramBatch&) = delete;
  ProgramBatch& operator=(const ProgramBatch&) = delete;

  u64 workspace_size() const { return ws_total_; }
  u64 n_lanes() const { return lanes_.size(); }
  u64 size() const { return progs_.size(); }
  int mode() const { return mode_; }
  // part -1: every program's forward (plain execute); part 0: forward + reverse of gradient programs.
  // inputs[j] / grads[j] are program j's arrays of device pointers, outputs[j] / grad_outs[j] its tensors.
  void run(int part, const void* const* const* inputs, const void* const* grad_outs, void* const* const* grads,
           void* const* outputs, void* ws, u64 ws_bytes, cudaStream_t st);
  // Synchronises `st`; the first nonzero device error word among the programs of the last run (and the
  // interpreter's own), or 0.
  int device_status(void* ws, cudaStream_t st);
  // JSON: mode, lanes, workspace and, per part, the interpreter's stages, steps and tasks; detail = 1
  // adds every interpreter step (program, op, stage, level, tasks, dependencies) and every staged launch.
  std::string describe(int detail) const;

 private:
  // The interpreter's plan for one part (slot 0: part -1, slot 1: part 0).
  struct Slot {
    bool valid = false;
    int part = -1;
    int n_stages = 0;
    std::vector<std::vector<std::pair<int, int>>> ext;  // per stage: (program, op) launched before it
    std::vector<int> stage_begin;                       // tasks of stage t: [stage_begin[t], stage_begin[t+1])
    std::vector<std::pair<int, int>> src;               // per interpreter step: (program, op)
    std::vector<int> sub, stage, level;                 // per step: descriptor index within its op, stage, level
    std::vector<std::vector<int>> deps;                 // per step: the same-stage steps it waits for
    std::vector<IOp> iops;
    std::vector<int> succ;                  // dependents of every step (IOp::succ0 / nsucc index it)
    std::vector<int> ctr0;                  // [error word, heads, tails, wait counts, done counts] at launch
    std::vector<unsigned long long> queue0;  // per stage: its root tasks first, then zeros
    u64 n_tasks = 0;
    IOp* d_ops = nullptr;
    int* d_succ = nullptr;
    int* d_ctr0 = nullptr;
    unsigned long long* d_queue0 = nullptr;
    int** d_errp = nullptr;
    cudaEvent_t used = nullptr;  // recorded after the last launch that reads the device tables
    bool launched = false;
  };

  void enqueue(int part, const void* const* const* inputs, const void* const* grad_outs,
               void* const* const* grads, void* const* outputs, char* ws, cudaStream_t st);
  void plan_slot(int s);
  void bind_slot(int s, const void* const* const* inputs, const void* const* grad_outs, void* const* const* grads,
                 void* const* outputs, char* ws);
  void enqueue_persistent(int s, const void* const* const* inputs, const void* const* grad_outs,
                          void* const* const* grads, void* const* outputs, char* ws, cudaStream_t st);
  void ensure_streams();

  std::vector<Program*> progs_;
  int mode_ = PERSISTENT;
  std::vector<std::vector<size_t>> lanes_;  // program indices per lane, in launch order
  std::vector<int> lane_of_;                // program -> lane
  std::vector<char> interp_;                // persistent mode: the program runs inside the interpreter
  std::vector<std::vector<size_t>> side_lanes_;  // persistent mode: the other programs per lane
  std::vector<u64> prog_off_;               // byte offset of each program's workspace region
  u64 status_off_ = 0;  // per-program error words, then the interpreter's counters (Slot::ctr0 layout)
  u64 queue_off_ = 0;   // the interpreter's queue
  u64 ws_total_ = 0;
  int device_ = 0;
  Slot slot_[2];
  int grid_ = 0;  // resident interpreter CTAs
  std::vector<cudaStream_t> streams_;
  cudaEvent_t fork_ = nullptr;
  std::vector<cudaEvent_t> join_;
  cudaGraphExec_t gexec_[2] = {nullptr, nullptr};  // [plain execute, gradient]
  std::vector<const void*> gkey_[2];
  std::mutex mu_;
};

// Runs the interpreter on one task whose dependency never completes and returns the error word it left
// (kInterpErrCode once the bounded wait expired); the device stays usable.  Test hook, about 2 s.
int interp_wait_selftest(cudaStream_t st);

}  // namespace ab2

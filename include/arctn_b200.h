/*
 * arctn_b200 -- B200-native executor for ArcTN's numerical contraction path.
 *
 * C ABI.  Plain pointers and sizes only; no C++ or torch types cross this
 * boundary.  Every entry point returns an int status (ARCTN_B200_OK == 0) and
 * records a message readable through arctn_b200_last_error() on the calling
 * thread.  No exception or unwinding crosses the ABI.
 *
 * Reference interfaces replaced (paths inside the ArcTN repository):
 *   TensorNetwork{inputs,output,size_dict}         src/network.rs:134-143
 *   CompiledContraction::compile                    src/compiled.rs:254
 *   CompiledContraction::execute / execute_stripped src/compiled.rs:369-381
 *   input_preps() / pair_steps() / finalize()       src/compiled.rs:241-250
 *   CompiledPairContraction accessors + execute     src/compiled.rs:102-153
 *   CompiledInputPrep::execute                      src/compiled.rs:60-63
 *   CompiledFinalize::execute                       src/compiled.rs:206-209
 *   contract_network_sliced                         src/slice.rs:960
 *   slice_parallel_chunks                           src/slice.rs:893-905
 *   simulate_path_full (metrics)                    src/path.rs:239-434
 *   greedy                                          src/paths/greedy.rs:317-320
 *   find_slices_to_size                             src/slice.rs:209-215
 *   find_slices_with_output                         src/slice.rs:254-289
 *   PyO3 CompiledContraction.compile/execute/stats  pybind/src/lib.rs:384-454
 *   PyO3 contract_sliced                            pybind/src/lib.rs:692-765
 */
#ifndef ARCTN_B200_H
#define ARCTN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ARCTN_B200_ABI_VERSION 1u

/* Status codes. */
enum {
  ARCTN_B200_OK = 0,
  ARCTN_B200_ERR_INVALID = 1,        /* network / path / shape / argument rejected before any launch */
  ARCTN_B200_ERR_CUDA = 2,           /* a CUDA runtime call failed */
  ARCTN_B200_ERR_UNSUPPORTED = 3,    /* valid input outside what this build executes */
  ARCTN_B200_ERR_DEVICE_TIMEOUT = 4, /* a bounded device-side wait expired */
  ARCTN_B200_ERR_WORKSPACE = 5       /* caller workspace smaller than required */
};

/* Element types; every input of one call shares the dtype
 * (pybind/src/lib.rs:287-330).  Complex values are (re, im) pairs. */
enum {
  ARCTN_B200_F32 = 0,
  ARCTN_B200_F64 = 1,
  ARCTN_B200_C64 = 2,  /* complex64  = 2 x f32 */
  ARCTN_B200_C128 = 3  /* complex128 = 2 x f64 */
};

/* Arithmetic used for the pairwise GEMMs of f32 / c64 contractions.
 * f64 / c128 always compute in FP64. */
enum {
  ARCTN_B200_PREC_FP32 = 0,   /* plain FP32 FFMA on the CUDA cores */
  ARCTN_B200_PREC_TF32X3 = 1, /* split-TF32 (3 products) on tcgen05 tensor cores, FP32 accumulate,
                                 for steps dense enough to fill a tensor-core tile; thin steps FP32.
                                 f32 steps run on the complex kernel with K folded in half into the
                                 real and imaginary parts (the real part of the product is kept) */
  ARCTN_B200_PREC_BF16X3 = 2, /* split-BF16 (3 products, hi/lo BF16 pairs) on tcgen05 tensor cores, FP32
                                 accumulate; each operand carried to about 2^-18, for precision studies;
                                 the same step selection as TF32X3 */
  ARCTN_B200_PREC_BF16X6 = 3  /* three-piece split-BF16 (x = h + m + l, 6 products hh hm mh hl lh mm) on tcgen05
                                 tensor cores, FP32 accumulate: FP32-level accuracy from BF16 MMAs; the same step
                                 selection as TF32X3 (no epilogue-fused operand packs) */
};

/* A tensor network (TensorNetwork, src/network.rs:134-143).
 * inputs are CSR: tensor i holds input_legs[input_offsets[i] .. input_offsets[i+1]].
 * size_dict is given as parallel arrays (size_legs[j] -> size_dims[j]). */
typedef struct {
  uint64_t n_inputs;
  const uint64_t* input_offsets; /* n_inputs + 1 entries */
  const uint32_t* input_legs;
  uint64_t n_output;
  const uint32_t* output;
  uint64_t n_sizes;
  const uint32_t* size_legs;
  const uint64_t* size_dims;
} arctn_b200_network;

typedef struct arctn_b200_plan arctn_b200_plan;       /* CompiledContraction (immutable, shareable) */
typedef struct arctn_b200_program arctn_b200_program; /* plan + slices + dtype bound to a device */

uint32_t arctn_b200_abi_version(void);
/* Last error message of the calling thread ("" when none). */
const char* arctn_b200_last_error(void);

/* ------------------------------------------------------------ planning support (host only) */

/* Path metrics in the order: log10_flops, log2_max_size, log2_max_contraction_size,
 * log2_total_size, log2_read_write, log2_peak_size (src/path.rs:14-29). */
int arctn_b200_simulate_path(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                             double stats_out[6]);
/* Deterministic greedy SSA path (src/paths/greedy.rs:317-320).  ssa_out holds 2*(n_inputs-1) entries. */
int arctn_b200_greedy(const arctn_b200_network* net, uint64_t* ssa_out, uint64_t* n_steps_out);
/* find_slices_to_size (src/slice.rs:209-215).  legs_out holds n_sizes entries; *found = 0 where the
 * reference returns None. */
int arctn_b200_find_slices_to_size(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                                   uint64_t target_size, uint32_t* legs_out, uint64_t* n_legs_out, int* found);
/* The same search with output legs allowed when allow_output_slicing != 0: the opt-in output-index slicing of
 * find_slices_until_for_target_with_output_slicing with no deadline (src/slice.rs:254-289, 557-589); a unary
 * network's output counts as its one intermediate. */
int arctn_b200_find_slices_with_output(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                                       uint64_t target_size, int allow_output_slicing, uint32_t* legs_out,
                                       uint64_t* n_legs_out, int* found);
/* Audit of a saved slice plan (src/execution_plan.rs:817-890, src/slice.rs:102-130): validates the sliced
 * legs (validate_slice_legs, src/slice.rs:152-176), writes the per-slice path metrics (sliced legs set to
 * dimension 1; same order as arctn_b200_simulate_path) and, for target_size > 0, *fits_out = 1 when every
 * per-slice intermediate holds at most target_size elements (exact integer test), else 0. */
int arctn_b200_slice_plan_check(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                                uint64_t n_sliced, const uint32_t* sliced_legs, uint64_t target_size,
                                double per_slice_stats_out[6], int* fits_out);
/* Deterministic chunk count of sliced summation (src/slice.rs:893-905). */
uint64_t arctn_b200_slice_parallel_chunks(uint64_t n_slices, uint64_t out_numel);

/* ------------------------------------------------------------ CompiledContraction */

int arctn_b200_plan_compile(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                            arctn_b200_plan** plan_out);
void arctn_b200_plan_destroy(arctn_b200_plan* plan);

uint64_t arctn_b200_plan_n_inputs(const arctn_b200_plan* plan);
uint64_t arctn_b200_plan_n_steps(const arctn_b200_plan* plan);
double arctn_b200_plan_log10_flops(const arctn_b200_plan* plan);
double arctn_b200_plan_log2_peak_size(const arctn_b200_plan* plan);

/* Views into the plan's immutable metadata; valid until arctn_b200_plan_destroy. */
typedef struct {
  uint64_t left_slot, right_slot, result_slot;
  uint64_t n_left, n_right, n_result;        /* ranks */
  const uint32_t* left_legs;
  const uint32_t* right_legs;
  const uint32_t* result_legs;               /* [batch, free_left, free_right] */
  const uint64_t* left_shape;
  const uint64_t* right_shape;
  const uint64_t* result_shape;
  uint64_t n_sum_a, n_sum_b;
  const uint64_t* sum_a;                     /* axes reduced from the left operand, in order */
  const uint64_t* sum_b;
  const uint64_t* a_perm;                    /* n_left - n_sum_a entries -> [batch, free_a, con] */
  const uint64_t* b_perm;                    /* n_right - n_sum_b entries -> [batch, con, free_b] */
  uint64_t bt, m, k, n;                      /* gemm_dims() */
} arctn_b200_step_info;

typedef struct {
  uint64_t n_input_shape;
  const uint64_t* input_shape;
  uint64_t n_traces;
  const uint64_t* traces;                    /* n_traces triples (ax_i, ax_j, is_diag) */
  uint64_t n_legs;
  const uint32_t* legs;
  const uint64_t* shape;
} arctn_b200_prep_info;

typedef struct {
  uint64_t slot;
  uint64_t n_input;
  const uint32_t* input_legs;
  const uint64_t* input_shape;
  uint64_t n_sum;
  const uint64_t* sum;
  uint64_t n_output;
  const uint64_t* perm;
  const uint64_t* output_shape;
} arctn_b200_finalize_info;

int arctn_b200_plan_step_info(const arctn_b200_plan* plan, uint64_t step, arctn_b200_step_info* out);
int arctn_b200_plan_prep_info(const arctn_b200_plan* plan, uint64_t input, arctn_b200_prep_info* out);
int arctn_b200_plan_finalize_info(const arctn_b200_plan* plan, arctn_b200_finalize_info* out);

/* Stage-by-stage execution on device buffers (CompiledInputPrep::execute, CompiledPairContraction::execute,
 * CompiledFinalize::execute).  Operands are contiguous row-major device tensors with the shapes the plan
 * records.  Each stage may need scratch: pass at least the matching *_workspace_size bytes (0 is allowed
 * when the size is 0).  Results are bit-identical to the corresponding stage inside a program execute. */
uint64_t arctn_b200_plan_prep_workspace_size(const arctn_b200_plan* plan, int dtype, uint64_t input);
uint64_t arctn_b200_plan_step_workspace_size(const arctn_b200_plan* plan, int dtype, int precision, uint64_t step);
uint64_t arctn_b200_plan_finalize_workspace_size(const arctn_b200_plan* plan, int dtype);
int arctn_b200_plan_prep_execute(const arctn_b200_plan* plan, int dtype, uint64_t input, const void* in, void* out,
                                 void* workspace, uint64_t workspace_bytes, void* cuda_stream);
int arctn_b200_plan_step_execute(const arctn_b200_plan* plan, int dtype, int precision, uint64_t step,
                                 const void* left, const void* right, void* out, void* workspace,
                                 uint64_t workspace_bytes, void* cuda_stream);
int arctn_b200_plan_finalize_execute(const arctn_b200_plan* plan, int dtype, const void* in, void* out,
                                     void* workspace, uint64_t workspace_bytes, void* cuda_stream);

/* ------------------------------------------------------------ device programs (execute / contract_sliced) */

typedef struct {
  int dtype;                     /* ARCTN_B200_F32 .. ARCTN_B200_C128 */
  int precision;                 /* ARCTN_B200_PREC_* */
  int device;                    /* CUDA device ordinal the program is bound to */
  int use_graph;                 /* capture the launch sequence once and replay it as a CUDA graph */
  uint64_t max_slices_per_group; /* 0: all slices in one group when the workspace budget allows */
  uint64_t workspace_budget;     /* bytes; 0: 8 GiB */
  uint64_t slice_begin;          /* run only global slices [slice_begin, slice_end); both 0: all slices.  A */
  uint64_t slice_end;            /* partial range sums only its slices (one rank of a sharded contraction). */
  int gradient;                  /* also build the adjoint sweep (arctn_b200_program_gradient); unsliced only */
  uint64_t tc_k_chunk;           /* tf32x3 / bf16x3: K per CTA before an FP64 split-K reduce (a multiple of 16,
                                    of 32 for bf16x3); 0: all of K,
                                    except unsliced GEMMs too small to fill the GPU, which split K to do so */
} arctn_b200_program_options;

/* Builds a program that contracts `net` along `ssa_path`, summing internal sliced legs and assembling
 * output-leg slices as blocks (contract_network_sliced, src/slice.rs:960-1173).  n_sliced == 0 gives the
 * unsliced CompiledContraction::execute.  Validation happens here, before anything is launched. */
int arctn_b200_program_create(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                              uint64_t n_sliced, const uint32_t* sliced_legs,
                              const arctn_b200_program_options* options, arctn_b200_program** program_out);
/* GEMM kernel variants.  A program picks one per GEMM from its shape with built-in heuristics; a tuning
 * table (arctn_b200_program_create_tuned) pins the variant per shape instead.  The reference runs every GEMM
 * through matrixmultiply's cgemm/zgemm/sgemm/dgemm (src/tensor.rs:49-64,193-231,270-308); it has no
 * variants and no tuner. */
enum {
  ARCTN_B200_GEMM_AUTO = 0,        /* the built-in heuristics */
  ARCTN_B200_GEMM_SIMT_SMALL = 1,  /* one thread per output, serial K (CUDA cores) */
  ARCTN_B200_GEMM_SIMT_TILE64 = 2, /* 64 x 64 output tile per CTA (CUDA cores) */
  ARCTN_B200_GEMM_SIMT_TILE32 = 3, /* 32 x 32 output tile per CTA (CUDA cores) */
  ARCTN_B200_GEMM_SIMT_WARP = 4,   /* one warp per output, lanes split K (CUDA cores) */
  ARCTN_B200_GEMM_SIMT_TILE128 = 5,/* 128 x 128 output tile per CTA, float32 only (CUDA cores) */
  ARCTN_B200_GEMM_SIMT_DOT = 6,    /* one CTA per output (split over CTAs when K >= 16384) */
  ARCTN_B200_GEMM_TC_MFAST = 7,    /* tcgen05 tensor-core GEMM, output tiles walked with m fastest, K unsplit */
  ARCTN_B200_GEMM_TC_NFAST = 8,    /* the same, n fastest */
  ARCTN_B200_GEMM_TC_SPLITK = 9,   /* the same, K split across CTAs to cover the SMs twice (FP64 split sum) */
  ARCTN_B200_GEMM_TC_STREAM = 10,  /* split-TF32 only: two-stage operand ring and a double-buffered epilogue that
                                      stages the next 32 output rows while storing the previous ones (short K) */
  ARCTN_B200_GEMM_TC_DEEP = 11,    /* split-TF32 only: six operand stages of 8 of K (32-byte swizzle) instead of
                                      three of 16, more copies in flight (long K) */
  ARCTN_B200_GEMM_TC_PAIR = 12,    /* split-TF32 only: clusters of two CTAs share 256 x 128 output tiles through
                                      cta_group::2 MMAs, each CTA holding half of the B tile (less operand
                                      traffic per MMA, four operand stages) */
  ARCTN_B200_GEMM_TC_PAIR_STREAM = 13 /* split-TF32 only: CTA pairs with the streaming epilogue of TC_STREAM over a
                                      three-stage ring (short K) */
};
/* One GEMM shape and its variant.  phase: 1 for a slice-invariant GEMM (run once per execute), 2 for one run
 * per slice group; a_var / b_var: whether that operand differs per slice; bt, m, k, n: gemm_dims() of one
 * slice (src/compiled.rs:138-141).  The tensor-core variants need precision TF32X3, BF16X3 or BF16X6 and a C64 or
 * F32 network; SIMT_TILE128 needs F32. */
typedef struct {
  int dtype, precision, phase, a_var, b_var, variant;
  uint64_t bt, m, k, n;
} arctn_b200_gemm_choice;

/* arctn_b200_program_create with a tuning table: every GEMM whose shape key (all fields but variant) matches
 * an entry runs that entry's variant; the others keep the heuristics.  An entry naming a variant the
 * program's dtype or precision cannot run is rejected (ARCTN_B200_ERR_INVALID).  No reference counterpart. */
int arctn_b200_program_create_tuned(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                                    uint64_t n_sliced, const uint32_t* sliced_legs,
                                    const arctn_b200_program_options* options, const arctn_b200_gemm_choice* table,
                                    uint64_t n_table, arctn_b200_program** program_out);
/* The program's GEMMs in launch order (a per-slice GEMM once per slice group): shape key and the variant it
 * runs (never AUTO); tuned_out[i] = 1 where a table entry chose it.  Writes at most cap entries (tuned_out
 * may be null); *n_out = the full count.  Host-only.  No reference counterpart. */
int arctn_b200_program_gemms(const arctn_b200_program* program, arctn_b200_gemm_choice* out, int* tuned_out,
                             uint64_t cap, uint64_t* n_out);
/* K summed per TMEM accumulation chain by the split-TF32 tensor-core GEMMs before the FP32 register sum: 32, 64
 * or 128.  Programs default to 64 (32 for gradient programs, whose long-K adjoint GEMMs carry the tightest
 * error budget).  Longer chains drain TMEM less often and let the MMAs run further ahead of each epilogue,
 * at a longer truncated-FP32 chain per chunk.  Changes launch parameters only; the next execute re-captures
 * its graph.  Not thread-safe against a concurrent execute of the same program.  No reference counterpart. */
int arctn_b200_program_set_tc_chain(arctn_b200_program* program, uint64_t k_per_chain);
void arctn_b200_program_destroy(arctn_b200_program* program);
uint64_t arctn_b200_program_workspace_size(const arctn_b200_program* program);
uint64_t arctn_b200_program_n_slices(const arctn_b200_program* program);
uint64_t arctn_b200_program_slices_per_group(const arctn_b200_program* program);
/* Algorithmic real flops of one execution: 8 (complex) or 2 (real) x sum_steps bt*m*k*n x slices. */
double arctn_b200_program_flops(const arctn_b200_program* program);
/* Number of kernels one graph-replayed execute launches (independent thin steps of one level of the step
 * DAG count once: they share a grouped launch). */
uint64_t arctn_b200_program_launches(const arctn_b200_program* program);
/* Gradient programs: how many step results the adjoint sweep recomputes instead of keeping from the
 * forward, chosen at creation (largest results first) so that the workspace fits workspace_budget.
 * 0 when everything fits.  No reference counterpart: the reference has no adjoint. */
uint64_t arctn_b200_program_recomputed_steps(const arctn_b200_program* program);
/* JSON description of the program's launch sequence and workspace layout (op kinds with their GEMM /
 * pack / gather geometry, group size, recomputed steps).  Host-only: a program can be created and
 * described on a machine without a GPU (its tables are then uploaded on the first execute).  Writes at
 * most buf_bytes bytes including the terminating NUL; *needed receives the full size. */
int arctn_b200_program_describe(const arctn_b200_program* program, char* buf, uint64_t buf_bytes, uint64_t* needed);

/* Runs on `cuda_stream` (cudaStream_t; NULL = legacy default stream).  inputs[i] are contiguous device
 * tensors in net order; output receives the full output (native dtype).  The call is asynchronous. */
int arctn_b200_program_execute(arctn_b200_program* program, const void* const* inputs, void* output,
                               void* workspace, uint64_t workspace_bytes, void* cuda_stream);
/* Same, but writes the result in FP64 (f64 / c128) from the FP64 cross-slice sum. */
int arctn_b200_program_execute_f64out(arctn_b200_program* program, const void* const* inputs, void* output_f64,
                                      void* workspace, uint64_t workspace_bytes, void* cuda_stream);
/* execute_stripped (src/compiled.rs:376-441): unsliced programs only.  Synchronises the stream and writes
 * the accumulated decimal exponent to *log10_exponent. */
int arctn_b200_program_execute_stripped(arctn_b200_program* program, const void* const* inputs, void* output,
                                        void* workspace, uint64_t workspace_bytes, void* cuda_stream,
                                        double* log10_exponent);

/* Adjoint of the contraction (programs created with options.gradient = 1).  With grad_output G (the
 * output's shape), writes grad_inputs[i] = dL/d conj(T_i) in PyTorch's complex convention: for a step
 * C = A.B the sweep forms dA = dC.conj(B)^T and dB = conj(A)^T.dC, undoing each step's permutes and
 * broadcasting over the legs it summed away (src/compiled.rs:155-171 is the forward it reverses).
 * part 0: forward (result into `output`) then the reverse sweep; part 1: forward only, keeping the
 * intermediates in `workspace`; part 2: reverse sweep only, reusing the workspace of a preceding
 * part-1 call with the same inputs.  No counterpart in the reference, which has no differentiation. */
int arctn_b200_program_gradient(arctn_b200_program* program, int part, const void* const* inputs,
                                const void* grad_output, void* const* grad_inputs, void* output, void* workspace,
                                uint64_t workspace_bytes, void* cuda_stream);

/* Synchronises `cuda_stream` and reports the device status word the last execute on `workspace` left:
 * *code = 0 when every bounded device-side wait completed, else the code of the first wait that expired
 * (the call then returns ARCTN_B200_ERR_DEVICE_TIMEOUT). */
int arctn_b200_program_device_status(arctn_b200_program* program, void* workspace, void* cuda_stream, int* code);

/* Profiled execute: launches unit by unit (no graph; a grouped launch of thin steps is one unit) with a CUDA
 * event between consecutive launches on `cuda_stream`, synchronises, and writes per-launch duration (ms),
 * kind and algorithmic work (real flops for GEMM kinds, bytes moved for the others).  Arrays hold
 * arctn_b200_program_launches entries; unused entries keep their initial values.
 * Kinds: 0 gather, 1 gemm_small, 2 gemm_tile64, 3 gemm_tile32, 4 slice_accumulate, 5 slice_output,
 * 7 maxabs, 8 strip, 9 gemm_tc, 10 gemm_dot, 11 pack, 12 scatter, 13 pack_tiled, 14 gemm_warp, 15 grad_accum,
 * 16 narrow, 17 gemm_tile128. */
int arctn_b200_program_profile(arctn_b200_program* program, const void* const* inputs, void* output, void* workspace,
                               uint64_t workspace_bytes, void* cuda_stream, float* ms_out, int* kind_out,
                               double* work_out);

/* The same for a gradient program: forward + reverse sweep op by op, with grad_output and grads bound as in
 * arctn_b200_program_gradient part 0.  No reference counterpart (the reference has no adjoint). */
int arctn_b200_program_profile_gradient(arctn_b200_program* program, const void* const* inputs,
                                        const void* grad_output, void* const* grads, void* output, void* workspace,
                                        uint64_t workspace_bytes, void* cuda_stream, float* ms_out, int* kind_out,
                                        double* work_out);

/* No counterpart in the reference.  Batched complex64 GEMM C[b] = A[b] . B[b] (A: bt x m x k, B: bt x k x n,
 * C: bt x m x n, row-major complex64 device buffers) on the split-TF32 tensor-core path, for callers that
 * cannot allocate device memory (a framework holding the whole memory pool, code where an allocation
 * would synchronise the device or break a stream capture).  It allocates nothing: its scratch is a fixed
 * 64 MiB __device__ array that every GPU loading the library keeps until the process exits, and it
 * returns ARCTN_B200_ERR_UNSUPPORTED for problems whose packed operands exceed it.  The first call on a
 * device resolves the array's device address; make it before any stream capture.  All calls on a device
 * share the array, so calls that overlap on the GPU race: order them on one stream.  Asynchronous on
 * `cuda_stream`. */
int arctn_b200_cgemm_tf32x3_noalloc(const void* a, const void* b, void* c, uint64_t bt, uint64_t m, uint64_t k,
                                    uint64_t n, void* cuda_stream);
/* No counterpart in the reference.  Status of the last arctn_b200_cgemm_tf32x3_noalloc call on the current
 * device: waits for cuda_stream, then sets *code to its kernel's status word (0: complete; nonzero: a bounded
 * wait expired, C is incomplete; the codes are those of arctn_b200_program_device_status).  Allocates
 * nothing: a 4-byte copy into the caller's host memory.  *code = 0 when no call has run on the device. */
int arctn_b200_cgemm_noalloc_status(void* cuda_stream, int* code);

/* No counterpart in the reference (a measurement aid).  The dense tensor-pipe rate of the current GPU:
 * one CTA per SM streams `iters` tcgen05.mma instructions (M = 128, N = n in {128, 256}; kind 0: TF32,
 * K = 8; kind 1: BF16, K = 16) over operands resident in shared memory, with no TMA and no epilogue.
 * kind 2 (n = 128): `iters` K steps of the split-TF32 GEMM's own 12-MMA 4M sequence over planes laid out as
 * its three-stage operand ring, a new 64 KB stage every two steps -- the ceiling of the GEMM's MMA phase; every
 * operand is 1.0.  kind 3 (n = 128): the same stream over random TF32 hi / lo operands with random signs, whose
 * bit activity (and so power under the 1 kW cap, when run for seconds) is that of real packed operands.
 * kind 4 (n = 128): `iters` K steps of 16 of the three-piece split-BF16 GEMM's 24-MMA sequence (kind::f16,
 * K = 16) over random BF16 pieces laid out as its two-stage ring; the rate counts BF16 MMA work.
 * kind 5 (n = 128): a 3M split-TF32 complex product's 9-MMA sequence per K step (three accumulators, six
 * random planes per operand), a measurement of that form's sustained rate; it counts TF32 MMA work.
 * Synchronises cuda_stream and sets *tflops_out to 2*128*n*K*MMAs / elapsed (TF32 MMA work).  `status` is a
 * device int the caller zeroed: nonzero afterwards means the final bounded wait expired.  iters in [2, 2^22]. */
int arctn_b200_tc_peak(int kind, int n, uint64_t iters, void* status, void* cuda_stream, double* tflops_out);

/* ------------------------------------------------------------ batches of independent programs
 * No counterpart in the reference (it contracts one network per call).  A batch runs many programs --
 * uneven networks, mixed dtypes -- as one CUDA graph launch, in one of three modes:
 *   PERSISTENT (arctn_b200_batch_create's mode): the small programs made of SIMT steps only (up to 5e8
 *     flops a forward pass) run inside one persistent interpreter launch that follows the steps'
 *     dependencies on the device; the other programs run launch by launch on up to max_lanes streams
 *     (longest first onto the least-loaded lane) alongside it.  Every program has its own workspace region.
 *     A queue wait that expires (2 s) sets device error code 16.
 *   STAGED: every program inside the interpreter; the tensor-core GEMMs and their operand packs split the
 *     work into stages (each stage: those launches on the lane streams, then one interpreter launch).
 *   LANES: every program launch by launch on the lane streams, each lane running its programs in turn
 *     in one workspace region.
 * Both fork from and join back into cuda_stream, and both use the lane form on the legacy stream or
 * inside the caller's stream capture.  Results are the same bits in both modes.  The programs must outlive
 * the batch and be bound to one device; a batch locks them while it launches.  Creating and describing
 * a batch needs no GPU. */
typedef struct arctn_b200_batch arctn_b200_batch;
enum { ARCTN_B200_BATCH_LANES = 0, ARCTN_B200_BATCH_PERSISTENT = 1, ARCTN_B200_BATCH_STAGED = 2 };
int arctn_b200_batch_create(arctn_b200_program* const* programs, uint64_t n_programs, int max_lanes,
                            arctn_b200_batch** batch_out);
int arctn_b200_batch_create_mode(arctn_b200_program* const* programs, uint64_t n_programs, int max_lanes, int mode,
                                 arctn_b200_batch** batch_out);
/* JSON: mode, lanes, workspace, the interpreted programs, program regions and, per part (-1 execute,
 * 0 gradient), the interpreter's
 * stages, steps and tasks; detail = 1 adds every step [program, op, sub, stage, level, tasks, [deps]] and
 * every staged launch [stage, program, op].  Writes at most buf_bytes (NUL-terminated); *needed = full size. */
int arctn_b200_batch_describe(const arctn_b200_batch* batch, int detail, char* buf, uint64_t buf_bytes,
                              uint64_t* needed);
/* Test hook of the interpreter's bounded waits: runs it on one task whose dependency nothing completes,
 * synchronises cuda_stream and sets *code to the error word left (16 once the 2 s wait expired). */
int arctn_b200_batch_wait_selftest(void* cuda_stream, int* code);
/* Host-side fault injection for tests of the error paths; no counterpart in the reference.  Arms a countdown for
 * one site: the countdown-th next call of that site fails at its entry, before any CUDA work, with
 * ARCTN_B200_ERR_CUDA and the message of a failed CUDA allocation; 0 disarms.  Site 0: program and batch
 * execute, execute_stripped and gradient calls; site 1: program and batch creation.  Process-wide. */
int arctn_b200_debug_inject_failure(int site, int countdown);
void arctn_b200_batch_destroy(arctn_b200_batch* batch);
uint64_t arctn_b200_batch_workspace_size(const arctn_b200_batch* batch);
uint64_t arctn_b200_batch_lanes(const arctn_b200_batch* batch);
/* inputs[j] is program j's array of input device pointers, outputs[j] its output buffer.  Asynchronous. */
int arctn_b200_batch_execute(arctn_b200_batch* batch, const void* const* const* inputs, void* const* outputs,
                             void* workspace, uint64_t workspace_bytes, void* cuda_stream);
/* Forward + adjoint of every program (all built with options.gradient = 1): grad_outputs[j] and grads[j]
 * as in arctn_b200_program_gradient part 0.  Asynchronous. */
int arctn_b200_batch_gradient(arctn_b200_batch* batch, const void* const* const* inputs,
                              const void* const* grad_outputs, void* const* const* grads, void* const* outputs,
                              void* workspace, uint64_t workspace_bytes, void* cuda_stream);
/* Synchronises cuda_stream; *code = the first nonzero device error word of the last run (the programs'
 * in program order, then the interpreter's), else 0. */
int arctn_b200_batch_device_status(arctn_b200_batch* batch, void* workspace, void* cuda_stream, int* code);

/* One-shot host-buffer call (the reference-facing e2e path of contract_sliced): copies host inputs to the
 * device, executes, copies the result back and synchronises.  Allocates its own device memory. */
int arctn_b200_contract_sliced_host(const arctn_b200_network* net, uint64_t n_steps, const uint64_t* ssa_path,
                                    uint64_t n_sliced, const uint32_t* sliced_legs,
                                    const arctn_b200_program_options* options, const void* const* host_inputs,
                                    void* host_output);

#ifdef __cplusplus
}
#endif

#endif /* ARCTN_B200_H */

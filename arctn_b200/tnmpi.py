"""Slice-sharded execution of a saved plan across ranks, one GPU per rank.

The counterpart of the reference's MPI runner (src/bin/tnmpi.rs): rank 0 loads a version-2 execution plan
and broadcasts it; every rank contracts the contiguous slice range ``slice_range(n_slices, ranks, rank)``
with the product's slice-range program (``SlicedProgram(..., slice_begin, slice_end)``) into a zeroed
complete FP64 output, so an output-leg slice fills only its own block; one all-reduce(SUM) assembles the
result; rank 0 prints the reference's JSON stats line.  Launch it like any torch.distributed job::

    python -m torch.distributed.run --nproc-per-node 8 --master-addr 127.0.0.1 \\
        -m arctn_b200.tnmpi --load-path plan.json --data tensors.bin --dtype complex64 --precision tf32x3

Differences from the reference, each deliberate:
- the collective is NCCL over NVLink on the ranks' FP64 partials (``--backend gloo`` sums host copies instead);
- the sum is in FP64 whatever the dtype (the reference all-reduces in the dtype itself), so the result does
  not depend on the rank count beyond FP64 rounding;
- ``--precision`` selects the executor's GEMM form (fp32, tf32x3, bf16x3, bf16x6; the reference has one);
- example inputs (no ``--data``) are uniform in [-1, 1) per real component, as the reference's
  ``DenseTensor::random``, but drawn from NumPy's PCG64 seeded with ``seed ^ 0x5eed0000 ^ index``; the
  reference's ChaCha8 stream cannot be reproduced without its crates;
- ``--check`` compares with a single-process execution of all slices on rank 0's GPU;
- besides the wall clock, each rank times its execute and the all-reduce with CUDA events, and the line
  reports the maximum over ranks (``execution_device_seconds_max``);
- version-1 plans with ``--net`` are not read (only self-contained version-2 plans);
- ``--broadcast-inputs``: rank 0 alone reads (or generates) the inputs and one broadcast of all their bytes
  replicates them, over NVLink with NCCL, so the other ranks need no access to the data file.

Failures follow the reference's ``require_all`` (src/bin/tnmpi.rs:165-177): a rank that fails reports its
error, every rank learns of it through an all-reduce(MAX) of a failure flag before the next collective, and
all ranks leave with exit code 3.  Usage errors exit with 2, as the reference's argument parser does.
"""

from __future__ import annotations

import json
import sys
import time

import numpy as np

from .execution_plan import ExecutionPlan, PlanValidationError, load_tensors_bin

USAGE = """tnmpi (arctn_b200)
Usage: python -m torch.distributed.run ... -m arctn_b200.tnmpi --load-path <PLAN.json> [OPTIONS]

Execute the saved SSA path and sliced indices; no path search is performed.
  --data <tensors.bin> Row-major little-endian tensors in network input order
  --dtype <TYPE>       f32, f64, complex64 or complex128 (default f64)
  --precision <MODE>   fp32, tf32x3, bf16x3 or bf16x6 GEMMs for f32/complex64 (default fp32)
  --seed <N>           Seed for example inputs when --data is omitted (default 1)
  --backend <NAME>     nccl (default) or gloo for the all-reduce
  --check              Compare a small result with single-process execution
  --broadcast-inputs   Rank 0 alone reads (or generates) the inputs; one broadcast replicates them
  --help               Show this help

Version 2 plans contain the network; every rank must read identical input data.
Complex elements store the real component followed by the imaginary component.
Execution time includes the final all-reduce, but not loading or --check."""

DTYPES = {"f32": np.float32, "f64": np.float64, "complex64": np.complex64, "complex128": np.complex128}
# Tolerance of --check relative to the largest magnitude of the single-process result (src/bin/tnmpi.rs:53-58).
CHECK_TOLERANCE = {"f32": 1e-4, "complex64": 1e-4, "f64": 1e-6, "complex128": 1e-6}
# --check is skipped above these sizes (src/bin/tnmpi.rs:386-388).
CHECK_MAX_NUMEL, CHECK_MAX_SLICES = 1 << 22, 1 << 12


class UsageError(ValueError):
    """A command-line error (exit code 2)."""


class RankFailure(RuntimeError):
    """Some rank failed; every rank raises this at the same collective step (exit code 3)."""


class Args:
    def __init__(self):
        self.load_path = ""
        self.data_file = None
        self.dtype = "f64"
        self.precision = "fp32"
        self.seed = 1
        self.backend = "nccl"
        self.check = False
        self.broadcast_inputs = False


def parse_args(argv):
    """Parsed options, or None for --help (parse_args, src/bin/tnmpi.rs:95-129)."""
    args = Args()
    it = iter(argv)
    for flag in it:
        if flag in ("--help", "-h"):
            return None
        if flag == "--check":
            args.check = True
            continue
        if flag == "--broadcast-inputs":
            args.broadcast_inputs = True
            continue
        if flag == "--net":
            raise UsageError("--net (version 1 plans) is not supported; save a version 2 plan")
        if flag not in ("--load-path", "--data", "--seed", "--dtype", "--precision", "--backend"):
            raise UsageError(f"unknown option: {flag}; use --help")
        value = next(it, None)
        if value is None or value.startswith("--"):
            raise UsageError(f"{flag} requires a value")
        if flag == "--load-path":
            args.load_path = value
        elif flag == "--data":
            args.data_file = value
        elif flag == "--dtype":
            if value not in DTYPES:
                raise UsageError("--dtype must be f32, f64, complex64 or complex128")
            args.dtype = value
        elif flag == "--precision":
            if value not in ("fp32", "tf32x3", "bf16x3", "bf16x6"):
                raise UsageError("--precision must be fp32, tf32x3, bf16x3 or bf16x6")
            args.precision = value
        elif flag == "--backend":
            if value not in ("nccl", "gloo"):
                raise UsageError("--backend must be nccl or gloo")
            args.backend = value
        else:
            try:
                args.seed = int(value)
                if not 0 <= args.seed < 1 << 64:
                    raise ValueError
            except ValueError:
                raise UsageError("--seed requires an unsigned 64-bit integer") from None
    if not args.load_path:
        raise UsageError("--load-path <PLAN.json> is required")
    return args


def example_inputs(plan, dtype, seed):
    """Seeded inputs when no data file is given: every real component uniform in [-1, 1)."""
    dt = np.dtype(DTYPES[dtype])
    out = []
    for index, legs in enumerate(plan.inputs):
        shape = tuple(plan.size_dict[l] for l in legs)
        rng = np.random.default_rng((int(seed) ^ 0x5EED0000 ^ index) & ((1 << 64) - 1))
        if dt.kind == "c":
            a = rng.uniform(-1.0, 1.0, shape) + 1j * rng.uniform(-1.0, 1.0, shape)
        else:
            a = rng.uniform(-1.0, 1.0, shape)
        out.append(np.ascontiguousarray(a, dtype=dt))
    return out


class _Group:
    """The run's collective steps over the default torch.distributed group.  Every rank takes the same steps
    in the same order, failure paths included."""

    def __init__(self, backend, device):
        import torch
        import torch.distributed as dist

        self.torch, self.dist = torch, dist
        self.rank, self.size = dist.get_rank(), dist.get_world_size()
        self.backend = backend
        self.cdev = device if backend == "nccl" else torch.device("cpu")  # where collective tensors live

    def require_all(self, fn):
        """fn() on this rank; if it raised on any rank, every rank raises RankFailure here
        (require_all, src/bin/tnmpi.rs:165-177)."""
        try:
            value, err = fn(), None
        except Exception as exc:  # noqa: BLE001 -- every error becomes the ranks' common failure
            value, err = None, exc
        flag = self.torch.tensor([0 if err is None else 1], dtype=self.torch.int32, device=self.cdev)
        self.dist.all_reduce(flag, op=self.dist.ReduceOp.MAX)
        if int(flag.item()):
            if err is not None:
                print(f"tnmpi rank {self.rank}: {err}", file=sys.stderr, flush=True)
            raise RankFailure(str(err) if err is not None else "another rank failed")
        return value

    def broadcast_object(self, obj):
        box = [obj]
        self.dist.broadcast_object_list(box, src=0, device=self.cdev if self.backend == "nccl" else None)
        return box[0]

    def replicate_inputs(self, plan, dtype, load):
        """Every rank's copy of the inputs from one broadcast of rank 0's bytes.  Only rank 0 calls ``load``;
        a failure there stops every rank before the broadcast.  With NCCL the copies are device tensors."""
        torch = self.torch
        dt = np.dtype(DTYPES[dtype])
        shapes = [tuple(plan.size_dict[l] for l in legs) for legs in plan.inputs]
        counts = [int(np.prod(sh, dtype=np.int64)) for sh in shapes]
        arrays = self.require_all(lambda: load() if self.rank == 0 else None)
        buf = torch.empty(sum(counts) * dt.itemsize, dtype=torch.uint8, device=self.cdev)
        if self.rank == 0 and buf.numel():
            host = np.concatenate([np.ascontiguousarray(a, dtype=dt).reshape(-1) for a in arrays]).view(np.uint8)
            buf.copy_(torch.from_numpy(host))
        if buf.numel():
            self.dist.broadcast(buf, src=0)
        tdt = {"f": {4: torch.float32, 8: torch.float64}, "c": {8: torch.complex64, 16: torch.complex128}}
        out, off = [], 0
        for sh, n in zip(shapes, counts):
            piece = buf[off:off + n * dt.itemsize]
            off += n * dt.itemsize
            if self.backend == "nccl":
                out.append(piece.view(tdt[dt.kind][dt.itemsize]).reshape(sh))
            else:
                out.append(piece.numpy().view(dt).reshape(sh).copy())
        return out

    def sum_(self, t):
        """In-place all-reduce(SUM) of an FP64 (real or complex) tensor."""
        flat = self.torch.view_as_real(t) if t.is_complex() else t
        if self.backend == "nccl":
            self.dist.all_reduce(flat)
            return t
        host = flat.cpu()
        self.dist.all_reduce(host)
        flat.copy_(host)
        return t

    def max_(self, x):
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.cdev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())


def gpu_range_executor(plan, arrays, args, begin, end, device):
    """The product's executor for slices [begin, end): a slice-range program with FP64 output, its inputs and
    workspace on ``device``.  Returns a callable giving the FP64 partial as a device tensor, after checking the
    program's bounded-wait status word."""
    import torch

    from .api import SlicedProgram

    n_slices = int(np.prod([plan.size_dict[l] for l in plan.sliced_legs], dtype=np.int64)) if plan.sliced_legs else 1
    whole = begin == 0 and end == n_slices
    prog = SlicedProgram(plan.inputs, plan.output, plan.size_dict, plan.ssa_path, plan.sliced_legs,
                         dtype=DTYPES[args.dtype], precision=args.precision, device=device.index,
                         slice_begin=0 if whole else begin, slice_end=0 if whole else end)
    x = [a.to(device) if torch.is_tensor(a) else torch.from_numpy(np.ascontiguousarray(a)).to(device)
         for a in arrays]
    ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device=device)

    def call():
        out = prog.execute(x, workspace=ws, f64_out=True)
        status = prog.device_status(ws)
        if status:
            raise RuntimeError(f"device status {status}: a bounded wait in a kernel expired")
        return out

    return call


def _wide_dtype(dtype):
    import torch

    return torch.complex128 if np.dtype(DTYPES[dtype]).kind == "c" else torch.float64


def _check_result(plan, arrays, args, total, n_slices, executor, device):
    """Single-process comparison on rank 0 (check_result, src/bin/tnmpi.rs:378-401)."""
    if total.size > CHECK_MAX_NUMEL or n_slices > CHECK_MAX_SLICES:
        return "skipped: reference exceeds size limit"
    ref = executor(plan, arrays, args, 0, n_slices, device)().cpu().numpy()
    diff = float(np.max(np.abs(ref - total))) if total.size else 0.0
    scale = max(1.0, float(np.max(np.abs(ref)))) if ref.size else 1.0
    if not (np.all(np.isfinite(ref)) and np.all(np.isfinite(total)) and np.isfinite(diff)) or \
            diff > CHECK_TOLERANCE[args.dtype] * scale:
        raise RuntimeError(f"single-process comparison failed: max_abs_diff={diff}, scale={scale}")
    return f"PASS(max_abs_diff={diff:.3e})"


def run(args, *, device=None, executor=gpu_range_executor):
    """One sharded execution on the default process group (run, src/bin/tnmpi.rs:404-496).  Returns
    (stats, total): the JSON stats dict (the same on every rank) and the all-reduced FP64 output as NumPy.
    ``executor`` builds the callable that contracts a slice range (the product's GPU program)."""
    import math

    import torch

    from .api import slice_range

    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else \
            torch.device("cpu")
    g = _Group(args.backend, device)
    load_start = time.perf_counter()

    # Rank 0 loads and validates the plan; the others receive its artifact, or its error (broadcast_input,
    # src/bin/tnmpi.rs:179-200).
    payload = None
    if g.rank == 0:
        try:
            payload = {"ok": ExecutionPlan.load(args.load_path).to_dict()}
        except (PlanValidationError, OSError, ValueError) as exc:
            payload = {"err": str(exc)}
    payload = g.broadcast_object(payload)

    def decode():
        if "err" in payload:
            raise PlanValidationError(payload["err"])
        return ExecutionPlan.from_dict(payload["ok"])

    plan = g.require_all(decode)
    n_slices = int(math.prod(plan.size_dict[l] for l in plan.sliced_legs))
    out_shape = tuple(plan.size_dict[l] for l in plan.output)
    def load():
        if args.data_file:
            return load_tensors_bin(args.data_file, plan.inputs, plan.size_dict, DTYPES[args.dtype])
        return example_inputs(plan, args.dtype, args.seed)

    arrays = g.replicate_inputs(plan, args.dtype, load) if args.broadcast_inputs else g.require_all(load)
    begin, end = slice_range(n_slices, g.size, g.rank)
    call = g.require_all(lambda: executor(plan, arrays, args, begin, end, device) if begin < end else None)
    wide = _wide_dtype(args.dtype)
    load_seconds = time.perf_counter() - load_start

    g.dist.barrier()
    timed = device.type == "cuda"
    if timed:
        torch.cuda.synchronize(device)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(torch.cuda.current_stream(device))
    exec_start = time.perf_counter()
    local = g.require_all(lambda: call() if call is not None else torch.zeros(out_shape, dtype=wide, device=device))
    local = local.to(device=device, dtype=wide).contiguous()
    g.sum_(local)
    if timed:
        ev1.record(torch.cuda.current_stream(device))
        torch.cuda.synchronize(device)
    exec_seconds = time.perf_counter() - exec_start
    device_seconds = ev0.elapsed_time(ev1) / 1e3 if timed else float("nan")
    total = local.cpu().numpy()

    check = g.require_all(lambda: _check_result(plan, arrays, args, total, n_slices, executor, device)
                          if args.check and g.rank == 0 else "not requested")
    check = g.broadcast_object(check)
    load_max, exec_max, dev_max = g.max_(load_seconds), g.max_(exec_seconds), g.max_(device_seconds)
    per = plan.per_slice_metrics
    stats = {
        "ranks": g.size,
        "network": plan.name,
        "mode": "saved-path",
        "dtype": args.dtype,
        "precision": args.precision,
        "backend": args.backend,
        "sliced_indices": list(plan.sliced_legs),
        "n_slices": n_slices,
        "target_size": plan.target_size,
        "target_log2_size": math.log2(plan.target_size) if plan.target_size else None,
        "per_slice_log10_flops": per["log10_flops"],
        "per_slice_log2_max_size": per["log2_max_size"],
        "per_slice_log2_peak_size": per["log2_peak_size"],
        "per_slice_log2_max_contraction_size": per["log2_max_contraction_size"],
        "output_shape": list(out_shape),
        "load_wall_seconds_max": load_max,
        "execution_wall_seconds_max": exec_max,
        "execution_device_seconds_max": dev_max if timed else None,
        "check": check,
    }
    return stats, total


def main(argv=None):
    """Command-line entry: exit 0 on success, 2 on a usage error, 3 when any rank failed."""
    import datetime
    import os
    import socket

    try:
        args = parse_args(sys.argv[1:] if argv is None else argv)
    except UsageError as exc:
        print(f"tnmpi: {exc}", file=sys.stderr)
        return 2
    if args is None:
        print(USAGE)
        return 0
    import torch
    import torch.distributed as dist

    if "RANK" not in os.environ:  # a single process without a launcher: a one-rank group
        with socket.socket() as s:
            s.bind(("127.0.0.1", 0))
            os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(s.getsockname()[1]), RANK="0",
                              WORLD_SIZE="1", LOCAL_RANK="0")
    device = None
    if args.backend == "nccl":
        if not torch.cuda.is_available():
            print("tnmpi: the nccl backend needs a CUDA device; use --backend gloo for host collectives",
                  file=sys.stderr)
            return 2
    if torch.cuda.is_available():
        device = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")) % torch.cuda.device_count())
        torch.cuda.set_device(device)
    dist.init_process_group(args.backend, timeout=datetime.timedelta(seconds=300))
    code = 0
    try:
        stats, _ = run(args, device=device)
        if dist.get_rank() == 0:
            print(json.dumps(stats), flush=True)
    except RankFailure:
        code = 3
    finally:
        dist.destroy_process_group()
    return code


if __name__ == "__main__":
    sys.exit(main())

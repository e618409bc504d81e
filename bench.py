#!/usr/bin/env python
"""Benchmark: sliced complex64 tensor-network contraction TFLOP/s on B200.

Workload (default): random 3-regular graph, bond dimension 2 on every edge,
graph seed 1, complex64 entries N(0,1)/sqrt(8), scalar output, greedy SSA path,
sliced with find_slices_to_size(target 2^24) into 2^8 = 256 slices, all slices
summed in FP64.  n = 172 nodes: the smallest graph of this family whose greedy
path needs slicing at 2^24 and lands in 2^8..2^10 slices (n = 64 peaks at 2^13
elements and needs no slicing at 2^24).

One step = one full sliced contraction (all 256 slices) of inputs resident in
HBM.  TFLOP/s counts 8 real flops per complex MAC over every pairwise GEMM of
every slice (the reference's per-slice work x n_slices).

    python bench.py [--gpus N --steps K --warmup W] [--impl b200|reference] [--precision fp32|tf32x3]

Under torchrun each rank contracts a contiguous range of slices (the
reference's MPI slice_range, src/bin/tnmpi.rs:279-284) and one NCCL
all-reduce sums the FP64 partial outputs; the printed value is total flops
over the max-over-ranks device time.
"""

from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "c64 sliced TN contraction TFLOP/s"
KIND_NAMES = {0: "k_gather_reduce", 1: "k_gemm_small", 2: "k_gemm_tile<64,64>", 3: "k_gemm_tile<32,32>",
              4: "k_slice_accumulate", 5: "k_slice_output", 7: "k_maxabs", 8: "k_strip_scale", 9: "k_gemm_tc"}
GEMM_KINDS = {1, 2, 3, 9}


def parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--precision", choices=["fp32", "tf32x3"], default="fp32")
    ap.add_argument("--nodes", type=int, default=172)
    ap.add_argument("--target-log2", type=int, default=24)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-profile", action="store_true")
    return ap.parse_args()


def workload(n_nodes, target_log2):
    import arctn_b200 as A
    from arctn_b200 import networks as N

    net, arrays = N.workload_rand3reg(n_nodes, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** target_log2)
    if sliced is None:
        raise SystemExit("no slicing meets the target")
    name = f"rand3reg_n{n_nodes}_bond2_seed1_c64_greedy_target2^{target_log2}_{2 ** len(sliced)}slices"
    return net, arrays, path, sliced, name


def slice_range(count, ranks, rank):
    """Contiguous slice range of one rank (src/bin/tnmpi.rs:279-284)."""
    chunk, extra = divmod(count, ranks)
    begin = rank * chunk + min(rank, extra)
    return begin, begin + chunk + (1 if rank < extra else 0)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"],
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained", d["bf16_tflops"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(net, arrays, path, sliced, total_slices, flops_total):
    """The oracle (CPU restatement of the reference executor) on a bounded sample of slices."""
    from oracle import oracle as O

    O.build()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    threads = max(1, min(cores, 32, total_slices))
    t0 = time.perf_counter()
    O.contract_slice_range(*net.as_tuple(), path, sliced, 0, threads, arrays, threads=threads)
    dt = time.perf_counter() - t0
    flops = flops_total / total_slices * threads
    return {"value": flops / dt / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": "port",
            "sample": f"slices [0,{threads}) of {total_slices}, one contiguous range per host thread, "
                      f"{dt:.1f} s wall, oracle complex64 executor (k-ascending row-panel GEMM)",
            "wall_s": dt, "host_cores": cores}


def run_reference(args, net, arrays, path, sliced, name, rank):
    """--impl reference: the reference's CPU executor path (oracle port) on the host cores."""
    if rank != 0:
        return
    import arctn_b200 as A

    total = 2 ** len(sliced)
    sub = dict(net.size_dict)
    for l in sliced:
        sub[l] = 1
    macs = sum(s.gemm_dims()[0] * s.gemm_dims()[1] * s.gemm_dims()[2] * s.gemm_dims()[3]
               for s in A.CompiledContraction.compile(net.inputs, net.output, sub, ssa_path=path).pair_steps())
    flops_total = 8.0 * macs * total
    vals = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(net, arrays, path, sliced, total, flops_total)
        if i >= args.warmup:
            vals.append(cb)
    v = statistics.median([c["value"] for c in vals])
    ms = statistics.median([c["wall_s"] for c in vals]) * 1e3
    cb = dict(vals[0])
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "TFLOP/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": name, "sample": cb["sample"]},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference Rust executor cannot be built here (no cargo/rustc, crates not vendored); "
                    "timed its CPU restatement"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    net, arrays, path, sliced, name = workload(args.nodes, args.target_log2)
    if args.impl == "reference":
        run_reference(args, net, arrays, path, sliced, name, rank)
        return

    import torch

    import arctn_b200 as A

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    total = 2 ** len(sliced)
    begin, end = slice_range(total, world, rank)
    prog = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision=args.precision,
                           device=local, use_graph=True, workspace_budget=100 << 30,
                           **({"slice_begin": begin, "slice_end": end} if world > 1 else {}))
    x = [torch.from_numpy(a).to(dev) for a in arrays]
    ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device=dev)
    out = torch.empty((), dtype=torch.complex128, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    # A non-default stream: the launch sequence is captured once and replayed as a CUDA graph.
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    def step():
        r = prog.execute(x, f64_out=True, workspace=ws, stream=stream)
        if dist is not None:
            dist.all_reduce(r)
        return r

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)  # L2 flush between timed iterations
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize(dev)
    total_ms = sum(times)
    if dist is not None:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    flops_all = prog.flops
    if dist is not None:
        f = torch.tensor([prog.flops], dtype=torch.float64, device=dev)
        dist.all_reduce(f)
        flops_all = float(f.item())
    ms_per_step = total_ms / args.steps
    value = flops_all / (ms_per_step * 1e-3) / 1e12
    clocks = clk.summary()

    # End-to-end through the public API: host (NumPy) inputs copied in, the scalar result copied out.
    e2e = None
    if world == 1:
        host_in = [np.ascontiguousarray(a) for a in arrays]
        prog.execute(host_in)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            res = prog.execute(host_in)
        e2e_s = (time.perf_counter() - t0) / args.steps
        e2e = {"value": prog.flops / e2e_s / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": int(sum(a.nbytes for a in host_in)), "d2h_bytes_per_step": int(res.nbytes)}

    # Roofline of the dominant kernel from a profiled (op-by-op, CUDA-event) run.
    roof = None
    pk = peaks()
    if not args.no_profile:
        ms, kinds, work = prog.profile(x, workspace=ws)
        by = {}
        for t_, k_, w_ in zip(ms, kinds, work):
            d = by.setdefault(int(k_), [0.0, 0.0, 0])
            d[0] += float(t_)
            d[1] += float(w_)
            d[2] += 1
        top = max(by, key=lambda k: by[k][0])
        tms, tw, tn = by[top]
        if top in GEMM_KINDS:
            achieved = tw / (tms * 1e-3) / 1e12
            roof = {"bound": "tensor", "kernel": KIND_NAMES.get(top, str(top)), "achieved": achieved,
                    "peak": pk["bf16_tflops"], "unit": "TFLOP/s", "frac": achieved / pk["bf16_tflops"],
                    "peak_source": f"{pk['source']} bf16 dense (burst)", "traffic": None, "launches": tn,
                    "avg_launch_ms": tms / tn, "share_of_profiled_time": tms / max(sum(v[0] for v in by.values()), 1e-9)}
        else:
            achieved = tw / (tms * 1e-3) / 1e9
            roof = {"bound": "hbm", "kernel": KIND_NAMES.get(top, str(top)), "achieved": achieved,
                    "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                    "peak_source": f"{pk['source']} HBM copy", "traffic": None, "launches": tn,
                    "avg_launch_ms": tms / tn}
        roof["kernels"] = {KIND_NAMES.get(k, str(k)): {"ms": v[0], "launches": v[2]} for k, v in sorted(by.items())}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(net, arrays, path, sliced, total, prog.flops)
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "c64", "data": "synthetic",
                "config": {"workload": name, "n_nodes": args.nodes, "bond": 2, "graph_seed": 1,
                           "target_size": 2 ** args.target_log2, "n_slices": total,
                           "slices_per_group": prog.slices_per_group, "precision": args.precision,
                           "cross_slice_sum": "fp64", "l2": "flushed (256 MiB write) between timed iterations",
                           "parallelism": f"slice-sharded x{world}"},
                "gpu_launches": prog.launches * args.steps, "e2e": e2e, "roofline": roof, "cpu_baseline": cpu,
                "clocks": clocks, "result": [float(r.real), float(r.imag)] if hasattr(r, "real") else None}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

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
every slice (the reference's per-slice work x n_slices).  The headline runs
the split-TF32 tensor-core path; the same line reports the plain-FP32 form's
TFLOP/s and both results' relative error against an FP64 contraction.

    python bench.py [--gpus N --steps K --warmup W] [--impl b200|reference] [--precision tf32x3|fp32]

Under torchrun each rank contracts a contiguous range of slices (the
reference's MPI slice_range, src/bin/tnmpi.rs:279-284) and one NCCL
all-reduce sums the FP64 partial outputs; the printed value is total flops
over the max-over-ranks device time.
"""

from __future__ import annotations

import argparse
import datetime
import json
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
              4: "k_slice_accumulate", 5: "k_slice_output", 7: "k_maxabs", 8: "k_strip_scale",
              9: "k_tc_cgemm_tf32x3", 10: "k_gemm_dot", 11: "k_pack_planar"}
GEMM_KINDS = {1, 2, 3, 9, 10}


def parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--precision", choices=["fp32", "tf32x3"], default="tf32x3")
    ap.add_argument("--nodes", type=int, default=172)
    ap.add_argument("--target-log2", type=int, default=24)
    ap.add_argument("--group", type=int, default=0, help="slices per group (0: as many as the workspace allows)")
    ap.add_argument("--workspace-gb", type=float, default=24.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-profile", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip e2e, the FP32 comparison and the FP64 check")
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


def profiled_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "k_tc_cgemm_tf32x3_rand3reg_n172.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_full_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


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


def per_slice_flops(net, path, sliced):
    import arctn_b200 as A

    sub = dict(net.size_dict)
    for leg in sliced:
        sub[leg] = 1
    cc = A.CompiledContraction.compile(net.inputs, net.output, sub, ssa_path=path)
    return 8.0 * sum(a * b * c * d for a, b, c, d in (s.gemm_dims() for s in cc.pair_steps()))


def cpu_baseline(net, arrays, path, sliced, total_slices, flops_total, threads=None):
    """The oracle (CPU restatement of the reference executor) on a bounded sample of slices."""
    from oracle import oracle as O

    O.build()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    threads = threads or max(1, min(cores, 32, total_slices))
    t0 = time.perf_counter()
    O.contract_slice_range(*net.as_tuple(), path, sliced, 0, threads, arrays, threads=threads)
    dt = time.perf_counter() - t0
    flops = flops_total / total_slices * threads
    return {"value": flops / dt / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": "port",
            "sample": f"slices [0,{threads}) of {total_slices}, one slice per host thread, {dt:.1f} s wall; "
                      "oracle complex64 executor (reference step algorithm, k-ascending row-panel GEMM)",
            "wall_s": dt, "host_cores": cores}


def run_reference(args, net, arrays, path, sliced, name, rank):
    """--impl reference: the reference's CPU executor path (its oracle restatement) on the host cores."""
    if rank != 0:
        return
    total = 2 ** len(sliced)
    flops_total = per_slice_flops(net, path, sliced) * total
    from oracle import oracle as O
    from arctn_b200 import networks as N

    small, small_arrays = N.workload_rand3reg(64, 2, 1, np.complex64, seed=0)
    spath = O.greedy(*small.as_tuple())
    for _ in range(args.warmup):  # warm-up: load the library and touch the allocator on a small contraction
        O.contract_sliced(*small.as_tuple(), spath, [], small_arrays)
    vals = [cpu_baseline(net, arrays, path, sliced, total, flops_total) for _ in range(args.steps)]
    v = statistics.median([c["value"] for c in vals])
    ms = statistics.median([c["wall_s"] for c in vals]) * 1e3
    cb = dict(vals[0])
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "TFLOP/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": name, "sample": cb["sample"]},
            "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": cb["cores"], "kind": "port",
                             "sample": cb["sample"]},
            "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference Rust executor cannot be built in this image (no cargo/rustc, crates not "
                    "vendored); its CPU restatement (oracle/) is timed instead"}
    print(json.dumps(line), flush=True)


def timed(prog, x, ws, stream, steps, warmup, dist, dev, flush, clock=None):
    import torch

    def step():
        r = prog.execute(x, f64_out=True, workspace=ws, stream=stream)
        if dist is not None:
            dist.all_reduce(r)
        return r

    for _ in range(warmup):
        step()
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    times = []
    r = None
    sampler = ClockSampler(dev.index) if clock else None
    if sampler:
        sampler.__enter__()
    try:
        for _ in range(steps):
            flush.fill_(1)  # L2 flush between timed iterations (inputs are smaller than L2)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    finally:
        if sampler:
            sampler.__exit__(None, None, None)
    torch.cuda.synchronize(dev)
    total_ms = sum(times)
    if dist is not None:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    return total_ms / steps, r, (sampler.summary() if sampler else None)


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
    common = dict(dtype=np.complex64, device=local, use_graph=True, workspace_budget=int(args.workspace_gb * (1 << 30)),
                  max_slices_per_group=args.group)
    if world > 1:
        common.update(slice_begin=begin, slice_end=end)
    prog = A.SlicedProgram(*net.as_tuple(), path, sliced, precision=args.precision, **common)
    x = [torch.from_numpy(a).to(dev) for a in arrays]
    ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    # A non-default stream: the launch sequence is captured once and replayed as a CUDA graph.
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    ms_per_step, r, clocks = timed(prog, x, ws, stream, args.steps, args.warmup, dist, dev, flush, clock=True)
    status = prog.device_status(ws, stream)
    flops_all = prog.flops
    if dist is not None:
        f = torch.tensor([prog.flops], dtype=torch.float64, device=dev)
        dist.all_reduce(f)
        flops_all = float(f.item())
    value = flops_all / (ms_per_step * 1e-3) / 1e12

    extras = {}
    e2e = None
    if world == 1 and not args.no_extras:
        # End to end through the public API: host (NumPy) inputs copied in, the scalar result copied out.
        host_in = [np.ascontiguousarray(a) for a in arrays]
        prog.execute(host_in)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            res = prog.execute(host_in)
        e2e_s = (time.perf_counter() - t0) / args.steps
        e2e = {"value": prog.flops / e2e_s / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": int(sum(a.nbytes for a in host_in)), "d2h_bytes_per_step": int(res.nbytes)}
        # The plain FP32 GPU form on the same workload, and both results against an FP64 contraction.
        other = "fp32" if args.precision == "tf32x3" else "tf32x3"
        prog2 = A.SlicedProgram(*net.as_tuple(), path, sliced, precision=other, **common)
        ws2 = torch.empty(max(prog2.workspace_bytes, 1), dtype=torch.uint8, device=dev)
        ms2, r2, _ = timed(prog2, x, ws2, stream, max(1, min(args.steps, 2)), 1, None, dev, flush)
        del ws2, prog2
        c64 = dict(common)
        c64["dtype"] = np.complex128
        prog64 = A.SlicedProgram(*net.as_tuple(), path, sliced, precision="fp32", **c64)
        x64 = [t.to(torch.complex128) for t in x]
        ws64 = torch.empty(max(prog64.workspace_bytes, 1), dtype=torch.uint8, device=dev)
        ref = complex(prog64.execute(x64, workspace=ws64, stream=stream).item())
        del ws64, prog64
        rel = lambda v: abs(complex(v) - ref) / abs(ref)  # noqa: E731
        extras = {"other_precision": other, "other_value": prog.flops / (ms2 * 1e-3) / 1e12,
                  "speedup_vs_other": ms2 / ms_per_step, "rel_err_vs_fp64": rel(r.item()),
                  "other_rel_err_vs_fp64": rel(r2.item()), "fp64_result": [ref.real, ref.imag]}

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
        tot = max(sum(v[0] for v in by.values()), 1e-9)
        top = max(by, key=lambda k: by[k][0])
        tms, tw, tn = by[top]
        if top in GEMM_KINDS:
            achieved = tw / (tms * 1e-3) / 1e12
            roof = {"bound": "tensor", "kernel": KIND_NAMES.get(top, str(top)), "achieved": achieved,
                    "peak": pk["bf16_tflops"], "unit": "TFLOP/s", "frac": achieved / pk["bf16_tflops"],
                    "peak_source": f"{pk['source']} bf16 dense burst (MEASURED_PEAKS.json)",
                    "traffic": profiled_traffic(), "launches": tn, "avg_launch_ms": tms / tn,
                    "share_of_profiled_time": tms / tot}
            if top == 9:
                # split-TF32 4M: 12 TF32 MMAs per complex MAC step = 24 pipe flops per 8 algorithmic flops;
                # TF32 dense rate taken as half the measured bf16 rate.
                tf32_peak = pk["bf16_tflops"] / 2
                roof["pipe_tflops"] = achieved * 3
                roof["pipe_frac_of_tf32_peak"] = achieved * 3 / tf32_peak
        else:
            achieved = tw / (tms * 1e-3) / 1e9
            roof = {"bound": "hbm", "kernel": KIND_NAMES.get(top, str(top)), "achieved": achieved,
                    "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                    "peak_source": f"{pk['source']} HBM copy", "traffic": None, "launches": tn,
                    "avg_launch_ms": tms / tn}
        roof["kernels"] = {KIND_NAMES.get(k, str(k)): {"ms": round(v[0], 3), "launches": v[2],
                                                       "share": round(v[0] / tot, 4)} for k, v in sorted(by.items())}

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
                "clocks": clocks, "device_status": status, "workspace_bytes": int(prog.workspace_bytes),
                "result": [float(r.real), float(r.imag)]}
        line.update(extras)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

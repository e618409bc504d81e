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
the split-TF32 tensor-core path with its GEMM kernels autotuned before timing;
the same line reports the plain-FP32 form's TFLOP/s, both results' relative
error against an FP64 contraction, the oracle on a slice sample, the staged
scheduler's form, the roofline per tensor-core step and, under `configs`, the
other configurations (grid6, rand3reg n=64, brickwork, grid8, the 256-network
batch), each also available alone through --workload.

    python bench.py [--gpus N --steps K --warmup W] [--impl b200|reference] [--precision tf32x3|fp32|bf16x3|bf16x6]

Under torchrun each rank contracts a contiguous range of slices (the
reference's MPI slice_range, src/bin/tnmpi.rs:279-284) and one NCCL
all-reduce sums the FP64 partial outputs; the printed value is total flops
over the max-over-ranks device time.
"""

from __future__ import annotations

import argparse
import datetime
import contextlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "c64 sliced TN contraction TFLOP/s"
KIND_NAMES = {0: "k_gather_reduce", 1: "k_gemm_small", 2: "k_gemm_tile<64,64>", 3: "k_gemm_tile<32,32>",
              4: "k_slice_accumulate", 5: "k_slice_output", 7: "k_maxabs", 8: "k_strip_scale",
              9: "k_tc_cgemm_tf32x3", 10: "k_gemm_dot", 11: "k_pack_planar", 12: "k_scatter", 13: "k_pack_tiled",
              14: "k_gemm_warp"}
GEMM_KINDS = {1, 2, 3, 9, 10, 14}


def parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--precision", choices=["fp32", "tf32x3", "bf16x3", "bf16x6"], default="tf32x3")
    ap.add_argument("--nodes", type=int, default=172)
    ap.add_argument("--target-log2", type=int, default=24)
    ap.add_argument("--group", type=int, default=0, help="slices per group (0: as many as the workspace allows)")
    ap.add_argument("--workspace-gb", type=float, default=24.0)
    ap.add_argument("--tc-k-chunk", type=int, default=0, help="K per tensor-core accumulator (0: library default)")
    ap.add_argument("--no-tune", action="store_true", help="keep the built-in GEMM heuristics (skip the autotuner)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations (grid6, brickwork, grid8, batch) after the headline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-profile", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip e2e, the FP32 comparison and the FP64 check")
    ap.add_argument("--batch-size", type=int, default=256, help="networks of --workload batch (256: config 5)")
    ap.add_argument("--workload", choices=["rand3reg", "rand3reg_n64", "grid6", "brickwork", "grid8", "batch"],
                    default="rand3reg",
                    help="rand3reg: the sliced headline (default); rand3reg_n64: 256 slices of the n=64 graph in "
                         "one persistent launch; grid6 / brickwork: latency and precision; grid8: forward + adjoint; "
                         "batch: 256 uneven networks in one graph launch")
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


def per_step_roofline(prog, ms, tf32_pipe_tflops, hbm_gbs, sustained_tflops=None):
    """Each tensor-core GEMM shape of the program against its own bound, from the op-by-op profile `ms`:
    the tensor bound is its split-TF32 pipe work (3 TF32 products per real product) at the measured TF32 rate,
    the memory bound its algorithmic bytes (16 B per packed operand element read, 16 B per packed or 8 B per
    plain output element written) at the HBM rate; the step's bound is the larger of the two times.  With
    `sustained_tflops` (the TF32 rate held for seconds under the power cap, on random operands) each step
    also carries its tensor work against that rate."""
    ops = prog.describe()["ops"]
    units = {}
    for i, o in enumerate(ops):
        units.setdefault(o.get("unit", i), []).append(o)
    order = [u for u in sorted(units) if units[u][0]["kind"] != "memset"]
    agg = {}
    for u, t in zip(order, ms):
        o = units[u][0]
        if o["kind"] != "gemm_tc":
            continue
        S, bt, m, k, n = o["S"], o["bt"], o["m"], o["k"], o["n"]
        a = agg.setdefault((m, k, n), {"ms": 0.0, "flops": 0.0, "bytes": 0.0, "launches": 0,
                                       "fused_output": "pack_into" in o})
        a["ms"] += float(t)
        a["launches"] += 1
        a["flops"] += 8.0 * S * bt * m * k * n
        a["bytes"] += 16.0 * bt * ((S if o["a_var"] else 1) * m * k + (S if o["b_var"] else 1) * k * n) + \
            (16.0 if "pack_into" in o else 8.0) * S * bt * m * n
    out = []
    for (m, k, n), a in sorted(agg.items(), key=lambda kv: -kv[1]["ms"]):
        t_tensor = 3 * a["flops"] / (tf32_pipe_tflops * 1e12) * 1e3
        t_mem = a["bytes"] / (hbm_gbs * 1e9) * 1e3
        out.append({"m_k_n": [m, k, n], "ms": round(a["ms"], 3), "launches": a["launches"],
                    "fused_output": a["fused_output"], "tflops": a["flops"] / (a["ms"] * 1e-3) / 1e12,
                    "gbs": a["bytes"] / (a["ms"] * 1e-3) / 1e9, "bound": "tensor" if t_tensor >= t_mem else "hbm",
                    "frac_of_bound": max(t_tensor, t_mem) / a["ms"]})
        if sustained_tflops:
            out[-1]["tensor_frac_of_sustained"] = 3 * a["flops"] / (sustained_tflops * 1e12) * 1e3 / a["ms"]
    return out


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
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="arctn_b200_clocks_", suffix=".csv")
            self.f = os.fdopen(fd, "w")
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
        if not self.proc or not self.path or not os.path.exists(self.path):
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
        try:
            os.unlink(self.path)
        except OSError:
            pass
        self.path = None
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def per_slice_flops(net, path, sliced):
    import arctn_b200 as A

    sub = dict(net.size_dict)
    for leg in sliced:
        sub[leg] = 1
    cc = A.CompiledContraction.compile(net.inputs, net.output, sub, ssa_path=path)
    return 8.0 * sum(a * b * c * d for a, b, c, d in (s.gemm_dims() for s in cc.pair_steps()))


def load_networks():
    """The synthetic network generators (pure NumPy) loaded from their file, without importing the
    arctn_b200 package: the reference arm must not load the product library."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("_bench_networks", os.path.join(ROOT, "arctn_b200", "networks.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # dataclasses resolve annotations through sys.modules
    spec.loader.exec_module(mod)
    return mod


def oracle_workload(n_nodes, target_log2):
    """The headline workload planned by the oracle alone: its greedy path, slice search and flop count."""
    from oracle import oracle as O

    N = load_networks()
    net, arrays = N.workload_rand3reg(n_nodes, 2, 1, np.complex64, seed=0)
    path = O.greedy(*net.as_tuple())
    sliced = O.find_slices_to_size(*net.as_tuple(), path, 2 ** target_log2)
    if sliced is None:
        raise SystemExit("no slicing meets the target")
    sub = dict(net.size_dict)
    for leg in sliced:
        sub[leg] = 1
    plan = O.plan_json(net.inputs, net.output, sub, path)
    flops = 8.0 * sum(a * b * c * d for a, b, c, d in (st["gemm_dims"] for st in plan["steps"]))
    name = f"rand3reg_n{n_nodes}_bond2_seed1_c64_greedy_target2^{target_log2}_{2 ** len(sliced)}slices"
    return net, arrays, path, sliced, name, flops


def product_library_loaded():
    """Whether this process has mapped the product library (read from /proc/self/maps)."""
    try:
        with open("/proc/self/maps") as f:
            return any("libarctn_b200" in line for line in f)
    except OSError:
        return None


def host_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def cpu_baseline(net, arrays, path, sliced, total_slices, flops_total, threads=None):
    """The oracle (CPU restatement of the reference executor) on a bounded sample of slices."""
    from oracle import oracle as O

    O.build()
    cores = host_threads()
    threads = threads or max(1, min(cores, 64, total_slices))
    t0 = time.perf_counter()
    part = O.contract_slice_range(*net.as_tuple(), path, sliced, 0, threads, arrays, threads=threads)
    dt = time.perf_counter() - t0
    flops = flops_total / total_slices * threads
    return {"value": flops / dt / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": "port",
            "sample": f"slices [0,{threads}) of {total_slices}, one slice per host thread, {dt:.1f} s wall; "
                      "oracle complex64 executor (reference step algorithm, register-blocked k-ascending GEMM)",
            "wall_s": dt, "host_cores": cores, "partial": complex(np.asarray(part).sum())}


def numpy_tensordot_baseline(net, arrays, path, sliced, total_slices, flops_total, budget_s=10.0, max_slices=16):
    """A second CPU reference point: NumPy, one ``tensordot`` (BLAS) per pairwise step of the same plan, as the
    reference paper's NumPy executor does.  Slices 0, 1, ... of the sliced contraction run until about
    ``budget_s`` seconds have passed; inputs are narrowed along the sliced legs (last sliced leg fastest,
    src/slice.rs:881-888) and each step applies its dangling sums, contracts its shared legs and permutes the
    result to the plan's leg order (src/compiled.rs:155-171)."""
    import arctn_b200 as A

    sub = dict(net.size_dict)
    for leg in sliced:
        sub[leg] = 1
    cc = A.CompiledContraction.compile(net.inputs, net.output, sub, ssa_path=path)
    if any(not p.is_identity() for p in cc.input_preps()):  # traces / diagonals: not this executor's form
        return None
    dims = [net.size_dict[leg] for leg in sliced]

    def one_slice(si):
        digits = {}
        for leg, d in zip(reversed(sliced), reversed(dims)):
            digits[leg] = si % d
            si //= d
        slots = []
        for legs, a in zip(net.inputs, arrays):
            idx = tuple(slice(digits[l], digits[l] + 1) if l in digits else slice(None) for l in legs)
            slots.append(a[idx])
        for st in cc.pair_steps():
            a, b = slots[st.left_slot()], slots[st.right_slot()]
            wa, wb = list(st.left_legs()), list(st.right_legs())
            for ax in st.sum_a():
                a = a.sum(axis=ax)
                del wa[ax]
            for ax in st.sum_b():
                b = b.sum(axis=ax)
                del wb[ax]
            out = list(st.result_legs())
            con = [l for l in wa if l in wb and l not in out]
            if any(l in wb and l in out for l in wa):  # batch legs: no tensordot form
                letters = {l: chr(97 + i) for i, l in enumerate(dict.fromkeys(wa + wb))}
                spec = "".join(letters[l] for l in wa) + "," + "".join(letters[l] for l in wb) + "->" + \
                       "".join(letters[l] for l in out)
                c = np.einsum(spec, a, b, optimize=True)
            else:
                c = np.tensordot(a, b, axes=([wa.index(l) for l in con], [wb.index(l) for l in con]))
                got = [l for l in wa if l not in con] + [l for l in wb if l not in con]
                c = c.transpose([got.index(l) for l in out]).copy()  # contiguous, 0-d stays 0-d
            slots.append(c)
        fin = cc.finalize()
        r = slots[fin.slot()]
        for ax in fin.sum_axes():
            r = r.sum(axis=ax)
        return np.transpose(r, fin.perm()).astype(np.complex128)

    one_slice(0)  # warm-up: BLAS threads and page faults
    t0 = time.perf_counter()
    n = 0
    acc = 0
    while n < min(max_slices, total_slices) and (n == 0 or time.perf_counter() - t0 < budget_s):
        acc = acc + one_slice(n)
        n += 1
    dt = time.perf_counter() - t0
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    return {"value": flops_total / total_slices * n / dt / 1e12, "unit": "TFLOP/s", "cores": cores,
            "kind": "numpy", "sample": f"slices [0,{n}) of {total_slices} in sequence, {dt:.1f} s wall; NumPy "
                                       f"{np.__version__} tensordot per step on the host BLAS threads",
            "partial_sum": [float(np.real(acc).sum()), float(np.imag(acc).sum())]}


def run_reference(args, rank):
    """--impl reference: the reference's CPU executor path (its oracle restatement) on the host cores.

    Planning (greedy path, slice search), the flop count and the contraction all come from the oracle;
    the product library is never loaded in this process.  Each step contracts a bounded sample of the
    slices (one per host thread) and the rate is that sample's flops over its wall time."""
    if rank != 0:
        return
    from oracle import oracle as O

    O.build()
    net, arrays, path, sliced, name, per_slice = oracle_workload(args.nodes, args.target_log2)
    total = 2 ** len(sliced)
    flops_total = per_slice * total
    N = load_networks()
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
            "config": {"workload": name, "n_nodes": args.nodes, "bond": 2, "graph_seed": 1,
                       "target_size": 2 ** args.target_log2, "n_slices": total, "precision": "fp32 (CPU)",
                       "cross_slice_sum": "in the input dtype, the reference's chunk order",
                       "sample": cb["sample"], "planned_by": "oracle greedy + find_slices_to_size"},
            "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": cb["cores"], "kind": "port",
                             "sample": cb["sample"]},
            "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference Rust executor cannot be built in this image (no cargo/rustc, crates not "
                    "vendored); its CPU restatement (oracle/) is timed instead, on a sample of slices",
            "product_library_loaded": product_library_loaded()}
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


# ---------------------------------------------------------------------------------------------------
# Other measured configurations (--workload).  Each prints one JSON line with the same base keys.


def _line(args, metric, value, unit, hib, ms, config, dtype, **extra):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
         "ms_per_step": ms, "higher_is_better": hib, "scaling": "none", "vs_baseline": None, "dtype": dtype,
         "data": "synthetic", "config": config}
    d.update(extra)
    return d


def _events_ms(stream, fn):
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def _cpu_time(fn, reps):
    fn()
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return statistics.median(ts)


def run_latency(args, dev, which):
    """grid6 (6x6 grid, bond 4, c128) or brickwork (30 wires x depth 14, c64): microseconds per contraction,
    plus the precision study (split-TF32 / FP32 / split-BF16 / FP64 on the GPU, the FP32 CPU executor) for
    brickwork."""
    import torch

    import arctn_b200 as A
    from arctn_b200 import networks as N
    from oracle import oracle as O

    if which == "grid6":
        net, arrays = N.workload_grid6(np.complex128, seed=0)
        dtype, precisions = np.complex128, ["fp32"]
    else:
        net, arrays = N.brickwork_circuit(30, 14, seed=0)
        arrays = [a.astype(np.complex64) for a in arrays]
        dtype, precisions = np.complex64, ["tf32x3", "fp32", "bf16x3", "bf16x6"]
    path = A.greedy(*net.as_tuple())
    O.build()
    ref = complex(O.contract_sliced(*net.as_tuple(), path, [], [a.astype(np.complex128) for a in arrays]))
    cpu_native = complex(O.contract_sliced(*net.as_tuple(), path, [], arrays))
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    x = [torch.from_numpy(a).to(dev) for a in arrays]
    res = {}
    for prec in precisions:
        prog = A.SlicedProgram(*net.as_tuple(), path, (), dtype=dtype, precision=prec, device=dev.index)
        ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device=dev)
        out = torch.empty(prog.output_shape, dtype=torch.complex128 if dtype == np.complex128 else torch.complex64,
                          device=dev)
        launch = prog.bind(x, out, ws, stream)  # one C-ABI call (graph replay) per contraction
        for _ in range(max(args.warmup, 3)):
            launch()
        torch.cuda.synchronize(dev)
        times, api = [], []
        sampler = ClockSampler(dev.index)
        with sampler:
            for _ in range(args.steps):
                flush.fill_(1)  # L2 flush between timed contractions
                times.append(_events_ms(stream, launch))
        for _ in range(args.steps):  # the full Python API call, validation and marshalling included
            flush.fill_(1)
            api.append(_events_ms(stream, lambda: prog.execute(x, workspace=ws, stream=stream, out=out)))
        got = complex(out.item())
        res[prec] = {"us": 1e3 * statistics.mean(times), "us_p50": 1e3 * statistics.median(times),
                     "python_api_us": 1e3 * statistics.mean(api),
                     "rel_err_vs_fp64": abs(got - ref) / abs(ref), "launches": prog.launches, "flops": prog.flops,
                     "clocks": sampler.summary()}
    if dtype == np.complex64:
        c128 = A.SlicedProgram(*net.as_tuple(), path, (), dtype=np.complex128, device=dev.index)
        g64 = complex(c128.execute([t.to(torch.complex128) for t in x]).item())
        res["fp64_gpu_rel_err_vs_oracle"] = abs(g64 - ref) / abs(ref)
    head = precisions[0]
    host_in = [np.ascontiguousarray(a) for a in arrays]
    prog = A.SlicedProgram(*net.as_tuple(), path, (), dtype=dtype, precision=head, device=dev.index)
    prog.execute(host_in)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = prog.execute(host_in)
    e2e_us = (time.perf_counter() - t0) / args.steps * 1e6
    cpu_s = _cpu_time(lambda: O.contract_sliced(*net.as_tuple(), path, [], arrays), 5)
    name = "grid6x6_bond4_c128" if which == "grid6" else "brickwork_30x14_c64"
    line = _line(args, f"{name} contraction latency", res[head]["us"], "us", False, res[head]["us"] / 1e3,
                 {"workload": name, "n_tensors": len(net.inputs), "steps_in_path": len(path),
                  "precision": head, "l2": "flushed (256 MiB write) before each timed contraction"},
                 "c128" if dtype == np.complex128 else "c64",
                 gpu_launches=res[head]["launches"] * args.steps,
                 e2e={"value": e2e_us, "unit": "us", "h2d_bytes_per_step": int(sum(a.nbytes for a in host_in)),
                      "d2h_bytes_per_step": int(np.asarray(r).nbytes)},
                 roofline={"bound": "latency", "note": "launch/latency-bound: a few microseconds of work per step"},
                 cpu_baseline={"value": cpu_s * 1e6, "unit": "us", "cores": 1, "kind": "port",
                               "sample": "one full contraction, median of 5, oracle executor in the input dtype"},
                 clocks=res[head]["clocks"], precisions=res, fp64_oracle=[ref.real, ref.imag],
                 cpu_native_rel_err_vs_fp64=abs(cpu_native - ref) / abs(ref))
    return line


def run_grid8(args, dev):
    """8x8 grid, bond 6, c64: forward + adjoint (gradients of all 64 inputs) on the tensor cores."""
    import torch

    import arctn_b200 as A
    from arctn_b200 import networks as N

    net, arrays = N.workload_grid8(6, np.complex64, seed=0)
    arrays = [a * np.float32(4.0) for a in arrays]  # lifts the ~1e-35 scalar off FP32's underflow range
    path = A.greedy(*net.as_tuple())
    x = [torch.from_numpy(a).to(dev) for a in arrays]
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def measure(prog):
        ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device=dev)
        out = torch.empty((), dtype=torch.complex64, device=dev)
        g_out = torch.ones((), dtype=torch.complex64, device=dev)
        for _ in range(max(args.warmup, 3)):
            prog.gradient(x, g_out, part=1, workspace=ws, output=out, stream=stream)
            prog.gradient(x, g_out, part=2, workspace=ws, stream=stream)
        torch.cuda.synchronize(dev)
        f, b = [], []
        sampler = ClockSampler(dev.index)
        with sampler:
            for _ in range(args.steps):
                flush.fill_(1)
                f.append(_events_ms(stream, lambda: prog.gradient(x, g_out, part=1, workspace=ws, output=out,
                                                                  stream=stream)))
                b.append(_events_ms(stream, lambda: prog.gradient(x, g_out, part=2, workspace=ws, stream=stream)))
        return statistics.mean(f), statistics.mean(b), sampler.summary(), ws

    kw = dict(gradient=True, use_graph=False, device=dev.index)
    # The autotuner times every GEMM variant inside the gradient program (forward and adjoint GEMMs alike).
    tuning, tune_info = None, None
    if not args.no_tune:
        t0 = time.perf_counter()
        tuning = A.autotune(*net.as_tuple(), path, (), dtype=np.complex64, precision="tf32x3",
                            workspace_budget=40 << 30, **kw)
        tune_info = {"tune_s": round(time.perf_counter() - t0, 1), "gemm_shapes": len(tuning),
                     "changed_from_heuristic": sum(tuning.get(k) != tuning.timings(k).get("heuristic")
                                                   for k in tuning.keys()),
                     "program_ms": {"heuristics": tuning.meta.get("program_ms_before"),
                                    "tuned": tuning.meta.get("program_ms_after")}}
    p = A.SlicedProgram(*net.as_tuple(), path, (), dtype=np.complex64, precision="tf32x3", workspace_budget=40 << 30,
                        tuning=tuning, **kw)
    fwd_ms, bwd_ms, clocks, ws = measure(p)
    status = p.device_status(ws)
    del ws
    o_tc, g_tc = p.gradient(x)
    p64 = A.SlicedProgram(*net.as_tuple(), path, (), dtype=np.complex128, workspace_budget=40 << 30, **kw)
    o64, g64 = p64.gradient([t.to(torch.complex128) for t in x])
    pf = A.SlicedProgram(*net.as_tuple(), path, (), dtype=np.complex64, precision="fp32", workspace_budget=40 << 30,
                         **kw)
    o32, g32 = pf.gradient(x)
    ref = complex(o64.item())

    def norm_err(gs):
        return max(float(torch.linalg.norm(a.to(torch.complex128) - b) / torch.linalg.norm(b)) for a, b in zip(gs, g64))

    fwd32, bwd32, _, ws32 = measure(pf)
    del ws32
    del p64, pf
    # Op-by-op event profile of forward + reverse: where each sweep's time goes, per kernel kind.
    desc = p.describe()
    n_fwd = sum(1 for o in desc["ops"][: desc["backward_begin"]] if o["kind"] != "memset")
    ms_ops, kinds, _ = p.profile(x)
    sweep = {"forward": {}, "backward": {}}
    for i, (t, k) in enumerate(zip(ms_ops, kinds)):
        d = sweep["forward" if i < n_fwd else "backward"].setdefault(KIND_NAMES.get(int(k), str(k)), [0, 0.0])
        d[0] += 1
        d[1] = round(d[1] + float(t), 3)
    # Lowered budget: half the layout that keeps every intermediate -> the sweep recomputes.
    pr = A.SlicedProgram(*net.as_tuple(), path, (), dtype=np.complex64, precision="tf32x3",
                         workspace_budget=p.workspace_bytes // 2, tuning=tuning, **kw)
    fwd_r, bwd_r, _, wsr = measure(pr)
    o_r, g_r = pr.gradient(x, workspace=wsr)
    identical = bool(torch.equal(o_r, o_tc)) and all(torch.equal(a, b) for a, b in zip(g_r, g_tc))
    del wsr
    flops_fwd = p.flops
    total_ms = fwd_ms + bwd_ms
    value = 3 * flops_fwd / (total_ms * 1e-3) / 1e12  # forward F + two adjoint GEMMs per step (2F)
    # split-TF32 4M: 3 TF32 products per real product; the TF32 pipe rate measured by the library's probe
    tf32_pipe = max(A.tensor_pipe_peak("tf32", n, device=dev.index) for n in (128, 256))
    tf32_alg_peak = tf32_pipe / 3
    line = _line(args, "grid8 bond6 c64 forward+adjoint TFLOP/s", value, "TFLOP/s", True, total_ms,
                 {"workload": "grid8x8_bond6_c64_adjoint", "precision": "tf32x3", "inputs_scaled_by": 4,
                  "l2": "flushed (256 MiB write) before each timed part", "tuning": tune_info}, "c64",
                 gpu_launches=p.launches * args.steps,
                 e2e=None,
                 roofline={"bound": "tensor", "achieved": value, "peak": tf32_alg_peak, "unit": "TFLOP/s",
                           "frac": value / tf32_alg_peak,
                           "peak_source": "measured TF32 tensor pipe (arctn_b200_tc_peak) / 3 (split-TF32 products)",
                           "tf32_pipe_tflops": tf32_pipe, "traffic": None},
                 cpu_baseline=None, clocks=clocks, device_status=status,
                 fwd_ms=fwd_ms, bwd_ms=bwd_ms, bwd_over_fwd=bwd_ms / fwd_ms,
                 fp32_fwd_ms=fwd32, fp32_bwd_ms=bwd32, speedup_vs_fp32=(fwd32 + bwd32) / total_ms,
                 rel_err_scalar_vs_c128=abs(complex(o_tc.item()) - ref) / abs(ref),
                 fp32_rel_err_scalar_vs_c128=abs(complex(o32.item()) - ref) / abs(ref),
                 grad_norm_rel_err_max_vs_c128=norm_err(g_tc), fp32_grad_norm_rel_err_max_vs_c128=norm_err(g32),
                 workspace_bytes=p.workspace_bytes,
                 sweep_profile_ms=sweep,
                 recompute={"workspace_bytes": pr.workspace_bytes, "recomputed_steps": pr.recomputed_steps,
                            "fwd_ms": fwd_r, "bwd_ms": bwd_r, "bwd_over_fwd": bwd_r / fwd_r,
                            "bit_identical_to_kept": identical})
    return line


def run_rand3reg_n64(args, dev):
    """rand3reg n=64, bond 2, c64, greedy, sliced to 2^7 elements -> 256 slices (the configuration as written
    at n = 64; its stated 2^24 target needs no slicing): microseconds per sliced contraction as a graph of
    kernel launches and under the staged scheduler, where every slice runs inside one persistent launch."""
    import torch

    import arctn_b200 as A
    from arctn_b200 import networks as N
    from oracle import oracle as O

    net, arrays = N.workload_rand3reg(64, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 7)
    prog = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3", device=dev.index)
    x = [torch.from_numpy(a).to(dev) for a in arrays]
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device=dev)
    batch = A.ProgramBatch([prog], max_lanes=8, mode="staged")
    part = next(p for p in batch.describe()["parts"] if p["part"] == -1)
    run = batch.bind([x], stream=stream)
    forms = {"program": lambda: prog.execute(x, workspace=ws, stream=stream), "staged": run}
    res = {}
    sampler = ClockSampler(dev.index)
    with sampler:
        for name, fn in forms.items():
            for _ in range(max(args.warmup, 3)):
                fn()
            torch.cuda.synchronize(dev)
            ts = []
            for _ in range(max(args.steps, 10)):
                flush.fill_(1)
                ts.append(_events_ms(stream, fn))
            res[name] = 1e3 * statistics.mean(ts)
    got = complex(batch.execute([x], workspace=run.workspace, stream=stream)[0].item())
    want = complex(O.contract_sliced(*net.as_tuple(), path, sliced, O.promote(arrays), threads=8))
    return _line(args, "rand3reg n64 256-slice c64 contraction latency", res["staged"], "us", False,
                 res["staged"] / 1e3,
                 {"workload": "rand3reg_n64_bond2_seed1_c64_greedy_target2^7_256slices", "n_slices": 2 ** len(sliced),
                  "precision": "tf32x3", "form": "staged scheduler: one persistent interpreter launch for all slices",
                  "l2": "flushed (256 MiB write) before each timed contraction"}, "c64",
                 gpu_launches=(part["stages"] + sum(part["stage_launches"])) * max(args.steps, 10),
                 e2e=None, roofline={"bound": "latency", "note": "256 slices of 2^7-element steps"},
                 cpu_baseline=None, clocks=sampler.summary(), device_status=batch.device_status(run.workspace, stream),
                 interpreter_launches=part["stages"], tensor_core_launches=sum(part["stage_launches"]),
                 program_graph_us=res["program"], program_graph_launches=prog.launches,
                 rel_err_vs_fp64_oracle=abs(got - want) / abs(want))


def run_batch(args, dev):
    """256 uneven random 3-regular networks (half float32, half complex64): forward + adjoint of all of
    them as one graph launch; networks/s, TFLOP/s and the per-network latency distribution."""
    import torch

    import arctn_b200 as A
    from arctn_b200 import networks as N

    nets = N.workload_batch(args.batch_size, seed=0)
    paths = [A.greedy(*net.as_tuple()) for net, _ in nets]
    count = len(nets)
    world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        # The networks are independent: each rank runs its LPT share of the batch (balanced by flops) and the
        # only collective is the max over ranks of the device time.  Device-time line only.
        import torch.distributed as dist

        from arctn_b200.sharding import lpt_shard

        if count < world:
            raise SystemExit(f"--batch-size {count} is smaller than the {world} ranks")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
        costs = [10 ** A.simulate_path(*net.as_tuple(), p)["log10_flops"] for (net, _), p in zip(nets, paths)]
        mine = lpt_shard(costs, world)[rank]
        nets, paths = [nets[i] for i in mine], [paths[i] for i in mine]
        args.no_extras = True

    def build(tuning):
        return [A.SlicedProgram(*net.as_tuple(), path, (), dtype=arrays[0].dtype, precision="tf32x3", gradient=True,
                                use_graph=False, device=dev.index, tuning=tuning)
                for (net, arrays), path in zip(nets, paths)]

    progs = build(None)
    xs = [[torch.from_numpy(a).to(dev) for a in arrays] for _, arrays in nets]
    # One tuning table for the whole batch: the GEMM shapes of the networks with the most work (they set the
    # lane streams' time) are timed inside their own gradient programs; the other networks share the entries
    # whose shape keys they repeat.
    tune_info = None
    if not args.no_tune:
        t0 = time.perf_counter()
        table = A.TuneTable()
        order = sorted(range(len(progs)), key=lambda j: -progs[j].flops)[:8]
        for j in order:
            net, arrays = nets[j]
            A.autotune(*net.as_tuple(), paths[j], (), dtype=arrays[0].dtype, precision="tf32x3", gradient=True,
                       use_graph=False, table=table)
        progs = build(table)
        tune_info = {"tune_s": round(time.perf_counter() - t0, 1), "networks_tuned": len(order),
                     "gemm_shapes": len(table),
                     "gemms_pinned": sum(g["tuned"] for p in progs for g in p.gemms()),
                     "gemms_total": sum(len(p.gemms()) for p in progs)}
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def time_batch(batch, sampler=None):
        # Device time of the whole batch on resident inputs: the bound form allocates every output and
        # gradient once, so each timed call is one C-ABI call (a graph replay).
        run = batch.bind(xs, gradient=True, stream=stream)
        for _ in range(max(args.warmup, 3)):
            run()
        torch.cuda.synchronize(dev)
        times = []
        with sampler if sampler is not None else contextlib.nullcontext():
            for _ in range(args.steps):
                flush.fill_(1)
                times.append(_events_ms(stream, run))
        return statistics.mean(times), batch.device_status(run.workspace, stream)

    # The lane form (every step its own launch, networks spread over 128 streams) for comparison.
    lanes_ms, lanes_status = (None, 0) if args.no_extras else \
        time_batch(A.ProgramBatch(progs, max_lanes=128, mode="lanes"))
    batch = A.ProgramBatch(progs, max_lanes=128)
    sampler = ClockSampler(dev.index)
    ms, status = time_batch(batch, sampler)
    status = status or lanes_status
    if dist is not None:
        t = torch.tensor([ms, float(status)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, status = float(t[0].item()), int(t[1].item())
        dist.destroy_process_group()
    # Kernels per call: one interpreter launch per stage with tasks, the staged tensor-core steps and packs
    # (+1 for a split-K sum), every kernel of the lane programs, the status collection.
    desc = batch.describe(detail=True)
    part = next(p for p in desc["parts"] if p["part"] == 0)
    ops = [p.describe()["ops"] for p in progs]

    def kernels(o):
        return (o["kind"] != "memset") + (o["kind"] in ("gemm_tc", "gemm_dot") and o.get("splits", 1) > 1)

    staged = sum(kernels(ops[j][i]) for _, j, i in part["staged_launches"])
    interpreted = set(desc["interpreted"])
    lane_kernels = sum(kernels(o) for j in range(len(progs)) if j not in interpreted for o in ops[j])
    launches_per_call = 1 + sum(1 for t in part["stage_tasks"] if t) + staged + lane_kernels
    flops = sum(3 * p.flops for p in progs)
    # Per-network latency: each network's forward + adjoint alone (graph-free program launches).
    # End to end through the public API from host NumPy arrays: each call stages every network's inputs
    # (one pinned copy per network), runs the batch and returns outputs and gradients as NumPy arrays.
    host = [arrays for _, arrays in nets]
    if args.no_extras:  # device time only (profiling runs)
        return _line(args, "many-network forward+adjoint throughput", count / (ms * 1e-3),
                     "networks/s", True, ms, {"workload": f"{count} random 3-regular networks, n in "
                                              "[20,50], bond in {2,3,4}, f32/c64 alternating",
                                              "parallelism": f"LPT network shards x{world}"}, "f32+c64",
                     gpu_launches=launches_per_call * args.steps, e2e=None, roofline=None,
                     cpu_baseline=None, clocks=sampler.summary(), device_status=status, n_gpus=world,
                     scaling="strong" if world > 1 else "none")
    h2d = sum(a.nbytes for arrays in host for a in arrays)
    d2h = sum(int(np.prod(p.output_shape)) * a[0].itemsize for p, a in zip(progs, host)) + h2d
    ws_e2e = torch.empty(max(batch.workspace_bytes, 1), dtype=torch.uint8, device=dev)
    for _ in range(2):
        batch.gradient(host, workspace=ws_e2e, stream=stream)
    e2e_ms = []
    for _ in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        batch.gradient(host, workspace=ws_e2e, stream=stream)
        torch.cuda.synchronize(dev)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e = {"value": len(progs) / (statistics.median(e2e_ms) * 1e-3), "unit": "networks/s",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": statistics.median(e2e_ms),
           "path": "ProgramBatch.gradient on host NumPy arrays (wall clock, synchronised)"}
    lat = []
    for p, x in zip(progs, xs):
        w = torch.empty(max(p.workspace_bytes, 1), dtype=torch.uint8, device=dev)
        p.gradient(x, workspace=w, stream=stream)
        lat.append(_events_ms(stream, lambda: p.gradient(x, workspace=w, stream=stream)))
    lat.sort()
    line = _line(args, "many-network forward+adjoint throughput", len(progs) / (ms * 1e-3), "networks/s", True, ms,
                 {"workload": f"{len(progs)} random 3-regular networks, n in [20,50], bond in {{2,3,4}}, "
                              "f32/c64 alternating",
                  "form": "persistent interpreter for the small SIMT-only networks, lane streams for the rest",
                  "interpreted_networks": len(interpreted), "stages": part["stages"],
                  "interpreter_tasks": part["tasks"], "lane_network_kernels": lane_kernels,
                  "lanes": batch.lanes, "precision": "tf32x3 (c64) / fp32 (f32)",
                  "l2": "flushed (256 MiB write) before each timed batch", "tuning": tune_info}, "f32+c64",
                 gpu_launches=launches_per_call * args.steps,
                 lane_form_ms=lanes_ms, lane_form_launches_per_call=sum(p.launches for p in progs),
                 e2e=e2e, roofline={"bound": "latency", "achieved_tflops": flops / (ms * 1e-3) / 1e12},
                 cpu_baseline=None, clocks=sampler.summary(), device_status=status,
                 tflops=flops / (ms * 1e-3) / 1e12,
                 single_network_ms_p50=lat[len(lat) // 2], single_network_ms_p99=lat[min(len(lat) - 1,
                                                                                         int(0.99 * len(lat)))],
                 sum_of_single_network_ms=sum(lat), batch_speedup_vs_serial=sum(lat) / ms)
    return line


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload != "rand3reg":
        if rank != 0 and not (args.workload == "batch" and world > 1):
            return
        import torch

        torch.cuda.set_device(local)
        dev = torch.device("cuda", local)
        if args.workload in ("grid6", "brickwork"):
            line = run_latency(args, dev, args.workload)
        elif args.workload == "grid8":
            line = run_grid8(args, dev)
        elif args.workload == "rand3reg_n64":
            line = run_rand3reg_n64(args, dev)
        else:
            line = run_batch(args, dev)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    if args.impl == "reference":
        run_reference(args, rank)
        return
    net, arrays, path, sliced, name = workload(args.nodes, args.target_log2)

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
                  max_slices_per_group=args.group, tc_k_chunk=args.tc_k_chunk)
    if world > 1:
        common.update(slice_begin=begin, slice_end=end)
    # The GEMM autotuner times every kernel variant on every GEMM shape of the program (standalone, before
    # anything is timed) and pins the fastest; the table also serves the FP32 form below.
    tuning, tune_info = None, None
    if not args.no_tune:
        t0 = time.perf_counter()
        tuning = A.autotune(*net.as_tuple(), path, sliced, precision=args.precision, **common)
        tune_info = {"tune_s": round(time.perf_counter() - t0, 1), "gemm_shapes": len(tuning)}
    prog = A.SlicedProgram(*net.as_tuple(), path, sliced, precision=args.precision, tuning=tuning, **common)
    if tuning is not None:
        from arctn_b200 import tuning as T

        changed = [k for k in tuning.keys() if tuning.get(k) != tuning.timings(k).get("heuristic")]
        tune_info["changed_from_heuristic"] = len(changed)
        seen, picks = set(), []
        for g in prog.gemms():
            k = T.key_of(g)
            if k not in seen and g["bt"] * g["m"] * g["k"] * g["n"] >= 1 << 24:
                seen.add(k)
                picks.append({"bt_m_k_n": [g["bt"], g["m"], g["k"], g["n"]], "variant": g["variant"],
                              "heuristic": tuning.timings(k).get("heuristic"),
                              "ms": {v: (round(t, 4) if t is not None else None)
                                     for v, t in tuning.timings(k).items() if v in T.VARIANT_CODES},
                              "whole_program_ms": tuning.timings(k).get("whole_program_ms")})
        tune_info["program_ms"] = {"heuristics": tuning.meta.get("program_ms_before"),
                                   "tuned": tuning.meta.get("program_ms_after")}
        tune_info["large_gemms"] = picks
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
    # The reference's own unit (src/bin/tnexec.rs:4-5): Sum over steps of the product of the step's leg
    # dimensions, a complex multiply counted as 1, per slice (sliced legs at dimension 1) times the slices.
    sub = dict(net.size_dict)
    for leg in sliced:
        sub[leg] = 1
    ref_flops = 10 ** A.simulate_path(net.inputs, net.output, sub, path)["log10_flops"] * total
    reference_unit = {"unit": "GFLOPS (tnexec: Sum_steps prod(step leg dims), complex multiply = 1)",
                      "value": ref_flops / (ms_per_step * 1e-3) / 1e9, "flops_per_contraction": ref_flops}

    extras = {"reference_unit": reference_unit}
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
        t2 = A.autotune(*net.as_tuple(), path, sliced, precision=other, table=tuning, **common) \
            if tuning is not None else None
        prog2 = A.SlicedProgram(*net.as_tuple(), path, sliced, precision=other, tuning=t2, **common)
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
        extras.update({"other_precision": other, "other_value": prog.flops / (ms2 * 1e-3) / 1e12,
                       "speedup_vs_other": ms2 / ms_per_step, "rel_err_vs_fp64": rel(r.item()),
                       "other_rel_err_vs_fp64": rel(r2.item()), "fp64_result": [ref.real, ref.imag]})
        # The oracle (complex128 inputs, the reference's executor) on a sample of slices, against the same
        # slices on the GPU through a slice-range program of the benchmarked precision.
        from oracle import oracle as O

        O.build()
        samp = max(1, min(total, host_threads(), 32))
        t0 = time.perf_counter()
        want = complex(np.asarray(O.contract_slice_range(*net.as_tuple(), path, sliced, 0, samp, O.promote(arrays),
                                                         threads=samp)))
        t_or = time.perf_counter() - t0
        rs = dict(common)
        rs.update(slice_begin=0, slice_end=samp)
        ps = A.SlicedProgram(*net.as_tuple(), path, sliced, precision=args.precision, tuning=tuning, **rs)
        got = complex(ps.execute(x, f64_out=True, stream=stream).item())
        del ps
        extras["oracle_sample"] = {"slices": [0, samp], "rel_err": abs(got - want) / abs(want),
                                   "oracle": [want.real, want.imag], "gpu": [got.real, got.imag],
                                   "oracle_wall_s": t_or, "oracle_threads": samp}

    # The same contraction under the staged scheduler (ProgramBatch of one program): every slice's SIMT steps
    # inside persistent interpreter launches, the tensor-core GEMMs and packs launched between them.
    if world == 1 and not args.no_extras:
        sb = A.ProgramBatch([prog], max_lanes=8, mode="staged")
        part = next(p for p in sb.describe()["parts"] if p["part"] == -1)
        run = sb.bind([x], stream=stream)
        for _ in range(max(args.warmup, 3)):
            run()
        torch.cuda.synchronize(dev)
        st_ms = []
        for _ in range(args.steps):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run()
            e1.record(stream)
            e1.synchronize()
            st_ms.append(e0.elapsed_time(e1))
        same = bool(torch.equal(sb.execute([x], workspace=run.workspace, stream=stream)[0],
                                prog.execute(x, workspace=ws, stream=stream)))
        extras["staged_scheduler"] = {
            "ms_per_step": statistics.mean(st_ms), "value": prog.flops / (statistics.mean(st_ms) * 1e-3) / 1e12,
            "unit": "TFLOP/s", "interpreter_launches": part["stages"],
            "tensor_core_and_pack_launches": sum(part["stage_launches"]), "graph_launches_of_program": prog.launches,
            "bit_identical_to_program": same, "device_status": sb.device_status(run.workspace, stream)}
        del sb, run
        torch.cuda.empty_cache()

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
            # The profile times each kernel on its own (an event pair per launch).  `frac` divides by the burst
            # bf16 rate, the stricter denominator; the sustained one is reported beside it, and the split-TF32
            # GEMM below is also set against the TF32 rates measured on this GPU, burst and sustained.
            achieved = tw / (tms * 1e-3) / 1e12
            peak = pk["bf16_tflops"]
            traffic = profiled_traffic()  # scaled from an ncu capture of a smaller slice group
            roof = {"bound": "tensor", "kernel": KIND_NAMES.get(top, str(top)), "achieved": achieved,
                    "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                    "frac_of_sustained": achieved / pk["bf16_tflops_sustained"],
                    "peak_source": "measured bf16 dense burst (MEASURED_PEAKS.json)" if pk["source"] == "measured"
                    else "fallback bf16 dense burst of an earlier measurement (MEASURED_PEAKS.json absent)",
                    "traffic": traffic, "traffic_source": "ncu capture of a slice group of 4, scaled by slices "
                    "(profiles/k_tc_cgemm_tf32x3_rand3reg_n172.md)" if traffic else None,
                    "launches": tn, "avg_launch_ms": tms / tn,
                    "share_of_profiled_time": tms / tot}
            if traffic:
                roof["traffic_gbs"] = traffic / (tms / tn * 1e-3) / 1e9  # far below HBM: not memory-bound
            if top == 9:
                # split-TF32 4M: 12 TF32 MMAs per complex MAC step = 24 pipe flops per 8 algorithmic flops.
                # The TF32 denominator is measured on this GPU by the library's own tcgen05 probe (MMAs over
                # shared-memory-resident operands, no TMA, no epilogue); N = 128 is the MMA shape the GEMM
                # issues, N = 256 the pipe's best.
                pk_tc = {f"{kind}_n{n}": A.tensor_pipe_peak(kind, n, device=local)
                         for kind in ("tf32", "bf16") for n in (128, 256)}
                # the GEMM's own 12-MMA sequence over operands streaming through its ring layout
                pk_tc["tf32_gemm_stream_n128"] = A.tensor_pipe_peak("tf32_gemm_stream", 128, device=local)
                # The denominator is the highest TF32 MMA rate any probe reached on this GPU in this run (the
                # GEMM-stream probe, whose two interleaved accumulators hide the accumulation latency a single
                # chain pays, usually measures highest).
                tf32_peak = max(pk_tc["tf32_n128"], pk_tc["tf32_n256"], pk_tc["tf32_gemm_stream_n128"])
                roof["tensor_pipe_measured_tflops"] = pk_tc
                roof["pipe_tflops"] = achieved * 3
                roof["pipe_frac_of_tf32_peak"] = achieved * 3 / tf32_peak
                roof["pipe_frac_of_tf32_n128"] = achieved * 3 / pk_tc["tf32_n128"]
                roof["tf32_peak_source"] = ("measured: arctn_b200_tc_peak, the highest of kind::tf32 M=128 N=128/256 and "
                                            "the split-TF32 GEMM's own MMA stream")
                roof["pipe_frac_of_gemm_stream_ceiling"] = achieved * 3 / pk_tc["tf32_gemm_stream_n128"]
                # The same MMA stream held for seconds (one 1.7 s launch after a warm-up launch as long), as the
                # GEMM runs inside the step: under the 1 kW power cap the SM clock settles below its burst value,
                # and this is the TF32 rate the tensor pipe sustains there.
                sust = A.tensor_pipe_peak("tf32_gemm_stream", 128, iters=1 << 22, device=local, repeats=1)
                pk_tc["tf32_gemm_stream_sustained"] = sust
                roof["pipe_frac_of_sustained_gemm_stream"] = achieved * 3 / sust
                # The probes above stream operands that are all 1.0.  The tensor pipe's power follows its operand
                # bits, so the same stream over random TF32 hi / lo operands, held as long, is the rate the pipe
                # sustains on data like the GEMM's under the power cap.
                pk_tc["tf32_gemm_stream_random_n128"] = A.tensor_pipe_peak("tf32_gemm_stream_random", 128, device=local)
                sust_rand = A.tensor_pipe_peak("tf32_gemm_stream_random", 128, iters=1 << 22, device=local, repeats=1)
                pk_tc["tf32_gemm_stream_random_sustained"] = sust_rand
                roof["pipe_frac_of_sustained_random_stream"] = achieved * 3 / sust_rand
                roof["per_step"] = per_step_roofline(prog, ms, tf32_peak, pk["hbm_gbs"], sust_rand)
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
        try:
            cpu["numpy_tensordot"] = numpy_tensordot_baseline(net, arrays, path, sliced, total, prog.flops)
        except MemoryError:
            cpu["numpy_tensordot"] = None

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "c64", "data": "synthetic",
                "config": {"workload": name, "n_nodes": args.nodes, "bond": 2, "graph_seed": 1,
                           "target_size": 2 ** args.target_log2, "n_slices": total,
                           "slices_per_group": prog.slices_per_group, "precision": args.precision,
                           "cross_slice_sum": "fp64", "l2": "flushed (256 MiB write) between timed iterations",
                           "parallelism": f"slice-sharded x{world}", "tuning": tune_info},
                "gpu_launches": prog.launches * args.steps, "e2e": e2e, "roofline": roof, "cpu_baseline": cpu,
                "clocks": clocks, "device_status": status, "workspace_bytes": int(prog.workspace_bytes),
                "result": [float(r.real), float(r.imag)]}
        line.update(extras)
        if world == 1 and not args.no_extras and not args.no_configs:
            # The other configurations, each measured the way its own --workload run measures it, in the same
            # process after the headline's buffers are released.
            del prog, ws, x, flush
            torch.cuda.empty_cache()
            others = {}
            for which in ("grid6", "rand3reg_n64", "brickwork", "grid8", "batch"):
                t0 = time.perf_counter()
                try:
                    d = (run_latency(args, dev, which) if which in ("grid6", "brickwork") else
                         run_rand3reg_n64(args, dev) if which == "rand3reg_n64" else
                         run_grid8(args, dev) if which == "grid8" else run_batch(args, dev))
                    d["wall_s"] = round(time.perf_counter() - t0, 1)
                except Exception as e:  # one configuration failing must not hide the headline
                    d = {"error": f"{type(e).__name__}: {e}"}
                others[which] = d
                torch.cuda.empty_cache()
            line["configs"] = others
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

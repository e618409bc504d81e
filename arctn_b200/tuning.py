"""GEMM autotuner: picks the kernel variant of every GEMM shape a program runs from timed candidates.

A program chooses one kernel per pairwise GEMM with built-in heuristics (``csrc/program.cu``, ``emit_gemm``).
The tuner replaces those guesses with measurements.  For every distinct GEMM shape of a program -- its key
is (dtype, precision, phase, a_var, b_var, bt, m, k, n): phase 1 for a slice-invariant GEMM, 2 for one run
per slice group, a_var / b_var for the operands that differ per slice, and gemm_dims of one slice -- it
times each candidate variant inside the program itself: the program is rebuilt with the variant pinned
through a tuning table, run op by op on random inputs of the network's shapes, and the key's time is that of
its GEMMs plus the ops serving them (operand packs, split-K sums; a producer's epilogue that writes the next
GEMM's packed operand counts for the producer).  Every variant is pinned on all the keys it may serve in one
run, so a tuning pass costs one program run per variant, not per key and variant.
Candidates are the SIMT kernels (all dtypes) and, under precision tf32x3 / bf16x3 / bf16x6 for float32 and
complex64, the tensor-core GEMM with either tile order or with K split across CTAs.  A candidate whose time
cannot beat the current choice even at its kernel family's peak rate is skipped untimed.

The resulting :class:`TuneTable` goes to ``SlicedProgram(..., tuning=table)``; it saves to and loads from
JSON, so a table tuned once on a GPU serves later runs.  The reference has no counterpart: every GEMM there
is one ``matrixmultiply`` call (src/tensor.rs:49-64,193-231,270-308).
"""

from __future__ import annotations

import json
import time

from . import _capi as C

VARIANT_NAMES = ["auto", "simt_small", "simt_tile64", "simt_tile32", "simt_warp", "simt_tile128", "simt_dot",
                 "tc_mfast", "tc_nfast", "tc_splitk", "tc_stream", "tc_deep", "tc_pair", "tc_pair_stream"]
VARIANT_CODES = {name: code for code, name in enumerate(VARIANT_NAMES)}
SIMT_VARIANTS = ["simt_tile64", "simt_tile32", "simt_tile128", "simt_warp", "simt_small", "simt_dot"]
TC_VARIANTS = ["tc_mfast", "tc_nfast", "tc_splitk", "tc_stream", "tc_deep", "tc_pair", "tc_pair_stream"]
KEY_FIELDS = ("dtype", "precision", "phase", "a_var", "b_var", "bt", "m", "k", "n")

# Rate ceilings used only to skip candidates that cannot win (TFLOP/s of algorithmic flops): the CUDA cores'
# FP32 FMA rate of a B200 (148 SMs x 128 lanes x 2 flops x 1.965 GHz), half that in FP64, and the split
# products' share of the dense TF32 tensor pipe (3 TF32 MMAs per real product).
_SIMT_F32_TFLOPS = 75.0
_SIMT_F64_TFLOPS = 37.0
_TC_TFLOPS = 1100.0 / 3.0
_TILE_M = _TILE_N = 128   # tensor-core output tile
_TC_K_TILE = 16           # K per packed tensor-core row (TF32)
_SMS = 148


def key_of(d):
    """The 9-tuple key of a dict with the KEY_FIELDS."""
    return tuple(int(d[f]) for f in KEY_FIELDS)


def _flops(key, S):
    dtype, _, phase, _, _, bt, m, k, n = key
    mul = 8.0 if dtype in (C.C64, C.C128) else 2.0
    return mul * bt * m * k * n * (S if phase == 2 else 1)


def candidates(key, S=1):
    """Variants worth timing for one GEMM key at group size S (the heuristic's own pick is added by the
    caller).  Kinds that cannot run the dtype / precision are left out, as are shapes a kind is never fit for:
    the one-CTA-per-output dot beyond 4096 outputs, the serial-K small kernel beyond K = 1024, a second tile
    order when the output has a single tile row or column, and a K split with fewer than 16 K tiles."""
    dtype, precision, phase, _, _, bt, m, k, n = key
    outs = bt * m * n * (S if phase == 2 else 1)
    out = []
    if precision in (C.PREC_TF32X3, C.PREC_BF16X3, C.PREC_BF16X6) and dtype in (C.F32, C.C64):
        out.append("tc_mfast")
        mt, nt = -(-m // _TILE_M), -(-n // _TILE_N)
        if mt > 1 and nt > 1:
            out.append("tc_nfast")
        kk = (k + 1) // 2 if dtype == C.F32 else k
        if -(-kk // _TC_K_TILE) >= 16 and mt * nt * bt * (S if phase == 2 else 1) < 2 * _SMS:
            out.append("tc_splitk")
        if precision == C.PREC_TF32X3 and -(-kk // _TC_K_TILE) <= 32:  # the epilogue can outweigh the MMA work
            out.append("tc_stream")
        if precision == C.PREC_TF32X3 and -(-kk // _TC_K_TILE) >= 8:  # long enough K for TMA latency to show
            out.append("tc_deep")
        if precision == C.PREC_TF32X3 and m > _TILE_M:  # a 256-row pair tile would be half empty otherwise
            out.append("tc_pair")
            if -(-kk // _TC_K_TILE) <= 32:
                out.append("tc_pair_stream")
    for v in SIMT_VARIANTS:
        if v == "simt_tile128" and dtype != C.F32:
            continue
        if v == "simt_dot" and outs > 4096:
            continue
        if v == "simt_small" and k > 1024:
            continue
        out.append(v)
    return out


def _floor_ms(key, S, variant):
    """Lowest possible time of a variant on this key (ms), from its kernel family's peak rate."""
    dtype = key[0]
    if variant.startswith("tc_"):
        rate = _TC_TFLOPS
    else:
        rate = _SIMT_F64_TFLOPS if dtype in (C.F64, C.C128) else _SIMT_F32_TFLOPS
    return _flops(key, S) / (rate * 1e12) * 1e3


class TuneTable:
    """GEMM shape key -> chosen variant, with the measured time of every timed candidate."""

    def __init__(self, meta=None):
        self._e = {}
        self.meta = dict(meta or {})

    def __len__(self):
        return len(self._e)

    def __contains__(self, key):
        return tuple(key) in self._e

    def set(self, key, variant, ms=None, S=None):
        if variant not in VARIANT_CODES or variant == "auto":
            raise ValueError(f"unknown variant {variant!r}")
        key = tuple(int(x) for x in key)
        if len(key) != len(KEY_FIELDS):
            raise ValueError(f"a key has {len(KEY_FIELDS)} fields {KEY_FIELDS}")
        self._e[key] = {"variant": variant, "ms": dict(ms or {}), "S": S}

    def get(self, key):
        e = self._e.get(tuple(key))
        return e["variant"] if e else None

    def timings(self, key):
        e = self._e.get(tuple(key))
        return dict(e["ms"]) if e else {}

    def keys(self):
        return list(self._e)

    def entries_for(self, dtype, precision):
        """Entries for the C ABI (arctn_b200_gemm_choice field order) that a program of this dtype and
        precision can use."""
        out = []
        for key, e in self._e.items():
            if key[0] == dtype and key[1] == precision:
                d, p, ph, av, bv, bt, m, k, n = key
                out.append((d, p, ph, av, bv, VARIANT_CODES[e["variant"]], bt, m, k, n))
        return out

    def to_json(self):
        rows = []
        for key, e in sorted(self._e.items()):
            row = dict(zip(KEY_FIELDS, key))
            row.update(variant=e["variant"], ms=e["ms"], S=e["S"])
            rows.append(row)
        return json.dumps({"format": "arctn_b200.tune", "version": 1, "meta": self.meta, "entries": rows},
                          indent=1, sort_keys=True)

    @classmethod
    def from_json(cls, text):
        d = json.loads(text)
        if d.get("format") != "arctn_b200.tune" or d.get("version") != 1:
            raise ValueError("not an arctn_b200 tuning table (format arctn_b200.tune, version 1)")
        t = cls(d.get("meta"))
        for row in d["entries"]:
            t.set(key_of(row), row["variant"], row.get("ms"), row.get("S"))
        return t

    def save(self, path):
        with open(path, "w") as f:
            f.write(self.to_json())

    @classmethod
    def load(cls, path):
        with open(path) as f:
            return cls.from_json(f.read())


def _random_inputs(inputs, size_dict, dtype, device):
    import torch

    tdt = {C.F32: torch.float32, C.F64: torch.float64, C.C64: torch.complex64, C.C128: torch.complex128}[dtype]
    g = torch.Generator(device=device)
    g.manual_seed(0)
    return [torch.randn(*[size_dict[l] for l in t], dtype=tdt, device=device, generator=g) for t in inputs]


def _key_costs(prog, arrays, reps):
    """Per GEMM key of `prog`: device ms of one execute spent in its GEMMs and the ops that serve them (operand
    packs, split-K sums), min over `reps` op-by-op profiles; its variant; and its algorithmic flops."""
    import torch

    d = prog.describe()
    ops = d["ops"]
    gemm_key, variant, flops = {}, {}, {}
    mul = 8.0 if prog.code in (C.C64, C.C128) else 2.0
    for o in ops:
        if "variant" in o:
            key = (prog.code, prog.precision, o["phase"], o["a_var"], o["b_var"], o["bt"], o["m"], o["k"], o["n"])
            gemm_key[o["gemm"]] = key
            variant[key] = o["variant"]
            flops[key] = flops.get(key, 0.0) + mul * o["S"] * o["bt"] * o["m"] * o["k"] * o["n"]
    units = {}
    for i, o in enumerate(ops):
        units.setdefault(o.get("unit", i), []).append(o)
    order = [u for u in sorted(units) if units[u][0]["kind"] != "memset"]  # the profile's entries
    ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device=arrays[0].device)
    best, total = None, float("inf")
    for r in range(reps + 1):
        ms, _, _ = prog.profile(arrays, workspace=ws)
        if len(ms) != len(order):
            raise RuntimeError("profile entries do not match the program's launch units")
        cost = {key: 0.0 for key in variant}
        for u, t in zip(order, ms):
            owners = [gemm_key[o["gemm"]] for o in units[u] if o.get("gemm", -1) in gemm_key]
            for key in owners:  # a grouped launch of thin GEMMs splits its time evenly
                cost[key] += t / len(owners)
        if r:
            best = cost if best is None else {k: min(best[k], cost[k]) for k in best}
            total = min(total, float(sum(ms)))
    if prog.device_status(ws) != 0:
        raise RuntimeError("a bounded device wait expired while tuning")
    del ws
    return best, variant, flops, total


def autotune(inputs, output, size_dict, ssa_path, sliced_legs=(), *, dtype="complex64", precision="fp32",
             device=None, table=None, reps=2, log=None, margin=0.03, **program_kw):
    """Tunes every GEMM shape of the program these arguments describe (``program_kw``: the other
    ``SlicedProgram`` options -- workspace budget, group size, slice range, gradient) and returns the table;
    a given ``table`` is extended, and keys it already holds are not timed again.  Needs a GPU.

    The candidates are timed inside the program itself, on random inputs of the network's shapes: one run
    with the current choices, then one run per variant with that variant pinned on every untuned key it may
    serve; each key's time is the time of its GEMMs and the ops serving them (operand packs, split-K sums).
    A candidate that cannot beat the key's current time even at its kernel family's peak rate is not run.  A
    variant replaces the heuristic's choice only where it is faster by more than ``margin`` (a fraction of the
    heuristic's time): repeated runs of one program differ by a few percent, and a switch on a smaller
    difference is as likely to lose as to win."""
    import torch

    from .api import SlicedProgram

    if device is None:
        device = torch.cuda.current_device()
    dev = torch.device("cuda", device)
    table = table if table is not None else TuneTable()
    t0 = time.perf_counter()

    def build(t):
        return SlicedProgram(inputs, output, size_dict, ssa_path, sliced_legs, dtype=dtype, precision=precision,
                             device=device, tuning=t, **program_kw)

    base = build(table)
    arrays = _random_inputs(base.inputs, base.size_dict, base.code, dev)
    base_cost, base_var, flops, base_total = _key_costs(base, arrays, reps)
    S = base.slices_per_group
    todo = [k for k in base_var if k not in table]
    times = {k: {base_var[k]: base_cost[k]} for k in todo}
    for v in VARIANT_NAMES[1:]:
        pins = [k for k in todo if v != base_var[k] and v in candidates(k, S)
                and flops[k] / ((_TC_TFLOPS if v.startswith("tc_") else
                                 _SIMT_F64_TFLOPS if k[0] in (C.F64, C.C128) else _SIMT_F32_TFLOPS) * 1e9)
                < base_cost[k]]
        for k in todo:
            if v != base_var[k] and v in candidates(k, S) and k not in pins:
                times[k][v] = None  # cannot win even at its peak rate
        if not pins:
            continue
        trial = TuneTable()
        for k in table.keys():
            trial.set(k, table.get(k))
        for k in pins:
            trial.set(k, v)
        try:
            cost, var, _, _ = _key_costs(build(trial), arrays, reps)
        except torch.cuda.OutOfMemoryError:
            torch.cuda.empty_cache()
            continue
        for k in pins:
            if var.get(k) == v:
                times[k][v] = cost[k]
        if log:
            log(f"{v}: {len(pins)} GEMM shapes timed")
    def with_choices(extra):
        trial = TuneTable()
        for kk in table.keys():
            trial.set(kk, table.get(kk))
        for kk, vv in choice.items():
            trial.set(kk, vv)
        for kk, vv in extra.items():
            trial.set(kk, vv)
        return trial

    def program_ms(trial):
        try:
            return _key_costs(build(trial), arrays, reps)[3]
        except torch.cuda.OutOfMemoryError:
            torch.cuda.empty_cache()
            return None

    # Within one family a variant replaces the heuristic's choice where it beats it by more than the margin.
    choice = {}
    for k in todo:
        a = base_var[k]
        same = {v: t for v, t in times[k].items()
                if v in VARIANT_CODES and t is not None and v.startswith("tc_") == a.startswith("tc_")}
        best = min(same, key=same.get)
        choice[k] = best if same[best] < (1.0 - margin) * same[a] else a
    # A variant's in-situ time is taken with that variant pinned on every key it may serve, and all GEMMs share
    # one power budget: a variant that slows some other key draws less power and lets the clock of the whole
    # run rise.  So a switch on a key worth more than 5% of the run is kept only if the whole program gets
    # faster by 1% with it, tried one key at a time from the largest measured gain.
    current = base_total
    big = sorted(((times[k][base_var[k]] - times[k][choice[k]], k) for k in todo
                  if choice[k] != base_var[k] and times[k][base_var[k]] > 0.05 * base_total), reverse=True)
    confirmed_big = 0
    if big:
        pending = {k: choice[k] for _, k in big}
        for _, k in big:
            choice[k] = base_var[k]
        start = program_ms(with_choices({}))
        current = start if start is not None else base_total
        for _, k in big:
            total = program_ms(with_choices({k: pending[k]}))
            if total is None:
                continue
            times[k]["whole_program_ms"] = {"before": current, "after": total}
            if total < 0.99 * current:
                choice[k], current = pending[k], total
                confirmed_big += 1
    # A switch between a tensor-core and a SIMT variant changes more than its own GEMM: a tensor-core producer
    # writes its consumer's packed operand from its epilogue, and a tensor-core consumer needs packs its SIMT
    # form does not.  Such a switch is kept only if the whole program gets faster, tried one key at a time in
    # order of the gain measured on the key itself (the largest few, each worth at least 0.2% of the run).
    switches = []
    for k in todo:
        timed_ = {v: t for v, t in times[k].items() if v in VARIANT_CODES and t is not None}
        a = base_var[k]
        other = {v: t for v, t in timed_.items() if v.startswith("tc_") != a.startswith("tc_")}
        if other:
            b = min(other, key=other.get)
            if other[b] < timed_[choice[k]]:
                switches.append((timed_[choice[k]] - other[b], k, b))
    switches.sort(reverse=True)
    confirmed = 0
    for gain, k, v in switches[:8]:
        if gain < 0.002 * base_total:
            break
        total = program_ms(with_choices({k: v}))
        if total is None:
            continue
        times[k]["whole_program_ms"] = {"before": current, "after": total}
        if total < 0.998 * current:
            choice[k], current = v, total
            confirmed += 1
    for k in todo:
        times[k]["heuristic"] = base_var[k]
        table.set(k, choice[k], times[k], S)
    table.meta["program_ms_before"] = base_total
    table.meta["program_ms_after"] = current
    table.meta["family_switches_kept"] = confirmed
    table.meta["large_key_switches_kept"] = confirmed_big
    table.meta.setdefault("device", torch.cuda.get_device_name(device))
    table.meta["tune_seconds"] = table.meta.get("tune_seconds", 0.0) + (time.perf_counter() - t0)
    del arrays
    torch.cuda.empty_cache()
    return table

"""Saved execution plans (schema ``arctn-execution-plan`` version 2) and ``tensors.bin`` data files.

A version-2 plan is self-contained: a dense integer network, the SSA path and the exact slice set,
plus the metrics the planner reported.  Loading re-derives everything that can be re-derived and
rejects the file when a field disagrees, as the reference does before it runs a saved plan
(``parse_embedded_execution_plan``, src/execution_plan.rs:262-475); the plan then runs on the B200
executor (``ExecutionPlan.execute``, the counterpart of ``ArcTNExecutionPlan.execute``,
pybind/python/arctn/_execution_plan.py:489-577).  ``load_tensors_bin`` reads the reference's data
format: every input tensor's elements, row-major, little-endian, concatenated in network order
(src/network.rs:81-132).
"""

from __future__ import annotations

import ctypes
import json
import math
import os
import tempfile

import numpy as np

from . import _capi as C

SCHEMA = "arctn-execution-plan"
SCHEMA_VERSION = 2
PATH_FORMAT = "ssa-v1"
MEMORY_CONSTRAINT_METRIC = "max_intermediate_elements_per_slice"
_TARGET_DECLARATION_TOL_LOG2 = 1e-12  # src/execution_plan.rs:29-32
_METRIC_ABS_TOL = 1e-9
_METRIC_REL_TOL = 1e-12
_PATH_METRICS = ("log10_flops", "log2_max_size", "log2_max_contraction_size", "log2_total_size",
                 "log2_read_write", "log2_peak_size")
_LOG10_2 = math.log10(2.0)


class PlanValidationError(ValueError):
    """A saved plan that the loader rejects (pybind/python/arctn/_execution_plan.py:68-70)."""


def network_canon(inputs, output, size_dict):
    """Canonical network identity string (src/pathcache.rs:72-103)."""
    t = ";".join(",".join(str(int(l)) for l in legs) for legs in inputs)
    o = ",".join(str(int(l)) for l in output)
    d = ",".join(f"{int(l)}={int(size_dict[l])}" for l in sorted(size_dict))
    return f"t:{t}|o:{o}|d:{d}"


def _stats(inputs, output, size_dict, ssa_path, sliced=(), target=0):
    """(whole-network metrics, per-slice metrics, fits-target) through the executor's host code."""
    net = C.NetworkArgs(inputs, output, size_dict)
    n, p = C.path_array(ssa_path)
    full = (ctypes.c_double * 6)()
    C.check(C.lib().arctn_b200_simulate_path(net.ptr, n, p.ctypes.data_as(C.u64p), full), "ssa_path is invalid")
    sl = np.asarray(list(sliced) or [0], dtype=np.uint32)
    per = (ctypes.c_double * 6)()
    fits = ctypes.c_int(1)
    C.check(C.lib().arctn_b200_slice_plan_check(net.ptr, n, p.ctypes.data_as(C.u64p), len(sliced),
                                                sl.ctypes.data_as(C.u32p), int(target), per, ctypes.byref(fits)),
            "invalid slice set")
    return dict(zip(_PATH_METRICS, full)), dict(zip(_PATH_METRICS, per)), bool(fits.value)


def _is_int(v):
    return isinstance(v, int) and not isinstance(v, bool)


def _network_from_artifact(raw):
    """Dense network of a v2 artifact (ExecutionPlanNetwork::to_network, src/execution_plan.rs:62-108)."""
    if not isinstance(raw, dict) or set(raw) - {"inputs", "output", "size_dict"} or len(raw) != 3:
        raise PlanValidationError("execution plan network is invalid: expected inputs, output and size_dict")
    inputs, output, sd = raw["inputs"], raw["output"], raw["size_dict"]
    ok = (isinstance(inputs, list) and all(isinstance(t, list) and all(_is_int(l) and l >= 0 for l in t) for t in inputs)
          and isinstance(output, list) and all(_is_int(l) and l >= 0 for l in output)
          and isinstance(sd, list) and all(isinstance(e, list) and len(e) == 2 and _is_int(e[0]) and _is_int(e[1])
                                           and e[0] >= 0 and e[1] >= 0 for e in sd))
    if not ok:
        raise PlanValidationError("execution plan network is invalid: malformed fields")
    seen, nxt = set(), 0
    for leg in [l for t in inputs for l in t] + list(output):
        if leg not in seen:
            seen.add(leg)
            if leg != nxt:
                raise PlanValidationError("execution plan network legs must use dense first-occurrence order")
            nxt += 1
    if len(sd) != len(seen) or any(leg != i for i, (leg, _) in enumerate(sd)):
        raise PlanValidationError("execution plan network.size_dict must contain each dense leg once in order")
    size_dict = {int(l): int(d) for l, d in sd}
    return [list(t) for t in inputs], list(output), size_dict


def _check_labels(inputs, output, size_dict, labels):
    """validate_label_table (src/execution_plan.rs:892-910)."""
    if not isinstance(labels, list) or not all(isinstance(x, str) for x in labels):
        raise PlanValidationError("network_leg_labels is invalid: expected a list of strings")
    if len(labels) != len(size_dict):
        raise PlanValidationError("network_leg_labels length must match the embedded dense network")
    for leg in {l for t in inputs for l in t} | set(output):
        if leg >= len(labels):
            raise PlanValidationError(f"network_leg_labels has no entry for embedded LegId {leg}")
    if len(set(labels)) != len(labels):
        raise PlanValidationError("network_leg_labels must be unique")


def _slice_set(root, labels):
    """parse_slice_set with an explicit ``sliced.legs`` (src/execution_plan.rs:714-776)."""
    raw = root.get("sliced")
    if raw is None:
        raise PlanValidationError("versioned execution plans must provide sliced; an unsliced plan uses empty legs")
    if not isinstance(raw, dict):
        raise PlanValidationError("sliced must be an object")
    legs = raw.get("legs")
    if legs is None:
        raise PlanValidationError("versioned execution plans require sliced.legs")
    if not isinstance(legs, list) or not all(_is_int(l) and l >= 0 for l in legs):
        raise PlanValidationError("sliced.legs is invalid")
    named = raw.get("leg_labels")
    if named is not None:
        if not isinstance(named, list) or not all(isinstance(x, str) for x in named):
            raise PlanValidationError("sliced.leg_labels is invalid")
        if labels is None:
            raise PlanValidationError("sliced.leg_labels cannot be checked without network_leg_labels")
        expect = []
        for l in legs:
            if l >= len(labels):
                raise PlanValidationError(f"network_leg_labels has no entry for LegId {l}")
            expect.append(labels[l])
        if expect != named:
            raise PlanValidationError("sliced.legs and sliced.leg_labels do not identify the same legs")
    return [int(l) for l in legs]


def _check_metric_fields(obj, where, expected):
    """validate_metric_fields (src/execution_plan.rs:557-578)."""
    for name, want in expected:
        got = obj.get(name)
        if got is None:
            continue
        if isinstance(got, bool) or not isinstance(got, (int, float)) or not math.isfinite(got):
            raise PlanValidationError(f"{where}.{name} must be a finite number")
        tol = max(_METRIC_ABS_TOL, _METRIC_REL_TOL * max(abs(want), abs(got)))
        if not math.isfinite(want) or abs(got - want) > tol:
            raise PlanValidationError(f"{where}.{name}={got} does not match the recomputed value {want}")


def _check_metrics(root, full, per, n_log2_slices):
    """validate_reported_metrics (src/execution_plan.rs:477-555)."""
    path_metrics = [(k, full[k]) for k in _PATH_METRICS]
    _check_metric_fields(root, "execution plan", path_metrics)
    metrics = root.get("metrics")
    if metrics is not None and not isinstance(metrics, dict):
        raise PlanValidationError("execution plan metrics must be an object")
    if metrics is not None:
        _check_metric_fields(metrics, "execution plan metrics", path_metrics)
    total = per["log10_flops"] + n_log2_slices * _LOG10_2
    canonical = [("log2_n_slices", n_log2_slices), ("sliced_log10_flops_total", total),
                 ("sliced_log2_max_size", per["log2_max_size"]),
                 ("sliced_log2_max_contraction_size", per["log2_max_contraction_size"]),
                 ("sliced_log2_peak_size", per["log2_peak_size"]),
                 ("max_intermediate_log2_elements_per_slice", per["log2_max_size"])]
    _check_metric_fields(root, "execution plan", canonical)
    if metrics is not None:
        _check_metric_fields(metrics, "execution plan metrics", canonical)
    sliced = [("log2_n_slices", n_log2_slices), ("per_slice_log10_flops", per["log10_flops"]),
              ("per_slice_log2_write", per["log2_total_size"]), ("per_slice_log2_read_write", per["log2_read_write"]),
              ("per_slice_log2_max_size", per["log2_max_size"]),
              ("per_slice_log2_max_contraction_size", per["log2_max_contraction_size"]),
              ("per_slice_log2_peak_size", per["log2_peak_size"]), ("log10_flops_total", total),
              ("log2_write_total", per["log2_total_size"] + n_log2_slices),
              ("log2_read_write_total", per["log2_read_write"] + n_log2_slices)]
    _check_metric_fields(root["sliced"], "execution plan sliced", sliced)


def _target_declaration(root):
    """parse_target_declaration for version 2 (src/execution_plan.rs:778-840)."""
    exact = root.get("target_size")
    if exact is not None and (not _is_int(exact) or exact <= 0 or exact >= 1 << 64):
        raise PlanValidationError("target_size must be a positive usize integer")
    log2 = root.get("memory_target_log2_elements")
    if log2 is not None:
        if isinstance(log2, bool) or not isinstance(log2, (int, float)) or not math.isfinite(log2) or log2 < 0:
            raise PlanValidationError("memory_target_log2_elements must be a finite non-negative number")
    if exact is not None and log2 is not None:
        want = math.log2(float(exact))
        if abs(log2 - want) > _TARGET_DECLARATION_TOL_LOG2:
            raise PlanValidationError(f"target_size={exact} is inconsistent with memory_target_log2_elements={log2}; "
                                      f"expected {want}")
    metric = root.get("memory_constraint_metric")
    if exact is None and (log2 is not None or metric is not None):
        raise PlanValidationError("execution plan version 2 requires exact target_size for every memory target "
                                  "declaration")
    if exact is not None and log2 is None:
        raise PlanValidationError("execution plan version 2 target_size requires memory_target_log2_elements")
    if exact is not None and metric != MEMORY_CONSTRAINT_METRIC:
        raise PlanValidationError(f"memory_constraint_metric must be {MEMORY_CONSTRAINT_METRIC!r} when a target is "
                                  "declared")
    return exact


class ExecutionPlan:
    """A validated, immutable version-2 execution plan bound to the B200 executor."""

    def __init__(self, artifact):
        if not isinstance(artifact, dict):
            raise PlanValidationError("execution plan root must be an object")
        artifact = json.loads(json.dumps(artifact, allow_nan=False))  # a private, JSON-clean copy
        schema, version = artifact.get("schema"), artifact.get("schema_version")
        if schema is None and version is None:
            raise PlanValidationError("schema-less execution plans are not self-contained")
        if schema is None or version is None:
            raise PlanValidationError("execution plan must contain both schema and schema_version")
        if schema != SCHEMA:
            raise PlanValidationError(f"unsupported execution plan schema: {schema!r}")
        if not _is_int(version) or version < 0:
            raise PlanValidationError("execution plan schema_version must be an integer")
        if version != SCHEMA_VERSION:
            raise PlanValidationError(f"execution plan version {version} is not self-contained; version 2 is "
                                      "required")
        if artifact.get("path_format") != PATH_FORMAT:
            raise PlanValidationError(f"unsupported execution plan path_format: {artifact.get('path_format')!r}")
        if "net" in artifact and not isinstance(artifact["net"], str):
            raise PlanValidationError("plan net field must be a string")
        if "network" not in artifact:
            raise PlanValidationError("execution plan version 2 is missing network")
        inputs, output, size_dict = _network_from_artifact(artifact["network"])
        if not isinstance(artifact.get("network_canon"), str):
            raise PlanValidationError("execution plan network_canon must be a string")
        if artifact["network_canon"] != network_canon(inputs, output, size_dict):
            raise PlanValidationError("execution plan network_canon does not match embedded network")
        labels = artifact.get("network_leg_labels")
        if labels is not None:
            _check_labels(inputs, output, size_dict, labels)
        path = artifact.get("ssa_path")
        if (not isinstance(path, list) or
                not all(isinstance(s, list) and len(s) == 2 and all(_is_int(x) and x >= 0 for x in s) for s in path)):
            raise PlanValidationError("ssa_path is invalid")
        path = [(int(a), int(b)) for a, b in path]
        sliced = _slice_set(artifact, labels)
        exact = _target_declaration(artifact)
        try:
            full, per, fits = _stats(inputs, output, size_dict, path, sliced, exact or 0)
        except ValueError as exc:
            raise PlanValidationError(str(exc)) from exc
        n_log2 = float(sum(math.log2(size_dict[l]) for l in sliced))
        _check_metrics(artifact, full, per, n_log2)
        if exact is not None and not fits:
            raise PlanValidationError(f"execution plan exceeds declared target_size={exact}")
        self.inputs, self.output, self.size_dict = inputs, output, size_dict
        self.ssa_path, self.sliced_legs, self.target_size = path, sliced, exact
        self.leg_labels = labels
        self.metrics = full
        self.name = artifact.get("net", "network")
        self.per_slice_metrics = per
        self._artifact = artifact
        self._frozen = True

    def __setattr__(self, name, value):
        if getattr(self, "_frozen", False):
            raise AttributeError("ExecutionPlan is immutable")
        object.__setattr__(self, name, value)

    # ------------------------------------------------------------------ the reference plan object's properties
    # (pybind/python/arctn/_execution_plan.py:223-282)
    @property
    def schema(self):
        return SCHEMA

    @property
    def schema_version(self):
        return SCHEMA_VERSION

    @property
    def path_format(self):
        return PATH_FORMAT

    @property
    def planning(self):
        return json.loads(json.dumps(self._artifact.get("planning", {})))

    @property
    def provenance(self):
        return json.loads(json.dumps(self._artifact.get("provenance", {})))

    @property
    def network_canon(self):
        return self._artifact["network_canon"]

    @property
    def is_sliced(self):
        return bool(self.sliced_legs)

    def to_linear_path(self):
        """The opt_einsum linear form of the SSA path (pybind/python/arctn/_execution_plan.py:455-457)."""
        from .api import ssa_to_linear

        return tuple(tuple(p) for p in ssa_to_linear(self.ssa_path, len(self.inputs)))

    def __eq__(self, other):
        if not isinstance(other, ExecutionPlan):
            return NotImplemented
        return self.to_dict() == other.to_dict()

    __hash__ = None

    # ------------------------------------------------------------------ construction / persistence
    @classmethod
    def from_path(cls, inputs, output, size_dict, ssa_path, sliced_legs=(), *, target_size=None, labels=None,
                  name="network", planning=None, source="arctn_b200"):
        """A fresh v2 artifact for a network, path and slice set (complete_execution_plan_v2,
        src/execution_plan.rs:131-208).  The network must already be dense (legs 0.. in first-occurrence order)."""
        inputs = [[int(l) for l in t] for t in inputs]
        output = [int(l) for l in output]
        size_dict = {int(k): int(v) for k, v in size_dict.items()}
        labels = list(labels) if labels is not None else [str(l) for l in sorted(size_dict)]
        sliced = [int(l) for l in sliced_legs]
        full, per, _ = _stats(inputs, output, size_dict, ssa_path, sliced)
        n_log2 = float(sum(math.log2(size_dict[l]) for l in sliced))
        art = {
            "schema": SCHEMA, "schema_version": SCHEMA_VERSION, "path_format": PATH_FORMAT, "net": name,
            "network": {"inputs": inputs, "output": output, "size_dict": [[l, size_dict[l]] for l in sorted(size_dict)]},
            "network_canon": network_canon(inputs, output, size_dict), "network_leg_labels": labels,
            "ssa_path": [[int(a), int(b)] for a, b in ssa_path],
            "sliced": {"legs": sliced, "leg_labels": [labels[l] for l in sliced], "log2_n_slices": n_log2,
                       "per_slice_log10_flops": per["log10_flops"], "per_slice_log2_max_size": per["log2_max_size"],
                       "log10_flops_total": per["log10_flops"] + n_log2 * _LOG10_2},
            "metrics": dict(full, log2_n_slices=n_log2,
                            sliced_log10_flops_total=per["log10_flops"] + n_log2 * _LOG10_2,
                            sliced_log2_max_size=per["log2_max_size"]),
            "planning": dict(planning or {}), "provenance": {"source": source},
        }
        if target_size is not None:
            art.update(target_size=int(target_size), memory_target_log2_elements=math.log2(target_size),
                       memory_constraint_metric=MEMORY_CONSTRAINT_METRIC)
        return cls(art)

    @classmethod
    def from_dict(cls, artifact):
        return cls(artifact)

    @classmethod
    def load(cls, path):
        try:
            with open(os.fspath(path), "r", encoding="utf-8") as f:
                artifact = json.load(f)
        except (OSError, UnicodeError, json.JSONDecodeError) as exc:
            raise PlanValidationError(f"cannot load execution plan: {exc}") from exc
        return cls(artifact)

    def to_dict(self):
        return json.loads(json.dumps(self._artifact))

    def save(self, path):
        """Atomic write of the JSON artifact (pybind/python/arctn/_execution_plan.py:368-400)."""
        dest = os.fspath(path)
        fd, tmp = tempfile.mkstemp(prefix=f".{os.path.basename(dest)}.", suffix=".tmp",
                                   dir=os.path.dirname(os.path.abspath(dest)))
        try:
            with os.fdopen(fd, "w", encoding="utf-8") as f:
                json.dump(self._artifact, f, ensure_ascii=False, allow_nan=False, indent=2, sort_keys=True)
                f.write("\n")
            os.replace(tmp, dest)
        except BaseException:
            if os.path.exists(tmp):
                os.unlink(tmp)
            raise
        return dest

    # ------------------------------------------------------------------ execution
    def validate(self, inputs=None, output=None, size_dict=None, *, arrays=None):
        """A caller's network (any hashable labels, numbered densely in first-occurrence order) and the
        arrays' count, shapes and one shared dtype against the plan (pybind/python/arctn/_execution_plan.py:
        402-453)."""
        import operator

        given = (inputs is not None, output is not None, size_dict is not None)
        if any(given) and not all(given):
            raise TypeError("inputs, output, and size_dict must be provided together")
        if all(given):
            ids = {}
            for leg in [l for t in inputs for l in t] + list(output):
                ids.setdefault(leg, len(ids))
            try:
                cand = ([[ids[l] for l in t] for t in inputs], [ids[l] for l in output],
                        {ids[l]: int(d) for l, d in size_dict.items() if l in ids})
            except (TypeError, ValueError) as exc:
                raise PlanValidationError(f"caller network is invalid: {exc}") from exc
            if len(cand[2]) != len(size_dict) or cand != (self.inputs, self.output, self.size_dict):
                raise PlanValidationError("caller network does not match the embedded plan network")
        if arrays is None:
            return None
        try:
            arrays = tuple(arrays)
        except TypeError as exc:
            raise PlanValidationError("arrays must be a sequence") from exc
        if len(arrays) != len(self.inputs):
            raise PlanValidationError(f"arrays length {len(arrays)} does not match {len(self.inputs)} plan inputs")
        dt = None
        for i, (a, legs) in enumerate(zip(arrays, self.inputs)):
            if not hasattr(a, "shape") or not hasattr(a, "dtype"):
                raise PlanValidationError(f"arrays[{i}] must provide shape and dtype")
            try:
                got = tuple(operator.index(d) for d in a.shape)
            except TypeError as exc:
                raise PlanValidationError(f"arrays[{i}] has invalid shape or dtype: {exc}") from exc
            shape = tuple(self.size_dict[l] for l in legs)
            if got != shape:
                raise PlanValidationError(f"arrays[{i}] shape {got} does not match {shape}")
            if dt is None:
                dt = str(a.dtype)
            elif str(a.dtype) != dt:
                raise PlanValidationError("all arrays must use the same dtype")
        return None

    def program(self, *, dtype="complex64", precision="fp32", **kw):
        """A SlicedProgram for this plan (all slices, FP64 cross-slice sum)."""
        from .api import SlicedProgram

        return SlicedProgram(self.inputs, self.output, self.size_dict, self.ssa_path, self.sliced_legs,
                             dtype=dtype, precision=precision, **kw)

    def compile(self, *, backend="b200"):
        """An ``ArcTNCompiledContraction`` of an unsliced plan for repeated execution
        (pybind/python/arctn/_execution_plan.py:474-487); sliced plans are rejected as there."""
        from .api import ArcTNCompiledContraction

        if self.sliced_legs:
            raise PlanValidationError("sliced plans cannot be compiled by ArcTNCompiledContraction; call "
                                      "plan.execute(...)")
        return ArcTNCompiledContraction.compile(self.inputs, self.output, self.size_dict, ssa_path=self.ssa_path,
                                                backend=backend)

    def execute(self, arrays, *, backend="b200", return_info=False, precision="fp32", **kw):
        """Contract the plan's network on the GPU: sum internal slices, assemble output blocks
        (pybind/python/arctn/_execution_plan.py:489-577).  ``return_info`` adds the reference's timing fields;
        the wall time covers the synchronous call, inputs staged and the result returned."""
        import time

        from .api import _validate_backend

        backend = _validate_backend(backend)
        try:
            arrays = tuple(arrays)
        except TypeError as exc:
            raise PlanValidationError("arrays must be a sequence") from exc
        self.validate(arrays=arrays)
        t0 = time.perf_counter()
        prog = self.program(dtype=arrays[0].dtype, precision=precision, **kw)
        t1 = time.perf_counter()
        result = prog.execute(arrays)
        t2 = time.perf_counter()
        if not return_info:
            return result
        return result, {"plan_schema": SCHEMA, "plan_schema_version": SCHEMA_VERSION, "execution_backend": backend,
                        "execution_implementation": "arctn_b200.SlicedProgram", "precision": precision,
                        "expression_compile_wall_s": t1 - t0, "execution_setup_wall_s": t1 - t0,
                        "execution_dispatch_wall_s": t2 - t1, "execution_wall_s": t2 - t0,
                        "execution_timing_scope": "synchronous_host_wall", "sliced_legs": list(self.sliced_legs)}

    def __repr__(self):
        return (f"ExecutionPlan(n_inputs={len(self.inputs)}, n_steps={len(self.ssa_path)}, "
                f"n_sliced_legs={len(self.sliced_legs)}, target_size={self.target_size!r})")



# The reference's name for the plan object (pybind/python/arctn/_execution_plan.py:117).
ArcTNExecutionPlan = ExecutionPlan


def load_tensors_bin(path, inputs, size_dict, dtype):
    """Input tensors from a little-endian data file (load_tensors_bin, src/network.rs:81-132)."""
    dt = np.dtype(dtype).newbyteorder("<")
    if dt.kind not in "fc":
        raise ValueError(f"unsupported dtype {dtype}")
    shapes = [tuple(int(size_dict[l]) for l in t) for t in inputs]
    counts = [int(np.prod(s, dtype=np.int64)) if s else 1 for s in shapes]
    with open(os.fspath(path), "rb") as f:
        raw = f.read()
    expect = sum(counts) * dt.itemsize
    if len(raw) != expect:
        raise ValueError(f"data file has {len(raw)} bytes; the network expects {expect} (sum of numel x "
                         f"{dt.itemsize} bytes, little-endian; check that the dtype and file match the network)")
    out, off = [], 0
    for shape, n in zip(shapes, counts):
        a = np.frombuffer(raw, dtype=dt, count=n, offset=off).reshape(shape)
        out.append(np.array(a, dtype=dt.newbyteorder("="), order="C"))  # keeps 0-d shapes
        off += n * dt.itemsize
    return out


def save_tensors_bin(path, arrays):
    """The inverse of load_tensors_bin: every array row-major, little-endian, concatenated."""
    with open(os.fspath(path), "wb") as f:
        for a in arrays:
            a = np.asarray(a)
            f.write(np.array(a, dtype=a.dtype.newbyteorder("<"), order="C").tobytes())


def arctn_plan(inputs, output, size_dict, *, preset="heavy", seed=0, target_size=None, slicing_mode="fixed",
               max_time=None, flops_weight=1.0, read_write_weight=64.0, rate_enabled=True,
               allow_output_slicing=False):
    """Plan once and return an immutable ``ExecutionPlan`` (``arctn_plan``,
    pybind/python/arctn/_execution_plan.py:593-646), with the same keywords and checks.

    The reference plans with its closed-source engine; here the public greedy path (src/paths/greedy.rs:
    317-320) and the slice search (src/slice.rs:209-289) make the plan, so the engine-only options are checked
    and recorded under ``planning`` but do not change it.  Legs are numbered densely in first-occurrence order
    and the caller's labels are kept as ``network_leg_labels`` (as strings) when they stay distinct."""
    import math as _math

    from .api import _to_int_labels, _validate_planning_options, find_slices_to_size, greedy

    target_size, max_time, (flops_weight, read_write_weight) = _validate_planning_options(
        preset, seed, target_size, slicing_mode, max_time, flops_weight, read_write_weight, allow_output_slicing)
    if not isinstance(rate_enabled, bool):
        raise TypeError("rate_enabled must be a bool")
    inputs = tuple(tuple(term) for term in inputs)
    output = tuple(output)
    if not hasattr(size_dict, "items"):
        raise TypeError("size_dict must be a mapping from leg label to positive integer dimension")
    inputs_i, output_i, size_i, label_of = _to_int_labels(inputs, output, dict(size_dict.items()))
    path = greedy(inputs_i, output_i, size_i)
    sliced = []
    if target_size is not None:
        found = find_slices_to_size(inputs_i, output_i, size_i, path, target_size,
                                    allow_output_slicing=allow_output_slicing)
        if found is None:
            raise ValueError(f"target_size (log2={_math.log2(target_size):.6g}) is unreachable: no slicing meets it")
        sliced = found
    labels = [None] * len(label_of)
    for label, leg in label_of.items():
        labels[leg] = str(label)
    planning = {"preset": preset, "seed": seed, "slicing_mode": slicing_mode, "allow_output_slicing":
                allow_output_slicing, "flops_weight": flops_weight, "read_write_weight": read_write_weight,
                "method": "greedy"}
    return ExecutionPlan.from_path(inputs_i, output_i, size_i, path, sliced, target_size=target_size,
                                   labels=labels if len(set(labels)) == len(labels) else None, planning=planning,
                                   source="arctn_plan")

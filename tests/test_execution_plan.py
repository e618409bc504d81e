"""Saved execution plans (version 2) and tensors.bin files, host side.

The cases follow the reference's own tests of its plan reader (src/execution_plan.rs:960-1153): the
v2 round trip, tampered metrics, slice labels, path format, network identity, dense leg order and
the exact target declaration.
"""

import json
import math

import numpy as np
import pytest

import arctn_b200 as A
from arctn_b200.execution_plan import (MEMORY_CONSTRAINT_METRIC, ExecutionPlan, PlanValidationError,
                                       load_tensors_bin, network_canon, save_tensors_bin)

TRI_INPUTS = [[0, 1], [0, 2], [1, 2]]
TRI_SIZES = {0: 2, 1: 2, 2: 2}
TRI_PATH = [(0, 1), (2, 3)]
LABELS = ["a", "b", "c"]


def record(**kw):
    return ExecutionPlan.from_path(TRI_INPUTS, [], TRI_SIZES, TRI_PATH, labels=LABELS, name="triangle", **kw).to_dict()


def test_round_trip_embeds_the_network():
    rec = record()
    assert rec["schema_version"] == 2 and rec["path_format"] == "ssa-v1"
    assert rec["network"]["size_dict"] == [[0, 2], [1, 2], [2, 2]]
    assert rec["sliced"]["leg_labels"] == []
    assert rec["network_canon"] == "t:0,1;0,2;1,2|o:|d:0=2,1=2,2=2"
    plan = ExecutionPlan.from_dict(json.loads(json.dumps(rec)))
    assert plan.inputs == TRI_INPUTS and plan.size_dict == TRI_SIZES
    assert plan.ssa_path == TRI_PATH and plan.sliced_legs == []
    st = A.simulate_path(TRI_INPUTS, [], TRI_SIZES, TRI_PATH)
    assert plan.metrics["log10_flops"] == st["log10_flops"]


def test_tampered_metrics_are_rejected():
    rec = record()
    rec["metrics"]["log10_flops"] = -999.0
    with pytest.raises(PlanValidationError, match=r"metrics\.log10_flops.*recomputed value"):
        ExecutionPlan(rec)
    rec = record()
    rec["sliced"]["per_slice_log2_max_size"] = 99.0
    with pytest.raises(PlanValidationError, match="sliced.per_slice_log2_max_size"):
        ExecutionPlan(rec)


def test_slices_network_and_path_format_are_validated():
    rec = record()
    rec["sliced"]["legs"] = [0]
    rec["sliced"]["leg_labels"] = ["a"]
    rec["metrics"] = {}  # the sliced metrics of the unsliced record no longer apply
    for k in list(rec["sliced"]):
        if k not in ("legs", "leg_labels"):
            del rec["sliced"][k]
    ExecutionPlan(rec)
    bad = json.loads(json.dumps(rec))
    bad["sliced"]["leg_labels"] = ["b"]
    with pytest.raises(PlanValidationError, match="same legs"):
        ExecutionPlan(bad)
    bad = json.loads(json.dumps(rec))
    bad["path_format"] = "linear"
    with pytest.raises(PlanValidationError, match="path_format"):
        ExecutionPlan(bad)
    bad = json.loads(json.dumps(rec))
    bad["network"]["size_dict"][0][1] = 3
    with pytest.raises(PlanValidationError, match="network_canon"):
        ExecutionPlan(bad)
    bad = json.loads(json.dumps(rec))
    bad["network"] = {"inputs": [[4]], "output": [4], "size_dict": [[4, 2]]}
    with pytest.raises(PlanValidationError, match="dense first-occurrence"):
        ExecutionPlan(bad)
    bad = json.loads(json.dumps(rec))
    bad["sliced"] = {"legs": [0, 0]}
    with pytest.raises(PlanValidationError, match="twice"):
        ExecutionPlan(bad)
    bad = json.loads(json.dumps(rec))
    bad["ssa_path"] = [[0, 1], [0, 3]]
    with pytest.raises(PlanValidationError):
        ExecutionPlan(bad)


def test_exact_target_is_checked_against_the_slice_set():
    rec = record()
    log2_only = dict(rec, memory_target_log2_elements=1.0, memory_constraint_metric=MEMORY_CONSTRAINT_METRIC)
    with pytest.raises(PlanValidationError, match="exact target_size"):
        ExecutionPlan(log2_only)
    with pytest.raises(PlanValidationError):
        ExecutionPlan(dict(rec, memory_constraint_metric=MEMORY_CONSTRAINT_METRIC))
    with pytest.raises(PlanValidationError):
        ExecutionPlan(dict(rec, target_size=8, memory_constraint_metric=MEMORY_CONSTRAINT_METRIC))
    tgt = dict(rec, target_size=2, memory_target_log2_elements=1.0, memory_constraint_metric=MEMORY_CONSTRAINT_METRIC)
    with pytest.raises(PlanValidationError, match="exceeds declared target_size=2"):
        ExecutionPlan(tgt)
    ok = ExecutionPlan.from_path(TRI_INPUTS, [], TRI_SIZES, TRI_PATH, [0, 1], labels=LABELS, target_size=2)
    assert ok.sliced_legs == [0, 1] and ok.target_size == 2
    big = (1 << 53) + 1  # an exact target beyond f64's integers survives as an integer
    p = ExecutionPlan(dict(rec, target_size=big, memory_target_log2_elements=math.log2(big),
                           memory_constraint_metric=MEMORY_CONSTRAINT_METRIC))
    assert p.target_size == big


def test_versions_other_than_two_are_not_self_contained():
    rec = record()
    with pytest.raises(PlanValidationError, match="version 2 is required"):
        ExecutionPlan(dict(rec, schema_version=1))
    bare = {k: v for k, v in rec.items() if k not in ("schema", "schema_version")}
    with pytest.raises(PlanValidationError, match="schema-less"):
        ExecutionPlan(bare)
    with pytest.raises(PlanValidationError, match="both schema"):
        ExecutionPlan({k: v for k, v in rec.items() if k != "schema"})
    with pytest.raises(PlanValidationError, match="unsupported execution plan schema"):
        ExecutionPlan(dict(rec, schema="other"))


def test_save_and_load(tmp_path):
    net_inputs, sizes = [[0, 1, 2], [2, 3], [3, 0, 4], [4, 1]], {0: 2, 1: 3, 2: 2, 3: 4, 4: 2}
    path = A.greedy(net_inputs, [], sizes)
    plan = ExecutionPlan.from_path(net_inputs, [], sizes, path, [3], target_size=64)
    f = tmp_path / "plan.json"
    plan.save(f)
    again = ExecutionPlan.load(f)
    assert again.to_dict() == plan.to_dict() and again.sliced_legs == [3]
    f.write_text("{not json")
    with pytest.raises(PlanValidationError, match="cannot load"):
        ExecutionPlan.load(f)
    assert network_canon(net_inputs, [], sizes) == plan.to_dict()["network_canon"]


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.complex64, np.complex128])
def test_tensors_bin_round_trip_and_size_check(tmp_path, dtype):
    inputs, sizes = [[0, 1], [1, 2, 3], []], {0: 3, 1: 2, 2: 4, 3: 5}
    rng = np.random.default_rng(0)
    arrays = []
    for t in inputs:
        shape = tuple(sizes[l] for l in t)
        a = rng.standard_normal(shape) + (1j * rng.standard_normal(shape) if np.dtype(dtype).kind == "c" else 0)
        arrays.append(np.asarray(a, dtype=dtype))
    f = tmp_path / "tensors.bin"
    save_tensors_bin(f, arrays)
    assert f.stat().st_size == sum(a.nbytes for a in arrays)
    back = load_tensors_bin(f, inputs, sizes, dtype)
    for a, b in zip(arrays, back):
        assert b.shape == a.shape and b.dtype == np.dtype(dtype) and np.array_equal(a, b)
    raw = f.read_bytes()
    f.write_bytes(raw[:-1])
    with pytest.raises(ValueError, match="expects"):
        load_tensors_bin(f, inputs, sizes, dtype)
    # little-endian on disk: the first float32 element's bytes
    if dtype is np.float32:
        assert raw[:4] == np.float32(arrays[0].flat[0]).astype("<f4").tobytes()


@pytest.mark.gpu
def test_saved_sliced_plan_executes_on_the_gpu(tmp_path):
    from arctn_b200 import networks as N
    from oracle import oracle as O

    net, arrays = N.workload_rand3reg(64, 2, 1, np.complex64, seed=0)
    # the v2 network is dense: relabel legs by first occurrence
    order = {}
    for leg in [l for t in net.inputs for l in t] + list(net.output):
        order.setdefault(leg, len(order))
    inputs = [[order[l] for l in t] for t in net.inputs]
    sizes = {order[l]: d for l, d in net.size_dict.items()}
    path = A.greedy(inputs, [], sizes)
    sliced = A.find_slices_to_size(inputs, [], sizes, path, 2 ** 8)
    plan = ExecutionPlan.from_path(inputs, [], sizes, path, sliced, target_size=2 ** 8)
    plan.save(tmp_path / "plan.json")
    save_tensors_bin(tmp_path / "tensors.bin", arrays)
    loaded = ExecutionPlan.load(tmp_path / "plan.json")
    data = load_tensors_bin(tmp_path / "tensors.bin", loaded.inputs, loaded.size_dict, np.complex64)
    got = complex(loaded.execute(data))
    want = complex(O.contract_sliced(inputs, [], sizes, path, sliced, [a.astype(np.complex128) for a in data]))
    assert abs(got - want) <= 1e-5 * abs(want)


def test_compile_and_execute_options_follow_the_reference():
    # pybind/python/arctn/_execution_plan.py:474-500: compile() serves unsliced plans only; execute() takes an
    # explicit backend and checks it before anything runs.
    unsliced = ExecutionPlan.from_path(TRI_INPUTS, [], TRI_SIZES, TRI_PATH)
    compiled = unsliced.compile(backend="b200")
    assert isinstance(compiled, A.ArcTNCompiledContraction) and compiled.backend == "b200"
    assert [tuple(p) for p in compiled.ssa_path] == TRI_PATH
    sliced = ExecutionPlan.from_path(TRI_INPUTS, [], TRI_SIZES, TRI_PATH, [0])
    with pytest.raises(PlanValidationError, match="sliced plans cannot be compiled"):
        sliced.compile()
    arrays = [np.ones((2, 2))] * 3
    for bad in ("auto", "native", ""):
        with pytest.raises(ValueError, match="backend"):
            sliced.execute(arrays, backend=bad)
    with pytest.raises(PlanValidationError, match="sequence"):
        sliced.execute(5)
    with pytest.raises(PlanValidationError, match="arrays length"):
        sliced.execute(arrays[:2])


def test_plan_object_surface_follows_the_reference():
    # pybind/python/arctn/_execution_plan.py:220-282, 402-472, 579-582
    plan = ExecutionPlan.from_path(TRI_INPUTS, [], TRI_SIZES, TRI_PATH, [0], labels=LABELS, name="triangle")
    assert (plan.schema, plan.schema_version, plan.path_format) == ("arctn-execution-plan", 2, "ssa-v1")
    assert plan.is_sliced and not ExecutionPlan.from_path(TRI_INPUTS, [], TRI_SIZES, TRI_PATH).is_sliced
    assert plan.network_canon == network_canon(TRI_INPUTS, [], TRI_SIZES)
    assert plan.provenance["source"] == "arctn_b200" and plan.planning == {}
    assert plan.to_linear_path() == ((0, 1), (0, 1))
    with pytest.raises(AttributeError, match="immutable"):
        plan.ssa_path = []
    assert plan == ExecutionPlan.from_dict(plan.to_dict())
    assert plan != ExecutionPlan.from_path(TRI_INPUTS, [], TRI_SIZES, TRI_PATH, [1], labels=LABELS, name="triangle")
    # a caller's network with its own labels, numbered in first-occurrence order
    plan.validate([["i", "j"], ["i", "k"], ["j", "k"]], [], {"i": 2, "j": 2, "k": 2})
    with pytest.raises(PlanValidationError, match="does not match the embedded"):
        plan.validate([["i", "j"], ["i", "k"], ["j", "k"]], [], {"i": 2, "j": 3, "k": 2})
    with pytest.raises(PlanValidationError, match="does not match the embedded"):
        plan.validate([["i", "j"], ["i", "k"], ["j", "k"]], [], {"i": 2, "j": 2, "k": 2, "z": 2})
    with pytest.raises(TypeError, match="together"):
        plan.validate([["i", "j"]], [])
    plan.validate(arrays=[np.zeros((2, 2))] * 3)
    with pytest.raises(PlanValidationError, match="shape and dtype"):
        plan.validate(arrays=[[0.0, 0.0]] * 3)
    with pytest.raises(PlanValidationError, match="same dtype"):
        plan.validate(arrays=[np.zeros((2, 2)), np.zeros((2, 2)), np.zeros((2, 2), np.float32)])


def test_arctn_plan_plans_with_greedy_and_the_slice_search(tmp_path):
    # pybind/python/arctn/_execution_plan.py:593-646 with the public planner
    from arctn_b200 import networks as N
    from oracle import oracle as O

    net = N.rand_regular(40, 3, 2, 1)
    names = {l: f"e{l}" for l in net.size_dict}
    inputs = [[names[l] for l in t] for t in net.inputs]
    size = {names[l]: d for l, d in net.size_dict.items()}
    plan = A.arctn_plan(inputs, [], size, target_size=2 ** 6, preset="light", seed=3)
    ids = {}
    for lab in [l for t in inputs for l in t]:
        ids.setdefault(lab, len(ids))
    dense = ([[ids[l] for l in t] for t in inputs], [], {ids[l]: d for l, d in size.items()})
    path = O.greedy(*dense)
    assert [tuple(p) for p in plan.ssa_path] == [tuple(p) for p in path]
    assert plan.sliced_legs == O.find_slices_to_size(*dense, path, 2 ** 6) and plan.is_sliced
    assert plan.target_size == 2 ** 6 and plan.leg_labels == sorted(ids, key=ids.get)
    assert plan.planning["preset"] == "light" and plan.planning["seed"] == 3
    plan.validate(inputs, [], size)
    assert ExecutionPlan.load(plan.save(tmp_path / "plan.json")) == plan
    with pytest.raises(ValueError, match="unreachable"):
        A.arctn_plan([["a"], ["b"]], ["a", "b"], {"a": 2, "b": 2}, target_size=1)
    blocks = A.arctn_plan([["a"], ["b"]], ["a", "b"], {"a": 2, "b": 2}, target_size=2, allow_output_slicing=True)
    assert blocks.sliced_legs and set(blocks.sliced_legs) <= {0, 1}
    with pytest.raises(TypeError, match="rate_enabled"):
        A.arctn_plan([["a"]], ["a"], {"a": 2}, rate_enabled=1)
    with pytest.raises(ValueError, match="preset"):
        A.arctn_plan([["a"]], ["a"], {"a": 2}, preset="x")

"""Bit-exact bookkeeping parity: the product's host plan versus the oracle (CPU only).

Slots, legs, shapes, dangling sums, permutations and GEMM dims of every step
(src/compiled.rs:481-602), the finalize stage, path metrics, the greedy path
and slice selection must be identical -- integers bit for bit, metrics to the
last bit of the f64.
"""

import numpy as np
import pytest

import arctn_b200 as A
from arctn_b200 import networks as N
from oracle import oracle as O
from tests.helpers import SMALL_NETWORKS, known_answers, sd


def product_plan(inputs, output, size_dict, path):
    cc = A.CompiledContraction.compile(inputs, output, size_dict, ssa_path=path)
    steps = []
    for s in cc.pair_steps():
        steps.append(dict(left_slot=s.left_slot(), right_slot=s.right_slot(), result_slot=s.result_slot(),
                          left_legs=list(s.left_legs()), right_legs=list(s.right_legs()),
                          result_legs=list(s.result_legs()), left_shape=list(s.left_shape()),
                          right_shape=list(s.right_shape()), result_shape=list(s.result_shape()),
                          sum_a=list(s.sum_a()), sum_b=list(s.sum_b()), a_perm=list(s.a_perm()),
                          b_perm=list(s.b_perm()), gemm_dims=list(s.gemm_dims())))
    preps = [dict(input_shape=list(p.input_shape()), traces=[list(t) for t in p.traces()], legs=list(p.legs()),
                  shape=list(p.shape())) for p in cc.input_preps()]
    f = cc.finalize()
    fin = dict(slot=f.slot(), input_legs=list(f.input_legs()), input_shape=list(f.input_shape()),
               sum=list(f.sum_axes()), perm=list(f.perm()), output_shape=list(f.output_shape()))
    return dict(n_inputs=cc.n_inputs(), steps=steps, preps=preps, finalize=fin, log10_flops=cc.log10_flops,
                log2_peak_size=cc.log2_peak_size)


def oracle_plan(inputs, output, size_dict, path):
    j = O.plan_json(inputs, output, size_dict, path)
    for k in ("log10_flops", "log2_peak_size"):
        if isinstance(j[k], str):
            j[k] = float(j[k])
    return j


def networks():
    nets = dict(SMALL_NETWORKS)
    for seed in range(25):
        n = 3 + seed % 5
        net = N.random_connected(n, 2, [2, 3, 4], seed % 3, seed + 4200)
        nets[f"rc{seed}"] = net.as_tuple()
    nets["grid6x6_b4"] = N.grid_2d(6, 6, 4).as_tuple()
    nets["grid8x8_b6"] = N.grid_2d(8, 8, 6).as_tuple()
    nets["grid4x5_b2"] = N.grid_2d(4, 5, 2).as_tuple()
    nets["rr64_b2"] = N.rand_regular(64, 3, 2, 1).as_tuple()
    nets["rr172_b2"] = N.rand_regular(172, 3, 2, 1).as_tuple()
    nets["brick10x6"] = N.brickwork_circuit(10, 6, 3)[0].as_tuple()
    return nets


NETS = networks()


@pytest.mark.parametrize("name", sorted(NETS))
def test_greedy_and_plan_match_oracle(name):
    inputs, output, size_dict = NETS[name]
    path = A.greedy(inputs, output, size_dict)
    assert path == O.greedy(inputs, output, size_dict)
    assert product_plan(inputs, output, size_dict, path) == oracle_plan(inputs, output, size_dict, path)
    st = A.simulate_path(inputs, output, size_dict, path)
    so = O.simulate_path(inputs, output, size_dict, path)
    assert {k: float(v) for k, v in st.items()} == {k: float(v) for k, v in so.items()}


@pytest.mark.parametrize("name", ["mixed", "chain3", "hyper"])
def test_fixed_paths_match_oracle(name):
    inputs, output, size_dict = NETS[name]
    n = len(inputs)
    paths = {"mixed": [(0, 1), (2, 6), (3, 4), (8, 5), (7, 9)], "chain3": [(1, 2), (0, 3)],
             "hyper": [(1, 2), (0, 3)]}
    p = paths[name]
    assert len(p) == n - 1
    assert product_plan(inputs, output, size_dict, p) == oracle_plan(inputs, output, size_dict, p)


def test_two_node_geometry():
    # tests/compiled_pair_steps.rs:124-145
    cc = A.CompiledContraction.compile([[0, 1], [1, 2]], [0, 2], {0: 3, 1: 4, 2: 5}, ssa_path=[(0, 1)])
    st = cc.pair_steps()[0]
    assert st.gemm_dims() == (1, 3, 4, 5)
    assert st.result_legs() == (0, 2)
    assert all(p.is_identity() for p in cc.input_preps())
    assert cc.finalize().is_identity()


def test_single_tensor_uses_only_finalize():
    # tests/compiled_pair_steps.rs:147-162
    cc = A.CompiledContraction.compile([[0, 1, 2]], [2, 0], {0: 2, 1: 3, 2: 4}, ssa_path=[])
    assert cc.pair_steps() == []
    assert cc.finalize().slot() == 0 and not cc.finalize().is_identity()


@pytest.mark.parametrize("case", known_answers()["metrics"], ids=lambda c: c["source"])
def test_metric_known_answers(case):
    st = A.simulate_path(case["inputs"], case["output"], sd(case["size_dict"]), [tuple(p) for p in case["ssa_path"]])
    for key, value in case["expect"].items():
        got = 10 ** st[key] if key.startswith("log10") else 2 ** st[key]
        assert abs(got - value) < 1e-9 * value


@pytest.mark.parametrize("case", known_answers()["slice_targets"], ids=lambda c: f"{c['source']}-{c['target']}")
def test_slice_target_known_answers(case):
    got = A.find_slices_to_size(case["inputs"], case["output"], sd(case["size_dict"]),
                                [tuple(p) for p in case["ssa_path"]], case["target"])
    assert got == case["expect"]


@pytest.mark.parametrize("name,target", [("rr64_b2", t) for t in (2 ** 6, 2 ** 7, 2 ** 8, 2 ** 10, 2 ** 24)]
                         + [("rr172_b2", 2 ** 24), ("grid4x5_b2", 2 ** 4), ("grid8x8_b6", 2 ** 22)])
def test_find_slices_matches_oracle(name, target):
    inputs, output, size_dict = NETS[name]
    path = A.greedy(inputs, output, size_dict)
    assert A.find_slices_to_size(inputs, output, size_dict, path, target) == \
        O.find_slices_to_size(inputs, output, size_dict, path, target)


def test_slice_parallel_chunks_matches_oracle():
    for out in (1, 2, 1 << 10, 1 << 20, 1 << 21, 1 << 22, 1 << 24, (1 << 64) - 1):
        for n in list(range(0, 700)) + [1024, 1152, 3456, 4096, 65536, 1 << 40]:
            assert A.slice_parallel_chunks(n, out) == O.slice_parallel_chunks(n, out)


BAD = [
    ("zero dim", [[0, 1], [1, 2]], [0, 2], {0: 2, 1: 0, 2: 2}, [(0, 1)]),
    ("repeated output", [[0, 1], [1, 2]], [0, 0], {0: 2, 1: 2, 2: 2}, [(0, 1)]),
    ("unused size", [[0, 1], [1, 2]], [0, 2], {0: 2, 1: 2, 2: 2, 7: 2}, [(0, 1)]),
    ("missing size", [[0, 1], [1, 2]], [0, 2], {0: 2, 1: 2}, [(0, 1)]),
    ("self contraction", [[0, 1], [1, 2]], [0, 2], {0: 2, 1: 2, 2: 2}, [(0, 0)]),
    ("consumed slot", [[0], [0, 1], [1]], [], {0: 2, 1: 3}, [(0, 1), (0, 2)]),
    ("incomplete", [[0], [0]], [], {0: 2}, []),
    ("triple leg", [[0, 0, 0]], [], {0: 2}, []),
    ("overflow", [[0, 1], [1, 2]], [0, 2], {0: (1 << 63) - 1, 1: 3, 2: 2}, [(0, 1)]),
    ("output not held", [[0, 1], [1, 2]], [0, 3], {0: 2, 1: 2, 2: 2, 3: 2}, [(0, 1)]),
]


@pytest.mark.parametrize("label,inputs,output,size_dict,path", BAD, ids=[b[0] for b in BAD])
def test_invalid_networks_rejected_like_oracle(label, inputs, output, size_dict, path):
    with pytest.raises(O.OracleError):
        O.plan_json(inputs, output, size_dict, path)
    with pytest.raises(ValueError):
        A.CompiledContraction.compile(inputs, output, size_dict, ssa_path=path)


def test_linear_ssa_roundtrip():
    ssa = [(1, 2), (0, 3)]
    lin = A.ssa_to_linear(ssa, 3)
    assert A.linear_to_ssa(lin, 3) == ssa
    with pytest.raises(ValueError):
        A.linear_to_ssa([(0, 5)], 3)


def test_output_slicing_is_opt_in_for_a_unary_network():
    # src/slice.rs:1180-1196: a unary network's output can be fitted only by slicing one of its output legs.
    inputs, output, size_dict = [[0, 1]], [1, 0], {0: 2, 1: 3}
    for find in (A.find_slices_to_size, O.find_slices_to_size):
        assert find(inputs, output, size_dict, [], 2) is None
        assert find(inputs, output, size_dict, [], 2, allow_output_slicing=True) == [1]


def test_output_slicing_skips_a_leg_repeated_inside_one_input():
    # src/slice.rs:1226-1238: the traced output leg cannot be sliced, so no slicing meets the target.
    for find in (A.find_slices_to_size, O.find_slices_to_size):
        assert find([[0, 0]], [0], {0: 2}, [], 1, allow_output_slicing=True) is None


def _open_networks():
    nets = {}
    for seed in range(30):
        net = N.random_connected(3 + seed % 6, 2, [2, 3, 4], 1 + seed % 3, seed + 7300)
        nets[f"open{seed}"] = net.as_tuple()
    return nets


@pytest.mark.parametrize("name", sorted(_open_networks()))
def test_output_slicing_matches_oracle(name):
    inputs, output, size_dict = _open_networks()[name]
    path = A.greedy(inputs, output, size_dict)
    for target in (1, 2, 4, 8, 16, 64):
        got = A.find_slices_to_size(inputs, output, size_dict, path, target, allow_output_slicing=True)
        assert got == O.find_slices_to_size(inputs, output, size_dict, path, target, allow_output_slicing=True)
        assert A.find_slices_to_size(inputs, output, size_dict, path, target) == \
            O.find_slices_to_size(inputs, output, size_dict, path, target)
        if got is not None:
            # every per-slice intermediate fits
            sub = dict(size_dict)
            for l in got:
                sub[l] = 1
            assert A.simulate_path(inputs, output, sub, path)["log2_max_size"] <= np.log2(target) + 1e-12


def test_output_slicing_does_choose_output_legs():
    chosen = 0
    for inputs, output, size_dict in _open_networks().values():
        path = A.greedy(inputs, output, size_dict)
        got = A.find_slices_to_size(inputs, output, size_dict, path, 4, allow_output_slicing=True)
        chosen += got is not None and any(l in output for l in got)
    assert chosen >= 10


def test_max_leg_id_is_safe_and_an_unused_leg_is_rejected():
    # tests/sparse_leg_ids.rs:14-42: leg id u32::MAX in simulation, greedy and a program plan; a size_dict leg
    # that no input uses is rejected, as the reference's network validation does.
    top = 2 ** 32 - 1
    net = ([[top], [top]], [top], {top: 2})
    assert A.greedy(*net) == [(0, 1)]
    assert A.simulate_path(*net, [(0, 1)]) == O.simulate_path(*net, [(0, 1)])
    assert A.simulate_path(*net, [(0, 1)])["log10_flops"] == pytest.approx(np.log10(2.0))
    assert A.SlicedProgram(*net, [(0, 1)], (), dtype=np.float64).describe()["ops"]
    with pytest.raises(ValueError, match="not used by any input"):
        A.simulate_path([[0]], [0], {0: 2, top: 2}, [])

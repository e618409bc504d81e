"""GPU parity: the CUDA executor (through the C ABI) against the oracle.

Tolerances: f64/c128 results within 1e-12 relative of the oracle in the same
dtype; f32/c64 within 1e-5 relative of the FP64 oracle (inputs promoted), the
bound the workloads state for c64.  Relative means max|got - want| / max(1, max|want|).
"""

import itertools

import numpy as np
import pytest

import arctn_b200 as A
from arctn_b200 import networks as N
from oracle import oracle as O
from tests.helpers import SMALL_NETWORKS, case_arrays, case_expected, known_answers, random_arrays, rel_err, sd

pytestmark = pytest.mark.gpu

DTYPES = [np.float32, np.float64, np.complex64, np.complex128]
TOL = {np.dtype(np.float32): 1e-5, np.dtype(np.complex64): 1e-5, np.dtype(np.float64): 1e-12,
       np.dtype(np.complex128): 1e-12}


def oracle_ref(inputs, output, size_dict, path, sliced, arrays):
    """Same-dtype oracle for FP64 dtypes, FP64 oracle for FP32 dtypes."""
    if arrays[0].dtype in (np.float32, np.complex64):
        arrays = O.promote(arrays)
    return O.contract_sliced(inputs, output, size_dict, path, sliced, arrays)


@pytest.mark.parametrize("case", known_answers()["cases"], ids=lambda c: c["name"])
def test_known_answers(case):
    arrays = case_arrays(case)
    size_dict = sd(case["size_dict"])
    path = [tuple(p) for p in case["ssa_path"]]
    got = A.contract_sliced(case["inputs"], case["output"], size_dict, arrays, case["sliced"], ssa_path=path)
    want = case_expected(case)
    if want is None:
        want = O.naive_einsum(case["inputs"], case["output"], size_dict, arrays)
        assert np.max(np.abs(got - want)) < case["tol"]
    else:
        assert np.array_equal(got.ravel(), want.ravel().astype(got.dtype)), (got, want)


@pytest.mark.parametrize("dtype", DTYPES, ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("name", sorted(SMALL_NETWORKS))
def test_small_networks(name, dtype):
    inputs, output, size_dict = SMALL_NETWORKS[name]
    path = A.greedy(inputs, output, size_dict)
    arrays = random_arrays(inputs, size_dict, dtype, 7)
    cc = A.CompiledContraction.compile(inputs, output, size_dict, ssa_path=path)
    got = cc.execute(arrays)
    assert got.dtype == np.dtype(dtype) and got.shape == tuple(size_dict[l] for l in output)
    want = oracle_ref(inputs, output, size_dict, path, [], arrays)
    assert rel_err(got, want) <= TOL[np.dtype(dtype)], rel_err(got, want)


@pytest.mark.parametrize("seed", range(25))
def test_random_networks_f64_c64(seed):
    net = N.random_connected(3 + seed % 5, 2, [2, 3, 4], seed % 3, seed + 4200)
    path = A.greedy(*net.as_tuple())
    for dtype in (np.float64, np.complex64):
        arrays = random_arrays(net.inputs, net.size_dict, dtype, seed * 11)
        got = A.contract_sliced(*net.as_tuple(), arrays, [], ssa_path=path)
        want = oracle_ref(*net.as_tuple(), path, [], arrays)
        assert rel_err(got, want) <= TOL[np.dtype(dtype)]


def test_all_slice_subsets_shared_output_hyperedge():
    # tests/slice_output.rs:9-50: every subset of legs sliced (output-only, internal-only, mixed), reversed order.
    inputs, output = [[0, 1, 4], [1, 2, 4], [1, 3]], [3, 1, 0, 2]
    size_dict = {0: 2, 1: 3, 2: 2, 3: 2, 4: 5}
    path = [(0, 1), (3, 2)]
    for dtype, tol in ((np.float64, 1e-11), (np.float32, 1e-4), (np.complex128, 1e-11), (np.complex64, 1e-4)):
        arrays = random_arrays(inputs, size_dict, dtype, 9817)
        want = O.naive_einsum(inputs, output, size_dict, O.promote(arrays))
        labels = sorted(size_dict)
        for mask in range(1 << len(labels)):
            sliced = [l for i, l in enumerate(labels) if mask >> i & 1][::-1]
            got = A.contract_sliced(inputs, output, size_dict, arrays, sliced, ssa_path=path)
            assert got.shape == want.shape
            assert np.max(np.abs(got - want)) < tol, (dtype, sliced)


@pytest.mark.parametrize("seed", range(6))
def test_sliced_random_networks(seed):
    net = N.random_connected(6, 3, [2, 3], 1, seed + 900)
    path = A.greedy(*net.as_tuple())
    cand = sorted(l for l in net.size_dict if l not in net.output)[:3]
    arrays = random_arrays(net.inputs, net.size_dict, np.float64, seed * 31 + 7)
    got = A.contract_sliced(*net.as_tuple(), arrays, cand, ssa_path=path)
    want = O.contract_sliced(*net.as_tuple(), path, cand, arrays)
    assert rel_err(got, want) < 1e-12


def test_grid6_bond4_c128_and_c64():
    # 6x6 open grid, bond 4, N(0,1)/sqrt(4^rank), greedy, unsliced.
    net, arrays = N.workload_grid6(np.complex128, seed=0)
    path = A.greedy(*net.as_tuple())
    want = O.contract_sliced(*net.as_tuple(), path, [], arrays)
    got = A.contract_sliced(*net.as_tuple(), arrays, [], ssa_path=path)
    assert rel_err(got, want) <= 1e-12
    arr64 = [a.astype(np.complex64) for a in arrays]
    want64 = O.contract_sliced(*net.as_tuple(), path, [], O.promote(arr64))
    got64 = A.contract_sliced(*net.as_tuple(), arr64, [], ssa_path=path)
    assert abs(complex(got64) - complex(want64)) / abs(complex(want64)) <= 1e-5


def test_rand3reg_n64_256_slices_c64():
    # Random 3-regular n=64, bond 2, c64 N(0,1)/sqrt(8); target 2^7 gives 2^8 slices.
    net, arrays = N.workload_rand3reg(64, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 7)
    assert len(sliced) == 8
    want = O.contract_sliced(*net.as_tuple(), path, sliced, O.promote(arrays), threads=8)
    got = A.contract_sliced(*net.as_tuple(), arrays, sliced, ssa_path=path, f64_out=True)
    assert abs(complex(got) - complex(want)) / abs(complex(want)) <= 1e-5
    # Group size never changes a bit of the result (fixed per-slice arithmetic and chunk order).
    bits = set()
    for group in (1, 7, 64, 0):
        prog = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, max_slices_per_group=group)
        bits.add(np.asarray(prog.execute(arrays)).tobytes())
    assert len(bits) == 1


def test_stage_replay_bitwise_equals_execute():
    # tests/compiled_pair_steps.rs:95-122
    import torch

    inputs, output, size_dict = SMALL_NETWORKS["mixed"]
    for path in (A.greedy(inputs, output, size_dict), [(0, 1), (2, 6), (3, 4), (8, 5), (7, 9)]):
        cc = A.CompiledContraction.compile(inputs, output, size_dict, ssa_path=path)
        for dtype in (np.float64, np.complex128, np.complex64):
            arrays = [torch.from_numpy(a).cuda() for a in random_arrays(inputs, size_dict, dtype, 11)]
            want = cc.execute(arrays)
            slots = [p.execute(t) for p, t in zip(cc.input_preps(), arrays)]
            for s, st in enumerate(cc.pair_steps()):
                assert st.result_slot() == cc.n_inputs() + s == len(slots)
                left, right = slots[st.left_slot()], slots[st.right_slot()]
                assert tuple(left.shape) == st.left_shape() and tuple(right.shape) == st.right_shape()
                slots[st.left_slot()] = slots[st.right_slot()] = None
                out = st.execute(left, right)
                assert tuple(out.shape) == st.result_shape()
                slots.append(out)
            got = cc.finalize().execute(slots[cc.finalize().slot()])
            assert torch.equal(got, want)


def test_execute_stripped_extremes_and_reconstruction():
    cc = A.CompiledContraction.compile([[], []], [], {}, ssa_path=[(0, 1)])
    m, e = cc.execute_stripped([np.array(1e200), np.array(1.0)])
    assert e > 199 and abs(abs(float(m)) - 1.0) < 1e-12
    assert abs(float(m) * 10 ** e - 1e200) / 1e200 < 1e-12
    z = np.array(1e200 - 1e200j)
    mc, ec = cc.execute_stripped([z, np.array(1.0 + 0j)])
    assert abs(complex(mc) * 10 ** ec - complex(z)) / abs(complex(z)) < 1e-12
    for seed in range(5):
        net = N.random_connected(3 + seed % 5, 2, [2, 3, 4], seed % 3, seed + 4200)
        path = A.greedy(*net.as_tuple())
        arrays = random_arrays(net.inputs, net.size_dict, np.float64, seed)
        c2 = A.CompiledContraction.compile(*net.as_tuple(), ssa_path=path)
        base = c2.execute(arrays)
        mant, ex = c2.execute_stripped(arrays)
        rebuilt = np.asarray(mant) * 10 ** ex
        assert np.max(np.abs(rebuilt - base) / np.maximum(np.abs(base), 1e-300)) < 1e-9


def test_rejections_before_launch():
    inputs, output, size_dict = [[0, 1], [1, 2]], [0, 2], {0: 2, 1: 3, 2: 4}
    cc = A.CompiledContraction.compile(inputs, output, size_dict, ssa_path=[(0, 1)])
    good = random_arrays(inputs, size_dict, np.float64, 1)
    assert cc.execute(good).shape == (2, 4)
    with pytest.raises(ValueError, match="shape"):
        cc.execute([np.zeros((2, 2)), good[1]])
    with pytest.raises(ValueError):
        cc.execute(good[:1])
    with pytest.raises(ValueError, match="dtype"):
        cc.execute([good[0], good[1].astype(np.float32)])
    with pytest.raises(ValueError):
        A.contract_sliced([[0], [0]], [], {0: 2}, [np.ones(2), np.ones(2)], [0, 0], ssa_path=[(0, 1)])
    with pytest.raises(ValueError, match="repeated inside one input"):
        A.contract_sliced([[0, 0]], [0], {0: 2}, [np.ones((2, 2))], [0], ssa_path=[])
    prog = A.SlicedProgram(inputs, output, size_dict, [(0, 1)], (), dtype=np.float64)
    import torch

    ws = torch.empty(max(prog.workspace_bytes - 1, 0), dtype=torch.uint8, device="cuda")
    if prog.workspace_bytes > 0:
        with pytest.raises(ValueError, match="workspace"):
            prog.execute(good, workspace=ws)


def test_graph_replay_matches_direct_launches():
    net, arrays = N.workload_rand3reg(64, 2, 1, np.complex64, seed=3)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 8)
    import torch

    dev = [torch.from_numpy(a).cuda() for a in arrays]
    g = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, use_graph=True)
    d = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, use_graph=False)
    r1 = g.execute(dev)
    r2 = g.execute(dev)
    r3 = d.execute(dev)
    assert torch.equal(r1, r2) and torch.equal(r1, r3)

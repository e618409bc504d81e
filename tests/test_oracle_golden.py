"""The oracle (CPU restatement of the reference executor) against the reference's own known answers.

Every case comes from a reference test (file:line recorded in tests/golden/known_answers.json).
"""

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import case_arrays, case_expected, known_answers, sd

KA = known_answers()


@pytest.mark.parametrize("case", KA["cases"], ids=lambda c: c["name"])
def test_oracle_execution_known_answers(case):
    arrays = case_arrays(case)
    got = O.contract_sliced(case["inputs"], case["output"], sd(case["size_dict"]), [tuple(p) for p in case["ssa_path"]],
                            case["sliced"], arrays)
    want = case_expected(case)
    if want is None:  # tolerance against the naive einsum, as the reference test does
        want = O.naive_einsum(case["inputs"], case["output"], sd(case["size_dict"]), arrays)
        assert np.max(np.abs(got - want)) < case["tol"]
    elif case["exact"]:
        assert np.array_equal(got.ravel(), want.ravel().astype(got.dtype)), (got, want)


@pytest.mark.parametrize("case", KA["metrics"], ids=lambda c: c["source"])
def test_oracle_metric_known_answers(case):
    st = O.simulate_path(case["inputs"], case["output"], sd(case["size_dict"]), [tuple(p) for p in case["ssa_path"]])
    for key, value in case["expect"].items():
        got = 10 ** st[key] if key.startswith("log10") else 2 ** st[key]
        assert abs(got - value) < 1e-9 * value, (key, got, value)


@pytest.mark.parametrize("case", KA["slice_targets"], ids=lambda c: f"{c['source']}-{c['target']}")
def test_oracle_slice_target_known_answers(case):
    got = O.find_slices_to_size(case["inputs"], case["output"], sd(case["size_dict"]),
                                [tuple(p) for p in case["ssa_path"]], case["target"])
    assert got == case["expect"]


def test_oracle_chunking_covers_ragged_tails():
    # tests/slice_parallel.rs:97-140: chunks are non-empty, contiguous and complete.
    def check(n, out):
        c = O.slice_parallel_chunks(n, out)
        assert c >= 1
        chunk = -(-n // c)
        covered = 0
        for i in range(c):
            lo, hi = i * chunk, min((i + 1) * chunk, n)
            assert lo < hi and lo == covered
            covered = hi
        assert covered == n
        return c

    n = check(257, 1)
    assert 257 % (-(-257 // n)) != 0
    check(3, 1 << 21)
    for out in (1, 1 << 10, 1 << 20, 1 << 21, 1 << 22, 1 << 24):
        for ns in list(range(1, 600, 7)) + [1024, 1152, 3456, 4096, 65536]:
            check(ns, out)
    assert check(1000, (1 << 64) - 1) == 1


def test_oracle_compiled_two_node_geometry():
    # tests/compiled_pair_steps.rs:124-145
    plan = O.plan_json([[0, 1], [1, 2]], [0, 2], {0: 3, 1: 4, 2: 5}, [(0, 1)])
    assert plan["steps"][0]["gemm_dims"] == [1, 3, 4, 5]
    assert plan["steps"][0]["result_legs"] == [0, 2]
    assert all(not p["traces"] for p in plan["preps"])
    assert plan["finalize"]["perm"] == [0, 1] and plan["finalize"]["sum"] == []


def test_oracle_strip_extreme_values():
    # src/compiled.rs:639-669: 1e200 scalars normalise to |m| = 1 with exponent > 199.
    m, e = O.execute([[], []], [], {}, [(0, 1)], [np.array(1e200), np.array(1.0)], strip=True)
    assert e > 199 and abs(abs(float(m)) - 1.0) < 1e-12
    assert abs(float(m) * 10 ** e - 1e200) / 1e200 < 1e-12
    z = np.array(1e200 - 1e200j)
    mc, ec = O.execute([[], []], [], {}, [(0, 1)], [z, np.array(1.0 + 0j)], strip=True)
    assert ec > 199 and abs(abs(complex(mc)) - 1.0) < 1e-12
    assert abs(complex(mc) * 10 ** ec - complex(z)) / abs(complex(z)) < 1e-12


@pytest.mark.parametrize("seed", range(6))
def test_oracle_sliced_matches_naive(seed):
    # tests/correctness.rs:349-371 pattern, with this repo's generator.
    from arctn_b200.networks import random_connected
    from tests.helpers import random_arrays

    net = random_connected(5, 3, [2, 3], 1, seed + 200)
    path = O.greedy(*net.as_tuple())
    cand = sorted(l for l in net.size_dict if l not in net.output)[:2]
    arrays = random_arrays(net.inputs, net.size_dict, np.float64, seed * 13 + 1)
    want = O.naive_einsum(*net.as_tuple(), arrays)
    for threads in (1, 3, 8):
        got = O.contract_sliced(*net.as_tuple(), path, cand, arrays, threads=threads)
        assert np.max(np.abs(got - want)) < 1e-9


def test_torch_step_replay_matches_oracle_execute():
    # The gradient oracle (per-stage einsum replay of the compiled plan) computes the same contraction.
    import torch

    from oracle.torch_replay import replay
    from tests.helpers import SMALL_NETWORKS, random_arrays

    for name, (inputs, output, size_dict) in SMALL_NETWORKS.items():
        path = O.greedy(inputs, output, size_dict)
        arrays = random_arrays(inputs, size_dict, np.complex128, 3)
        got = replay(inputs, output, size_dict, path, [torch.from_numpy(a) for a in arrays]).numpy()
        want = O.execute(inputs, output, size_dict, path, arrays)
        assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, float(np.max(np.abs(want)))), name


def test_oracle_rejects_invalid_slices():
    # tests/slice_output.rs:105-125, tests/slice_validation.rs:33-76
    a = [np.arange(4.0).reshape(2, 2)]
    for sl in ([0, 0], [0, 9]):
        with pytest.raises(O.OracleError):
            O.contract_sliced([[0, 1]], [0, 1], {0: 2, 1: 2}, [], sl, a)
    with pytest.raises(O.OracleError, match="repeated within one input"):
        O.contract_sliced([[0, 0]], [0], {0: 2}, [], [0], a)

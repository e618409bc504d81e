"""GPU parity of the tcgen05 split-TF32 complex GEMM path (precision='tf32x3').

Each case is a pairwise step (or a short contraction) whose dense GEMM is
routed to the tensor-core kernel; results are compared with the FP64 product
of the same complex64 inputs.  Tolerance: 1e-5 relative to max |C| (the c64
bound of the workloads); the device status word must stay 0 (no bounded wait
expired).
"""

import numpy as np
import pytest

import arctn_b200 as A
from oracle import oracle as O
from tests.helpers import random_arrays, rel_err

pytestmark = pytest.mark.gpu


def step_network(bt, m_dims, k_dims, n_dims, seed):
    """Two tensors whose contraction has gemm_dims (bt, prod m, prod k, prod n), legs shuffled."""
    rng = np.random.default_rng(seed)
    leg = iter(range(100))
    b_legs = [next(leg)] if bt > 1 else []
    m_legs = [next(leg) for _ in m_dims]
    k_legs = [next(leg) for _ in k_dims]
    n_legs = [next(leg) for _ in n_dims]
    size = {}
    if bt > 1:
        size[b_legs[0]] = bt
    size.update(zip(m_legs, m_dims))
    size.update(zip(k_legs, k_dims))
    size.update(zip(n_legs, n_dims))
    a = b_legs + m_legs + k_legs
    b = b_legs + k_legs + n_legs
    rng.shuffle(a)
    rng.shuffle(b)
    out = b_legs + m_legs + n_legs
    rng.shuffle(out)
    return [a, b], out, size


CASES = [
    (1, [128], [32], [128]),
    (1, [200], [48], [130]),
    (2, [16, 16], [8, 8], [8, 48]),
    (1, [384], [1000], [96]),
    (3, [97], [33], [99]),
    (1, [2] * 9, [2] * 10, [2] * 9),
]


# Split-TF32 carries each operand to about 2^-22 (1e-5 on these steps); split-BF16 to about 2^-18 and drops
# the lo x lo term, about 2^-17 of each product (1e-4); three-piece split-BF16 carries each operand to about
# 2^-26 and drops terms of at most about 2^-24 of each product (1e-5, like FP32).
PRECISIONS = [("tf32x3", 1e-5), ("bf16x3", 1e-4), ("bf16x6", 1e-5)]


@pytest.mark.parametrize("precision,tol", PRECISIONS, ids=[p for p, _ in PRECISIONS])
@pytest.mark.parametrize("case", CASES, ids=[str(c) for c in CASES])
def test_tc_step_matches_fp64(case, precision, tol):
    bt, md, kd, nd = case
    inputs, output, size = step_network(bt, md, kd, nd, seed=len(md) * 7 + bt)
    arrays = random_arrays(inputs, size, np.complex64, 5)
    prog = A.SlicedProgram(inputs, output, size, [(0, 1)], (), dtype=np.complex64, precision=precision)
    import torch

    x = [torch.from_numpy(a).cuda() for a in arrays]
    ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
    got = prog.execute(x, workspace=ws).cpu().numpy()
    assert prog.device_status(ws) == 0
    want = O.naive_einsum(inputs, output, size, O.promote(arrays)) if np.prod(list(size.values())) <= 2 ** 26 \
        else np.einsum(*sum(([a.astype(np.complex128), t] for a, t in zip(arrays, inputs)), []), output)
    err = rel_err(got, want)
    assert err <= tol, err
    ms, kinds, _ = prog.profile(x, workspace=ws)
    assert 9 in kinds, "the dense step did not run on the tensor-core kernel"


def test_tc_sliced_with_shared_operand():
    # T0[s,i,l] . T1[l,j] . T2[s] -> [i,j], s sliced: the dense step has a per-slice A and a shared B.
    inputs, output = [[0, 1, 2], [2, 3], [0]], [1, 3]
    size = {0: 3, 1: 160, 2: 96, 3: 200}
    arrays = random_arrays(inputs, size, np.complex64, 11)
    want = O.naive_einsum(inputs, output, size, O.promote(arrays))
    for precision, tol in PRECISIONS:
        for group in (1, 2, 0):
            got = A.SlicedProgram(inputs, output, size, [(0, 1), (2, 3)], [0], dtype=np.complex64,
                                  precision=precision, max_slices_per_group=group).execute(arrays)
            assert rel_err(got, want) <= tol, (precision, group)


def test_tc_grid_contraction_matches_fp64_oracle():
    # 5x5 open grid, bond 6: dense steps reach the tensor cores; whole contraction within 1e-5 of FP64.
    from arctn_b200 import networks as N

    net = N.grid_2d(5, 5, 6)
    arrays = N.gaussian_tensors(net, np.complex64, 3, scale_base=6)
    path = A.greedy(*net.as_tuple())
    want = complex(O.contract_sliced(*net.as_tuple(), path, [], O.promote(arrays), threads=8))
    got = complex(A.contract_sliced(*net.as_tuple(), arrays, [], ssa_path=path, precision="tf32x3"))
    got32 = complex(A.contract_sliced(*net.as_tuple(), arrays, [], ssa_path=path, precision="fp32"))
    got_bf = complex(A.contract_sliced(*net.as_tuple(), arrays, [], ssa_path=path, precision="bf16x3"))
    got_b6 = complex(A.contract_sliced(*net.as_tuple(), arrays, [], ssa_path=path, precision="bf16x6"))
    assert abs(got - want) / abs(want) <= 1e-5
    assert abs(got32 - want) / abs(want) <= 1e-5
    assert abs(got_bf - want) / abs(want) <= 1e-4
    assert abs(got_b6 - want) / abs(want) <= 1e-5


def test_epilogue_packs_are_bit_identical_to_separate_packs():
    # rand3reg n=104, 16 slices: tensor-core steps whose result feeds another tensor-core step write that
    # step's packed operand from their epilogue, with the result's legs laid out in the consumer's order.
    # A gradient program keeps the plan's leg order and separate packs; its forward gives the same bits.
    from arctn_b200 import networks as N

    net, arrays = N.workload_rand3reg(104, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 14)
    # the same TMEM chain length in both (forward programs default to 64 of K, gradient programs to 32)
    kw = dict(dtype=np.complex64, precision="tf32x3", max_slices_per_group=4, tc_chain_k=64)
    fused = A.SlicedProgram(*net.as_tuple(), path, sliced, **kw)
    plain = A.SlicedProgram(*net.as_tuple(), path, sliced, gradient=True, **kw)
    assert any("pack_into" in o for o in fused.describe()["ops"])
    assert not any("pack_into" in o for o in plain.describe()["ops"])
    got, ref = fused.execute(arrays), plain.execute(arrays)
    assert np.array_equal(got, ref)
    want = O.contract_sliced(*net.as_tuple(), path, sliced, O.promote(arrays), threads=8)
    assert rel_err(got, want) <= 1e-5


@pytest.mark.parametrize("kind", ["tf32", "bf16"])
def test_tensor_pipe_peak_probe(kind):
    # The probe's MMAs complete (no expired wait) and give a plausible dense rate: above 100 TFLOP/s for
    # either kind, and BF16 (K = 16 per MMA) faster than TF32 (K = 8) at the same N.
    rates = {n: A.tensor_pipe_peak(kind, n, iters=1 << 14, repeats=1) for n in (128, 256)}
    print(kind, rates)
    assert all(100.0 < r < 5000.0 for r in rates.values()), rates
    if kind == "bf16":
        assert rates[256] > A.tensor_pipe_peak("tf32", 256, iters=1 << 14, repeats=1)
        # the three-piece split-BF16 GEMM's MMA stream (random pieces) at the same order of rate
        six = A.tensor_pipe_peak("bf16x6_gemm_stream_random", 128, iters=1 << 11, repeats=1)
        print("bf16x6 gemm stream, random operands", six)
        assert 0.5 * max(rates.values()) < six < 2.0 * max(rates.values()), (six, rates)
    else:
        # the GEMM's own MMA sequence (two interleaved accumulators, operands streaming through its ring layout)
        # runs at the same order of rate as a single accumulator chain over resident operands
        stream = A.tensor_pipe_peak("tf32_gemm_stream", 128, iters=1 << 12, repeats=1)
        print("tf32 gemm stream", stream)
        assert 0.5 * max(rates.values()) < stream < 2.0 * max(rates.values()), (stream, rates)
        # the same stream over random hi / lo operands does the same MMA work
        rand = A.tensor_pipe_peak("tf32_gemm_stream_random", 128, iters=1 << 12, repeats=1)
        print("tf32 gemm stream, random operands", rand)
        assert 0.5 * stream < rand < 2.0 * stream, (rand, stream)
        # a 3M product's nine MMAs per K step into three accumulators (a measurement aid)
        gauss = A.tensor_pipe_peak("tf32_3m_stream_random", 128, iters=1 << 12, repeats=1)
        print("tf32 3M stream, random operands", gauss)
        assert 0.5 * stream < gauss < 2.0 * stream, (gauss, stream)


def test_bf16x6_rand3reg_n104_matches_fp64_oracle():
    # rand3reg n=104, 16 slices: every dense step on the three-piece split-BF16 tensor-core kernel, within the
    # 1e-5 the complex64 path is held to, and no further from FP64 than split-TF32 by more than 2x.
    from arctn_b200 import networks as N

    net, arrays = N.workload_rand3reg(104, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 14)
    want = complex(O.contract_sliced(*net.as_tuple(), path, sliced, O.promote(arrays), threads=8))
    errs = {}
    for precision in ("bf16x6", "tf32x3"):
        prog = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision=precision)
        ops = prog.describe()["ops"]
        assert any(o["kind"] == "gemm_tc" and o["bf16x6"] == (precision == "bf16x6") for o in ops)
        got = complex(prog.execute(arrays, f64_out=True))
        errs[precision] = abs(got - want) / abs(want)
    print("rand3reg n104 rel err", errs)
    assert errs["bf16x6"] <= 1e-5
    assert errs["bf16x6"] <= max(2 * errs["tf32x3"], 2e-6)


def test_tmem_chain_lengths_match_fp64_oracle():
    # 32, 64 (the forward default) and 128 of K per TMEM chain before the FP32 register sum: all within the
    # 1e-5 the complex64 path is held to on rand3reg n=104 (16 slices), the error growing with the chain.
    from arctn_b200 import _capi as C
    from arctn_b200 import networks as N

    net, arrays = N.workload_rand3reg(104, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 14)
    want = complex(O.contract_sliced(*net.as_tuple(), path, sliced, O.promote(arrays), threads=8))
    prog = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3")
    errs = {}
    for k in (32, 64, 128):
        C.check(C.lib().arctn_b200_program_set_tc_chain(prog._h, k))
        assert all(o["tmem_chunk_k"] == k for o in prog.describe()["ops"] if o["kind"] == "gemm_tc")
        errs[k] = abs(complex(prog.execute(arrays, f64_out=True)) - want) / abs(want)
    print("tmem chain errors", errs)
    assert max(errs.values()) <= 1e-5

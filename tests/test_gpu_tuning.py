"""GEMM autotuner on the GPU: every kernel variant a tuning table can pin gives results within tolerance of
the oracle, and a tuned program (the timed search of arctn_b200.tuning.autotune) matches the oracle with
every GEMM run by the variant its table chose.

Tolerances: f64/c128 within 1e-12 of the same-dtype oracle; f32/c64 within 1e-5 relative of the FP64
oracle, or, where the network's result cancels so far that the reference's own executor in that dtype misses
1e-5 (the float32 rand3reg n=64 case: 3.2e-5 for a result of 5.5e-19), no further from FP64 than that
executor.
"""

import numpy as np
import pytest

import arctn_b200 as A
from arctn_b200 import _capi as C
from arctn_b200 import networks as N
from arctn_b200 import tuning as T
from oracle import oracle as O
from tests.helpers import random_arrays

pytestmark = pytest.mark.gpu

CODES = {np.dtype(np.float32): C.F32, np.dtype(np.float64): C.F64, np.dtype(np.complex64): C.C64,
         np.dtype(np.complex128): C.C128}
PRECS = {"fp32": C.PREC_FP32, "tf32x3": C.PREC_TF32X3, "bf16x3": C.PREC_BF16X3, "bf16x6": C.PREC_BF16X6}


def valid(variant, dtype, precision):
    if variant in ("tc_stream", "tc_deep", "tc_pair", "tc_pair_stream"):
        return precision == "tf32x3" and dtype in (C.F32, C.C64)
    if variant.startswith("tc_"):
        return precision in ("tf32x3", "bf16x3", "bf16x6") and dtype in (C.F32, C.C64)
    return variant != "simt_tile128" or dtype == C.F32


def workload(n, dtype, target_log2):
    net, arrays = N.workload_rand3reg(n, 2, 1, dtype, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** target_log2) or []
    return net, arrays, path, sliced


def rel(got, want):
    """Relative error of a scalar (or max-norm relative error of a tensor) output."""
    got, want = np.asarray(got, dtype=np.complex128), np.asarray(want, dtype=np.complex128)
    return float(np.max(np.abs(got - want)) / np.max(np.abs(want)))


def expected(net, path, sliced, arrays):
    wide = arrays[0].dtype in (np.float32, np.complex64)
    return O.contract_sliced(*net.as_tuple(), path, sliced, O.promote(arrays) if wide else arrays, threads=8)


CASES = [  # (nodes, dtype, precision, slicing target): n=64 has small GEMMs, n=104 tensor-core sized ones
    (64, np.complex64, "tf32x3", 8),
    (104, np.complex64, "tf32x3", 14),
    (64, np.float32, "tf32x3", 8),
    (64, np.complex128, "fp32", 8),
    (64, np.float64, "fp32", 8),
]


@pytest.mark.parametrize("nodes,dtype,precision,target", CASES,
                         ids=[f"n{c[0]}-{np.dtype(c[1]).name}-{c[2]}" for c in CASES])
def test_every_variant_matches_oracle(nodes, dtype, precision, target):
    net, arrays, path, sliced = workload(nodes, dtype, target)
    want = expected(net, path, sliced, arrays)
    if np.dtype(dtype) in (np.float32, np.complex64):
        native = O.contract_sliced(*net.as_tuple(), path, sliced, arrays, threads=8)  # the reference's FP32 form
        tol = max(1e-5, rel(native, want))
    else:
        tol = 1e-12
    code, prec = CODES[np.dtype(dtype)], PRECS[precision]
    base = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=dtype, precision=precision)
    keys = sorted({T.key_of(g) for g in base.gemms()})
    ran = 0
    for v in T.VARIANT_NAMES[1:]:
        if not valid(v, code, prec):
            continue
        table = T.TuneTable()
        for k in keys:
            table.set(k, v)
        prog = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=dtype, precision=precision, tuning=table)
        assert all(g["variant"] == v and g["tuned"] for g in prog.gemms())
        got = prog.execute(arrays, f64_out=True)
        err = rel(got, want)
        assert err <= tol, (v, err)
        ran += 1
    assert ran >= 5


def test_autotune_picks_timed_winners_and_matches_oracle():
    net, arrays, path, sliced = workload(104, np.complex64, 14)
    table = A.autotune(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3")
    prog = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3", tuning=table)
    gs = prog.gemms()
    assert gs and all(g["tuned"] for g in gs)
    for g in gs:
        key = T.key_of(g)
        tm = table.timings(key)
        times = {v: t for v, t in tm.items() if v in T.VARIANT_CODES and t is not None}
        assert tm["heuristic"] in times  # the heuristic's own choice is always timed
        assert g["variant"] == table.get(key) in times
        # the pick is the fastest of its family (tensor core / SIMT) where that beats the heuristic's choice by
        # more than the margin (3%), else the heuristic's choice; a switch of family was kept only where the
        # whole program got faster
        fam = {v: t for v, t in times.items() if v.startswith("tc_") == g["variant"].startswith("tc_")}
        best = min(fam, key=fam.get)
        if g["variant"] != best:  # kept the heuristic's: within the margin, or the whole program said no
            assert g["variant"] == tm["heuristic"]
            w = tm.get("whole_program_ms")
            assert fam[best] >= 0.97 * fam[tm["heuristic"]] or (w and w["after"] >= 0.99 * w["before"])
        if g["variant"].startswith("tc_") != tm["heuristic"].startswith("tc_"):
            w = tm["whole_program_ms"]
            assert w["after"] < w["before"]
    got = prog.execute(arrays, f64_out=True)
    assert rel(got, expected(net, path, sliced, arrays)) <= 1e-5
    # a second run over the same network times nothing new
    again = A.autotune(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3", table=table)
    assert again is table and sorted(again.keys()) == sorted(table.keys())
    # and the table survives a JSON round trip with the same choices
    back = T.TuneTable.from_json(table.to_json())
    p2 = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3", tuning=back)
    assert [g["variant"] for g in p2.gemms()] == [g["variant"] for g in gs]
    assert np.array_equal(np.asarray(p2.execute(arrays, f64_out=True)), np.asarray(got))


PAIR_STEPS = [  # (bt, m dims, k dims, n dims): m >= 256, so both CTAs of a pair hold rows; 384 and 300 leave the
    (1, [512], [64], [256]),  # second CTA of the last 256-row tile partly or wholly past the operand
    (1, [384], [1000], [96]),
    (2, [300], [48], [130]),
]


@pytest.mark.parametrize("case", PAIR_STEPS, ids=[str(c) for c in PAIR_STEPS])
def test_cta_pair_step_matches_single_cta_bitwise_and_fp64(case):
    import torch

    from tests.test_gpu_tc import step_network

    bt, md, kd, nd = case
    inputs, output, size = step_network(bt, md, kd, nd, seed=11 + bt)
    arrays = random_arrays(inputs, size, np.complex64, 5)
    x = [torch.from_numpy(a).cuda() for a in arrays]
    outs = {}
    for v in ("tc_mfast", "tc_pair", "tc_pair_stream"):
        base = A.SlicedProgram(inputs, output, size, [(0, 1)], (), dtype=np.complex64, precision="tf32x3")
        table = T.TuneTable()
        for g in base.gemms():
            table.set(T.key_of(g), v)
        prog = A.SlicedProgram(inputs, output, size, [(0, 1)], (), dtype=np.complex64, precision="tf32x3",
                               tuning=table)
        assert [g["variant"] for g in prog.gemms()] == [v]
        ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
        outs[v] = prog.execute(x, workspace=ws).cpu().numpy()
        assert prog.device_status(ws) == 0
    # a pair computes each output element with the same MMA sequence as one CTA
    assert np.array_equal(outs["tc_pair"], outs["tc_mfast"])
    assert np.array_equal(outs["tc_pair_stream"], outs["tc_mfast"])
    want = np.einsum(*sum(([a.astype(np.complex128), t] for a, t in zip(arrays, inputs)), []), output)
    assert rel(outs["tc_pair"], want) <= 1e-5


def test_cta_pair_on_fused_pack_steps_of_rand3reg_n172():
    # slices 0..3 of the n=172 contraction: its large steps (m = 512 and 1024) write the next GEMM's packed
    # operand from the epilogue; pinned to CTA pairs they give the single-CTA kernel's bits
    net, arrays = N.workload_rand3reg(172, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 24)
    kw = dict(dtype=np.complex64, precision="tf32x3", slice_begin=0, slice_end=4, workspace_budget=8 << 30)
    base = A.SlicedProgram(*net.as_tuple(), path, sliced, **kw)
    big = [T.key_of(g) for g in base.gemms() if g["variant"].startswith("tc_") and g["m"] >= 256]
    assert big
    got = {}
    for v in ("tc_mfast", "tc_pair", "tc_pair_stream"):
        table = T.TuneTable()
        for k in big:
            table.set(k, v)
        prog = A.SlicedProgram(*net.as_tuple(), path, sliced, tuning=table, **kw)
        assert any("pack_into" in o for o in prog.describe()["ops"] if o.get("variant") == v)
        got[v] = np.asarray(prog.execute(arrays, f64_out=True))
    assert np.array_equal(got["tc_pair"], got["tc_mfast"])
    assert np.array_equal(got["tc_pair_stream"], got["tc_mfast"])

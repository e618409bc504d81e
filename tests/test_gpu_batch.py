"""GPU parity of ProgramBatch: many uneven networks (mixed float32 / complex64) as one graph launch.

The batch launches exactly the kernels each program launches on its own, on other streams and in
another order, so its outputs and gradients must equal the single-program results bit for bit; the
values are also checked against the oracle (FP64 CPU restatement) at the dtype's tolerance.
"""

import numpy as np
import pytest
import torch

import arctn_b200 as A
from arctn_b200 import networks as N
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def build(count, seed, gradient=False, precision="fp32"):
    nets = N.workload_batch(count, seed=seed)
    progs, xs = [], []
    for net, arrays in nets:
        path = A.greedy(*net.as_tuple())
        progs.append(A.SlicedProgram(*net.as_tuple(), path, (), dtype=arrays[0].dtype, precision=precision,
                                     gradient=gradient, use_graph=False))
        xs.append([torch.from_numpy(a).cuda() for a in arrays])
    return nets, progs, xs


MODES = [("persistent", True), ("staged", True), ("persistent", False), ("lanes", True)]


def run_batch(batch, fn, xs, ws, side_stream):
    """Two calls (the second replays the captured graph) on a side stream, where the graph form and the
    persistent interpreter run, or on the default stream, where the lane form launches directly."""
    st = torch.cuda.Stream() if side_stream else torch.cuda.current_stream()
    with torch.cuda.stream(st):
        for _ in range(2):
            res = getattr(batch, fn)(xs, workspace=ws, stream=st)
        st.synchronize()
        assert batch.device_status(ws, stream=st) == 0
    return res


@pytest.mark.parametrize("mode,side_stream", MODES)
@pytest.mark.parametrize("precision", ["fp32", "tf32x3"])
def test_batch_execute_equals_single_programs_and_oracle(precision, mode, side_stream):
    nets, progs, xs = build(24, 1, precision=precision)
    batch = A.ProgramBatch(progs, max_lanes=8, mode=mode)
    assert batch.lanes == 8
    ws = torch.empty(max(batch.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
    outs = run_batch(batch, "execute", xs, ws, side_stream)
    for (net, arrays), p, x, o in zip(nets, progs, xs, outs):
        single = p.execute(x)
        assert torch.equal(o, single)
        path = A.greedy(*net.as_tuple())
        want = complex(O.contract_sliced(*net.as_tuple(), path, [], [a.astype(np.complex128) for a in arrays]))
        native = complex(O.contract_sliced(*net.as_tuple(), path, [], arrays))  # the CPU executor in FP32
        got = complex(o.item())
        # 1e-5 relative to the FP64 value (these networks measure at most 5.2e-6 under tf32x3 and 3.3e-6
        # under fp32, where the FP32 CPU executor is at most 2.7e-6)
        assert abs(got - want) <= 1e-5 * abs(want), (got, native, want)


@pytest.mark.parametrize("mode,side_stream", MODES)
@pytest.mark.parametrize("precision", ["fp32", "tf32x3"])
def test_batch_gradient_equals_single_programs(precision, mode, side_stream):
    # seed 0: networks 5 and 7 have tensor-core steps under tf32x3 (staged launches between interpreter launches)
    nets, progs, xs = build(12, 0, gradient=True, precision=precision)
    batch = A.ProgramBatch(progs, max_lanes=4, mode=mode)
    ws = torch.empty(max(batch.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
    outs, grads = run_batch(batch, "gradient", xs, ws, side_stream)
    torch.cuda.synchronize()
    for p, x, o, g in zip(progs, xs, outs, grads):
        o1, g1 = p.gradient(x)
        assert torch.equal(o, o1)
        assert len(g) == len(g1)
        for a, b in zip(g, g1):
            assert torch.equal(a, b)


def test_batch_rejects_mismatched_inputs_before_launch():
    nets, progs, xs = build(3, 3)
    batch = A.ProgramBatch(progs)
    with pytest.raises(ValueError):
        batch.execute(xs[:2])
    bad = [list(x) for x in xs]
    bad[1][0] = bad[1][0].to(torch.complex128)
    with pytest.raises(ValueError):
        batch.execute(bad)
    with pytest.raises(ValueError, match="gradient"):
        batch.gradient(xs)


def test_interpreter_wait_expires_into_status():
    # a dependency that nothing completes: the bounded wait records code 16 and the launch drains; the
    # context stays usable for the next batch run
    import ctypes

    from arctn_b200 import _capi as C

    st = torch.cuda.Stream()
    code = ctypes.c_int(-1)
    C.check(C.lib().arctn_b200_batch_wait_selftest(ctypes.c_void_p(st.cuda_stream), ctypes.byref(code)), "selftest")
    assert code.value == 16
    nets, progs, xs = build(4, 3)
    batch = A.ProgramBatch(progs)
    ws = torch.empty(max(batch.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
    outs = run_batch(batch, "execute", xs, ws, True)
    for p, x, o in zip(progs, xs, outs):
        assert torch.equal(o, p.execute(x))


@pytest.mark.parametrize("fn", ["execute", "gradient"])
def test_batch_numpy_inputs_match_cuda_inputs(fn):
    # NumPy callers go through one staging copy in and one copy out, with the device buffers reused on the
    # next call on the same stream (graph replay); the results must equal the CUDA-tensor path bit for bit
    nets, progs, xs = build(10, 0, gradient=fn == "gradient", precision="tf32x3")
    host = [arrays for _, arrays in nets]
    batch = A.ProgramBatch(progs, max_lanes=4)
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        ref = getattr(batch, fn)(xs, stream=st)
        st.synchronize()
        for _ in range(2):
            got = getattr(batch, fn)(host, stream=st)
    if fn == "execute":
        ref, got = (ref, None), (got, None)
    for o_ref, o_got in zip(ref[0], got[0]):
        assert isinstance(o_got, np.ndarray) and np.array_equal(o_ref.cpu().numpy(), o_got)
    if fn == "gradient":
        for g_ref, g_got in zip(ref[1], got[1]):
            assert len(g_ref) == len(g_got)
            for a, b in zip(g_ref, g_got):
                assert b.shape == tuple(a.shape) and np.array_equal(a.cpu().numpy(), b)


@pytest.mark.parametrize("nodes,target,precision", [(64, 7, "fp32"), (64, 7, "tf32x3"), (104, 14, "tf32x3")])
def test_sliced_program_as_staged_batch(nodes, target, precision):
    # A sliced contraction run by the staged scheduler: all its slices' SIMT steps inside persistent interpreter
    # launches (one for rand3reg n=64, whose steps are all SIMT), the tensor-core steps launched between them.
    # The bits equal the program's own execute, and the value matches the oracle.
    net, arrays = N.workload_rand3reg(nodes, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** target)
    assert len(sliced) >= 4
    prog = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision=precision)
    x = [torch.from_numpy(a).cuda() for a in arrays]
    ref = prog.execute(x)
    batch = A.ProgramBatch([prog], max_lanes=8, mode="staged")
    part = next(p for p in batch.describe()["parts"] if p["part"] == -1)
    if nodes == 64:
        assert part["stages"] == 1 and sum(part["stage_launches"]) == 0  # one persistent launch for every slice
    else:
        assert sum(part["stage_launches"]) > 0
    ws = torch.empty(max(batch.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
    (out,) = run_batch(batch, "execute", [x], ws, True)
    assert torch.equal(out, ref)
    want = complex(O.contract_sliced(*net.as_tuple(), path, sliced, O.promote(arrays), threads=8))
    assert abs(complex(out.item()) - want) / abs(want) <= 1e-5

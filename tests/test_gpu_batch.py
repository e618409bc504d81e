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


@pytest.mark.parametrize("precision", ["fp32", "tf32x3"])
def test_batch_execute_equals_single_programs_and_oracle(precision):
    nets, progs, xs = build(24, 1, precision=precision)
    batch = A.ProgramBatch(progs, max_lanes=8)
    assert batch.lanes == 8
    ws = torch.empty(max(batch.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
    for _ in range(2):  # the second call replays the captured graph
        outs = batch.execute(xs, workspace=ws)
    assert batch.device_status(ws) == 0
    for (net, arrays), p, x, o in zip(nets, progs, xs, outs):
        single = p.execute(x)
        assert torch.equal(o, single)
        path = A.greedy(*net.as_tuple())
        want = complex(O.contract_sliced(*net.as_tuple(), path, [], [a.astype(np.complex128) for a in arrays]))
        native = complex(O.contract_sliced(*net.as_tuple(), path, [], arrays))  # the CPU executor in FP32
        got = complex(o.item())
        # 1e-5 relative, or within 8x of the FP32 CPU executor's own error where the network cancels
        assert abs(got - want) <= max(1e-5 * abs(want), 8 * abs(native - want)), (got, native, want)


def test_batch_gradient_equals_single_programs():
    nets, progs, xs = build(12, 2, gradient=True)
    batch = A.ProgramBatch(progs, max_lanes=4)
    outs, grads = batch.gradient(xs)
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

"""A program and a batch keep working after a failure injected on the host (arctn_b200_debug_inject_failure).

The injected failure happens at the call's entry, before any CUDA work, so nothing faults on the GPU; the
call raises ArcTNB200Error with the CUDA status, and the next call returns the same bits as before it.
"""

import numpy as np
import pytest
import torch

import arctn_b200 as A
from arctn_b200 import _capi as C
from arctn_b200 import networks as N

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def disarmed():
    yield
    for site in (0, 1):
        assert C.lib().arctn_b200_debug_inject_failure(site, 0) == 0


def test_program_recovers_after_an_injected_execute_failure():
    net, arrays = N.workload_rand3reg(64, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 8)
    prog = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3")
    x = [torch.from_numpy(a).cuda() for a in arrays]
    before = prog.execute(x).clone()
    assert C.lib().arctn_b200_debug_inject_failure(0, 1) == 0
    with pytest.raises(A.ArcTNB200Error, match="injected") as info:
        prog.execute(x)
    assert info.value.code == C.ERR_CUDA
    assert torch.equal(prog.execute(x), before)


def test_batch_recovers_after_an_injected_gradient_failure():
    nets = N.workload_batch(6, seed=0)
    progs = [A.SlicedProgram(*net.as_tuple(), A.greedy(*net.as_tuple()), (), dtype=arrays[0].dtype, gradient=True,
                             use_graph=False) for net, arrays in nets]
    xs = [[torch.from_numpy(a).cuda() for a in arrays] for _, arrays in nets]
    batch = A.ProgramBatch(progs, max_lanes=2)
    outs0, grads0 = batch.gradient(xs)
    outs0 = [o.clone() for o in outs0]
    grads0 = [[g.clone() for g in gs] for gs in grads0]
    assert C.lib().arctn_b200_debug_inject_failure(0, 1) == 0
    with pytest.raises(A.ArcTNB200Error, match="injected"):
        batch.gradient(xs)
    outs1, grads1 = batch.gradient(xs)
    torch.cuda.synchronize()
    for o0, o1, g0, g1 in zip(outs0, outs1, grads0, grads1):
        assert torch.equal(o0, o1)
        assert all(torch.equal(a, b) for a, b in zip(g0, g1))

"""Many uneven networks sharded by LPT, each share run as one ProgramBatch (forward + adjoint) on the GPU.

One GPU per call, so the ranks are emulated in one process: each rank's share runs as its own ProgramBatch in
turn, and run_sharded assembles the results through a gather that returns every rank's part (the multi-process
protocol over gloo is covered on CPU by tests/test_sharding.py).  Each network's output and input gradients
must equal that network's own program run alone bit for bit: a batch launches the same kernels as its single
programs, whichever networks share it.
"""

import numpy as np
import pytest
import torch

import arctn_b200 as A
from arctn_b200 import networks as N
from arctn_b200.sharding import lpt_shard, run_sharded

pytestmark = pytest.mark.gpu

COUNT, SEED = 16, 0


def _networks():
    nets = N.workload_batch(COUNT, seed=SEED)
    paths = [A.greedy(*net.as_tuple()) for net, _ in nets]
    costs = [10 ** A.simulate_path(*net.as_tuple(), p)["log10_flops"] for (net, _), p in zip(nets, paths)]
    return nets, paths, costs


def _program(net, arrays, path):
    return A.SlicedProgram(*net.as_tuple(), path, (), dtype=arrays[0].dtype, precision="tf32x3", gradient=True,
                           use_graph=False)


def _run_share(nets, paths, indices):
    """One rank's share as one ProgramBatch: (output, input gradients) per network, as NumPy arrays."""
    progs = [_program(*nets[i], paths[i]) for i in indices]
    xs = [[torch.from_numpy(a).cuda() for a in nets[i][1]] for i in indices]
    batch = A.ProgramBatch(progs, max_lanes=4)
    ws = torch.empty(max(batch.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        outs, grads = batch.gradient(xs, workspace=ws, stream=st)
        st.synchronize()
        assert batch.device_status(ws, stream=st) == 0
    return [(o.cpu().numpy(), [g.cpu().numpy() for g in gs]) for o, gs in zip(outs, grads)]


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_batches_equal_single_programs(world):
    nets, paths, costs = _networks()
    shares = lpt_shard(costs, world)
    assert all(shares)  # every rank gets work
    parts = [list(zip(share, _run_share(nets, paths, share))) for share in shares]
    for rank in range(world):
        mine = dict(parts[rank])
        results = run_sharded(costs, lambda idx: [mine[i] for i in idx], rank, world, gather=lambda obj: parts)
        assert len(results) == COUNT
        for (net, arrays), path, (out, grads) in zip(nets, paths, results):
            o1, g1 = _program(net, arrays, path).gradient([torch.from_numpy(a).cuda() for a in arrays])
            assert np.array_equal(out, o1.cpu().numpy())
            assert len(grads) == len(g1)
            for a, b in zip(grads, g1):
                assert np.array_equal(a, b.cpu().numpy())

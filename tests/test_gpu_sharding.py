"""Many uneven networks sharded across ranks by LPT, each share run as one ProgramBatch (forward + adjoint).

Two and three ranks are spawned processes sharing cuda:0; their batches are independent (no kernel waits on
another rank) and the one gather runs over gloo.  Each network's output and input gradients, gathered in
network order on every rank, must equal that network's own program run alone bit for bit: the batch launches
the same kernels as the single programs.
"""

import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import arctn_b200 as A
from arctn_b200 import networks as N
from arctn_b200.sharding import lpt_shard, run_sharded

pytestmark = pytest.mark.gpu

COUNT, SEED = 16, 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _networks():
    nets = N.workload_batch(COUNT, seed=SEED)
    paths = [A.greedy(*net.as_tuple()) for net, _ in nets]
    costs = [10 ** A.simulate_path(*net.as_tuple(), p)["log10_flops"] for (net, _), p in zip(nets, paths)]
    return nets, paths, costs


def _program(net, arrays, path):
    return A.SlicedProgram(*net.as_tuple(), path, (), dtype=arrays[0].dtype, precision="tf32x3", gradient=True,
                           use_graph=False)


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        nets, paths, costs = _networks()

        def execute_share(indices):
            progs = [_program(*nets[i], paths[i]) for i in indices]
            xs = [[torch.from_numpy(a).cuda() for a in nets[i][1]] for i in indices]
            batch = A.ProgramBatch(progs, max_lanes=4)
            ws = torch.empty(max(batch.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                outs, grads = batch.gradient(xs, workspace=ws, stream=st)
                st.synchronize()
                if batch.device_status(ws, stream=st) != 0:
                    raise RuntimeError("a bounded wait in the batch expired")
            return [(o.cpu().numpy(), [g.cpu().numpy() for g in gs]) for o, gs in zip(outs, grads)]

        results = run_sharded(costs, execute_share, rank, world)
        q.put((rank, results))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_batches_equal_single_programs(world):
    nets, paths, costs = _networks()
    shares = lpt_shard(costs, world)
    assert all(shares)  # every rank gets work
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    mp.start_processes(_worker, args=(world, _free_port(), q), nprocs=world, join=True, start_method="spawn")
    got = sorted((q.get(timeout=120) for _ in range(world)), key=lambda r: r[0])
    for (net, arrays), path, *per_rank in zip(nets, paths, *[r[1] for r in got]):
        o1, g1 = _program(net, arrays, path).gradient([torch.from_numpy(a).cuda() for a in arrays])
        for out, grads in per_rank:  # the same gathered result on every rank
            assert np.array_equal(out, o1.cpu().numpy())
            assert len(grads) == len(g1)
            for a, b in zip(grads, g1):
                assert np.array_equal(a, b.cpu().numpy())

"""The product's slice-sharded contraction across ranks, on one GPU.

Mirrors the reference's MPI path (src/bin/tnmpi.rs): each rank takes the contiguous slice range
slice_range(n, ranks, rank), contracts it with the product's slice-range program (SlicedProgram with
slice_begin / slice_end) into an FP64 partial, and one all-reduce(SUM) assembles the result.  The ranks are
spawned processes that share cuda:0; their kernels never wait on one another (each rank's program is
independent and the sum runs over gloo on host copies of the partials), so sharing one GPU changes nothing but
the timing.  bench.py's multi-GPU form runs the same programs with the all-reduce over NCCL.
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
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _workload():
    net, arrays = N.workload_rand3reg(64, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 8)
    return net, arrays, path, sliced


def _worker(rank, world, port, precision, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        net, arrays, path, sliced = _workload()
        size = net.as_tuple()[2]
        n = int(np.prod([size[leg] for leg in sliced]))
        b, e = A.slice_range(n, world, rank)
        part = torch.zeros(2, dtype=torch.float64)
        status, got = 0, 0j
        if b < e:
            prog = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision=precision,
                                   slice_begin=b, slice_end=e)
            ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device="cuda:0")
            x = [torch.from_numpy(a).cuda() for a in arrays]
            got = complex(prog.execute(x, workspace=ws, f64_out=True).item())
            status = prog.device_status(ws)
            part[:] = torch.tensor([got.real, got.imag], dtype=torch.float64)
        dist.all_reduce(part)
        mine = torch.tensor([float(status), float(b), float(e), got.real, got.imag], dtype=torch.float64)
        gathered = [torch.zeros(5, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(gathered, mine)
        if rank == 0:
            q.put((complex(part[0].item(), part[1].item()), [g.tolist() for g in gathered]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision", ["fp32", "tf32x3"])
@pytest.mark.parametrize("world", [2, 3])
def test_product_slice_ranges_all_reduce_to_the_single_rank_result(world, precision):
    net, arrays, path, sliced = _workload()
    full = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision=precision)
    single = complex(full.execute(arrays, f64_out=True).item())
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    mp.start_processes(_worker, args=(world, _free_port(), precision, q), nprocs=world, join=True,
                       start_method="spawn")
    got, ranks = q.get(timeout=60)
    assert all(int(r[0]) == 0 for r in ranks)  # no bounded device wait expired on any rank
    covered = 0
    for _, lo, hi, _, _ in ranks:  # the ranges tile [0, n) in rank order
        assert int(lo) == covered and hi >= lo
        covered = int(hi)
    size = net.as_tuple()[2]
    assert covered == int(np.prod([size[leg] for leg in sliced]))
    # the all-reduced partials sum to the single program's FP64 sum up to the order of the additions
    scale = sum(abs(complex(r[3], r[4])) for r in ranks)
    assert abs(got - single) <= 1e-12 * scale, (got, single, ranks)
    want = complex(O.contract_sliced(*net.as_tuple(), path, sliced, O.promote(arrays), threads=8))
    assert abs(got - want) <= 1e-5 * abs(want), (got, want)

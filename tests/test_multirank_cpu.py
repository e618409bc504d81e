"""Slice-sharded contraction across ranks, on CPU with torch.distributed gloo (world size 2 and 3).

Mirrors the reference's MPI path (src/bin/tnmpi.rs): each rank takes the contiguous
slice range slice_range(n, ranks, rank), contracts it into a zeroed full output
(the oracle's contract_slice_range), and one all-reduce(SUM) assembles the result.
Each rank also builds the product's slice-range program (SlicedProgram with
slice_begin/slice_end, host-only) for its range: the ranges it reports, gathered over
the group, tile [0, n) in rank order, and its flops add up to the full program's.  The
GPU path runs those programs and all-reduces their FP64 partials over NCCL; here the
partition and the collective are exercised without a GPU.  Also covers more ranks
than slices (empty ranges) and output-leg slicing.
"""

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import arctn_b200 as A
from oracle import oracle as O
from tests.helpers import random_arrays


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


CASES = {
    "internal": ([[0, 1], [1, 2], [2, 3]], [0, 3], {0: 2, 1: 3, 2: 5, 3: 2}, [(0, 1), (3, 2)], [1, 2]),
    "output_and_internal": ([[0, 1, 4], [1, 2, 4], [1, 3]], [3, 1, 0, 2], {0: 2, 1: 3, 2: 2, 3: 2, 4: 5},
                            [(0, 1), (3, 2)], [4, 0]),
    "one_slice": ([[0], [0]], [], {0: 2}, [(0, 1)], [0]),
}


def _worker(rank, world, port, name, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        inputs, output, size_dict, path, sliced = CASES[name]
        arrays = random_arrays(inputs, size_dict, np.float64, 7)
        n = int(np.prod([size_dict[l] for l in sliced]))
        b, e = A.slice_range(n, world, rank)
        shape = tuple(size_dict[l] for l in output)
        part = O.contract_slice_range(inputs, output, size_dict, path, sliced, b, e, arrays) if b < e \
            else np.zeros(shape)
        t = torch.from_numpy(np.array(part, dtype=np.float64, order="C")).reshape(-1)
        dist.all_reduce(t)
        # The product's program for this rank's range (built and described on the host).
        rng_flops = torch.zeros(3, dtype=torch.float64)
        if b < e:
            prog = A.SlicedProgram(inputs, output, size_dict, path, sliced, dtype=np.float64, slice_begin=b,
                                   slice_end=e)
            d = prog.describe()
            rng_flops[:] = torch.tensor([d["slice_begin"], d["slice_end"], prog.flops], dtype=torch.float64)
        else:
            rng_flops[:] = torch.tensor([b, e, 0.0], dtype=torch.float64)
        gathered = [torch.zeros(3, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(gathered, rng_flops)
        if rank == 0:
            q.put((t.numpy().reshape(shape), [g.tolist() for g in gathered]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", sorted(CASES))
def test_slice_sharded_allreduce_matches_single_rank(name, world):
    inputs, output, size_dict, path, sliced = CASES[name]
    arrays = random_arrays(inputs, size_dict, np.float64, 7)
    want = O.contract_sliced(inputs, output, size_dict, path, sliced, arrays)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    mp.start_processes(_worker, args=(world, _free_port(), name, q), nprocs=world, join=True, start_method="spawn")
    got, ranges = q.get(timeout=30)
    assert np.max(np.abs(got - want)) < 1e-12
    n = int(np.prod([size_dict[l] for l in sliced]))
    full = A.SlicedProgram(inputs, output, size_dict, path, sliced, dtype=np.float64)
    covered = 0
    for lo, hi, _ in ranges:
        assert int(lo) == covered and hi >= lo
        covered = int(hi)
    assert covered == n
    assert sum(f for _, _, f in ranges) == pytest.approx(full.flops)


def test_slice_range_partition():
    for n in range(0, 40):
        for ranks in range(1, 9):
            covered = 0
            for r in range(ranks):
                b, e = A.slice_range(n, ranks, r)
                assert b == covered and e >= b
                covered = e
            assert covered == n

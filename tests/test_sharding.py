"""LPT sharding of independent networks across ranks, and the one gather that assembles their results.

The assignment is checked for being a partition, deterministic and within the LPT bound of the best split
(brute-forced on small cases).  The rank protocol runs on gloo ranks on CPU (world size 2 and 3), each rank
contracting its share with the oracle: every rank ends with every network's result, in network order, equal to
contracting each network alone.  tests/test_gpu_sharding.py runs the shares as ProgramBatches on the GPU.
"""

import datetime
import itertools
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist

import arctn_b200 as A
from arctn_b200 import networks as N
from arctn_b200.sharding import lpt_shard, run_sharded
from oracle import oracle as O
from tests.helpers import spawn_ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _best_max_load(costs, ranks):
    best = float("inf")
    for assign in itertools.product(range(ranks), repeat=len(costs)):
        loads = [0.0] * ranks
        for c, r in zip(costs, assign):
            loads[r] += c
        best = min(best, max(loads))
    return best


def test_known_assignment():
    # 5 -> r0, 4 -> r1, 3 -> r1 (7), 3 -> r0 (8), 3 -> r1 (10); the best split is 9 (5+4 | 3+3+3)
    assert lpt_shard([5, 4, 3, 3, 3], 2) == [[0, 3], [1, 2, 4]]
    assert lpt_shard([], 3) == [[], [], []]
    assert lpt_shard([1.0], 3) == [[0], [], []]
    assert lpt_shard([2, 2, 2, 2], 4) == [[0], [1], [2], [3]]


def test_partition_determinism_and_lpt_bound():
    rng = np.random.default_rng(5)
    for trial in range(200):
        n, ranks = int(rng.integers(0, 9)), int(rng.integers(1, 4))
        costs = list(rng.integers(0, 20, n).astype(float))
        shares = lpt_shard(costs, ranks)
        assert shares == lpt_shard(costs, ranks)
        assert sorted(i for s in shares for i in s) == list(range(n))
        assert all(s == sorted(s) for s in shares)
        loads = [sum(costs[i] for i in s) for s in shares]
        if n:
            best = _best_max_load(costs, ranks)
            assert max(loads) <= (4 / 3 - 1 / (3 * ranks)) * best + 1e-9


def test_rejects_bad_arguments():
    with pytest.raises(ValueError, match="ranks"):
        lpt_shard([1, 2], 0)
    for bad in ([1, -1], [float("nan")], [float("inf")]):
        with pytest.raises(ValueError, match="finite and non-negative"):
            lpt_shard(bad, 2)
    with pytest.raises(ValueError, match="returned 0 results"):
        run_sharded([1.0, 2.0], lambda idx: [], 0, 1, gather=lambda obj: [obj])


def _batch(count=12):
    nets = N.workload_batch(count, seed=3)
    out = []
    for net, arrays in nets:
        inputs, output, size_dict = net.as_tuple()
        path = A.greedy(inputs, output, size_dict)
        cost = 10 ** A.simulate_path(inputs, output, size_dict, path)["log10_flops"]
        out.append((inputs, output, size_dict, path, arrays, cost))
    return out


def _oracle_one(item):
    inputs, output, size_dict, path, arrays, _ = item
    return np.asarray(O.execute(inputs, output, size_dict, path, O.promote(arrays)))


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        batch = _batch()
        ran = []

        def execute_share(indices):
            ran.extend(indices)
            # each result also carries 64 KB, so every rank's report exceeds a pipe buffer
            return [(_oracle_one(batch[i]), np.full(8192, i, dtype=np.float64)) for i in indices]

        results = run_sharded([b[-1] for b in batch], execute_share, rank, world)
        q.put((rank, ran, results))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_run_their_shares_and_gather_every_result(world):
    batch = _batch()
    want = [_oracle_one(b) for b in batch]
    got = spawn_ranks(_worker, (world, _free_port()), world)
    shares = lpt_shard([b[-1] for b in batch], world)
    for rank, ran, results in got:
        assert ran == shares[rank]  # each rank contracted exactly its LPT share
        assert len(results) == len(batch)
        for i, ((r, pad), w) in enumerate(zip(results, want)):
            assert np.array_equal(r, w)
            assert np.array_equal(pad, np.full(8192, i, dtype=np.float64))

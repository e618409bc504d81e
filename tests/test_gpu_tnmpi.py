"""The slice-sharded plan runner (arctn_b200.tnmpi) with the product's GPU executor.

Each rank runs the product's slice-range program for its contiguous range of a saved version-2 plan and the
FP64 partials are summed by one all-reduce, as the reference's MPI runner does (src/bin/tnmpi.rs:404-496).
One GPU per call: ranks are spawned processes that share cuda:0 and sum over gloo (their kernels never wait on
one another); the single-rank command line runs its all-reduce over NCCL.  Results are checked against the
oracle: 1e-5 relative for complex64, 1e-12 for float64/complex128.
"""

import datetime
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist

import arctn_b200 as A
from arctn_b200 import networks as N
from arctn_b200 import tnmpi as T
from oracle import oracle as O
from tests.helpers import random_arrays, spawn_ranks

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rand3reg_plan(tmp):
    """rand3reg n = 64, bond 2, sliced to at most 2^8 elements per intermediate, complex64 inputs."""
    net, arrays = N.workload_rand3reg(64, 2, 1, np.complex64, seed=0)
    order = {}  # a version-2 network is dense: legs renumbered in first-occurrence order
    for leg in [l for t in net.inputs for l in t] + list(net.output):
        order.setdefault(leg, len(order))
    inputs = [[order[l] for l in t] for t in net.inputs]
    output = [order[l] for l in net.output]
    size_dict = {order[l]: d for l, d in net.size_dict.items()}
    path = A.greedy(inputs, output, size_dict)
    sliced = A.find_slices_to_size(inputs, output, size_dict, path, 2 ** 8)
    plan = A.ExecutionPlan.from_path(inputs, output, size_dict, path, sliced, target_size=2 ** 8, name="rand3reg64")
    data = os.path.join(tmp, "rand3reg64.bin")
    A.save_tensors_bin(data, arrays)
    return plan.save(os.path.join(tmp, "rand3reg64.json")), data, plan, arrays


def _blocks_plan(tmp):
    """Output-leg and internal slices of a small network, float64 / complex128 inputs."""
    inputs, output, size_dict = [[0, 1, 2], [1, 3, 2], [1, 4]], [4, 1, 0, 3], {0: 2, 1: 3, 2: 5, 3: 2, 4: 2}
    path, sliced = [(0, 1), (3, 2)], [2, 0]
    plan = A.ExecutionPlan.from_path(inputs, output, size_dict, path, sliced, name="blocks")
    arrays = random_arrays(inputs, size_dict, np.complex128, 11)
    data = os.path.join(tmp, "blocks.bin")
    A.save_tensors_bin(data, arrays)
    return plan.save(os.path.join(tmp, "blocks.json")), data, plan, arrays


def _worker(rank, world, port, argv, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        stats, total = T.run(T.parse_args(argv), device=torch.device("cuda", 0))
        q.put((rank, stats, total))
    finally:
        dist.destroy_process_group()


def _run_ranks(world, argv):
    return spawn_ranks(_worker, (world, _free_port(), argv), world)


@pytest.mark.parametrize("precision", ["fp32", "tf32x3"])
def test_two_ranks_on_the_gpu_executor_match_the_oracle(tmp_path, precision):
    plan_path, data, plan, arrays = _rand3reg_plan(str(tmp_path))
    want = complex(O.contract_sliced(plan.inputs, plan.output, plan.size_dict, plan.ssa_path, plan.sliced_legs,
                                     O.promote(arrays), threads=8))
    results = _run_ranks(2, ["--load-path", plan_path, "--data", data, "--dtype", "complex64", "--precision",
                             precision, "--backend", "gloo", "--check"])
    for _, stats, total in results:
        got = complex(total)
        assert abs(got - want) <= 1e-5 * abs(want), (got, want)
        assert stats["n_slices"] == int(np.prod([plan.size_dict[l] for l in plan.sliced_legs])) >= 16
        assert stats["ranks"] == 2 and stats["check"].startswith("PASS(")
        assert stats["execution_device_seconds_max"] > 0
        assert stats["target_size"] == 256 and stats["target_log2_size"] == 8.0


@pytest.mark.parametrize("world", [2, 3])
def test_output_blocks_across_ranks_on_the_gpu_executor(tmp_path, world):
    plan_path, data, plan, arrays = _blocks_plan(str(tmp_path))
    want = O.contract_sliced(plan.inputs, plan.output, plan.size_dict, plan.ssa_path, plan.sliced_legs, arrays)
    results = _run_ranks(world, ["--load-path", plan_path, "--data", data, "--dtype", "complex128",
                                 "--backend", "gloo", "--check"])
    for _, stats, total in results:
        assert total.shape == want.shape
        assert np.max(np.abs(total - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))
        assert stats["check"].startswith("PASS(")


def test_command_line_single_rank_over_nccl(tmp_path):
    plan_path, data, plan, arrays = _rand3reg_plan(str(tmp_path))
    env = dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    for key in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(key, None)
    proc = subprocess.run([sys.executable, "-m", "arctn_b200.tnmpi", "--load-path", plan_path, "--data", data,
                           "--dtype", "complex64", "--precision", "tf32x3", "--check"],
                          capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert proc.returncode == 0, proc.stderr[-2000:]
    stats = json.loads(proc.stdout.strip().splitlines()[-1])
    assert stats["ranks"] == 1 and stats["backend"] == "nccl" and stats["check"].startswith("PASS(")
    assert stats["execution_device_seconds_max"] > 0


def test_command_line_under_the_launcher_with_two_ranks(tmp_path):
    plan_path, data, plan, arrays = _blocks_plan(str(tmp_path))
    env = dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    proc = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
                           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
                           "-m", "arctn_b200.tnmpi", "--load-path", plan_path, "--data", data,
                           "--dtype", "complex128", "--backend", "gloo", "--check"],
                          capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert proc.returncode == 0, proc.stderr[-2000:]
    stats = json.loads(proc.stdout.strip().splitlines()[-1])
    assert stats["ranks"] == 2 and stats["check"].startswith("PASS(")
    assert stats["output_shape"] == [2, 3, 2, 2]



def _ranks_sum(inputs, output, size_dict, path, sliced, arrays, ranks, dtype):
    """The product's slice-range programs of ``ranks`` ranks, run in turn and summed in FP64, as the reference's
    in-process rank tests do (src/bin/tnmpi.rs:540-583); ranks whose range is empty contribute nothing."""
    n = int(np.prod([size_dict[l] for l in sliced])) if sliced else 1
    total = None
    for rank in range(ranks):
        b, e = A.slice_range(n, ranks, rank)
        if b == e:
            continue
        prog = A.SlicedProgram(inputs, output, size_dict, path, sliced, dtype=dtype, slice_begin=b, slice_end=e)
        part = np.asarray(prog.execute(arrays, f64_out=True))
        total = part if total is None else total + part
    return total


def test_output_blocks_land_in_place_for_every_axis_position():
    # src/bin/tnmpi.rs:539-583: sliced output legs at the front, middle and back of a three-axis output,
    # alone and with the internal legs 3 and 4, over four ranks.
    inputs, output, size_dict = [[0, 3], [3, 1, 4], [4, 2]], [0, 1, 2], {0: 2, 1: 3, 2: 2, 3: 2, 4: 3}
    path = [(0, 1), (3, 2)]
    arrays = random_arrays(inputs, size_dict, np.float64, 7)
    want = O.execute(inputs, output, size_dict, path, arrays)
    for sliced in ([1], [2, 0], [1, 3], [4, 1, 0, 3], [0, 1, 2]):
        got = _ranks_sum(inputs, output, size_dict, path, sliced, arrays, 4, np.float64)
        assert got.shape == want.shape
        assert np.max(np.abs(got - want)) < 1e-12, sliced


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.complex64, np.complex128])
def test_matrix_slice_products_over_three_ranks_are_exact(dtype):
    # src/bin/tnmpi.rs:607-680: a 2x2 . 2x2 product with internal, output and mixed slices over three ranks
    # (some ranges empty); small integer parts keep every product and sum exact.
    real = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0, 8.0])
    imag = np.array([1.0, -1.0, 2.0, 0.0, 0.0, 1.0, -1.0, 2.0])
    vals = real + 1j * imag if np.dtype(dtype).kind == "c" else real
    a, b = (np.asarray(v, dtype=dtype).reshape(2, 2) for v in (vals[:4], vals[4:]))
    want = a.astype(np.complex128) @ b.astype(np.complex128)
    if np.dtype(dtype).kind == "f":
        assert np.array_equal(want.real, [[19.0, 22.0], [43.0, 50.0]])
    inputs, output, size_dict = [[0, 1], [1, 2]], [0, 2], {0: 2, 1: 2, 2: 2}
    for sliced in ([], [1], [0], [2, 0], [1, 2, 0]):
        got = _ranks_sum(inputs, output, size_dict, [(0, 1)], sliced, [a, b], 3, dtype)
        assert np.array_equal(got, want if np.dtype(dtype).kind == "c" else want.real), (sliced, got)

"""The slice-sharded plan runner (arctn_b200.tnmpi) on CPU: options, and the rank protocol over gloo.

Mirrors the reference's MPI runner tests (src/bin/tnmpi.rs:540-680): ranks take contiguous slice ranges of a
saved version-2 plan, sum their partials with one all-reduce, and agree on failures before each collective.
Here every rank's slice range is contracted by the oracle's contract_slice_range, injected as the executor,
so the runner's host-side protocol (plan broadcast, failure agreement, partition, sum, --check, stats line)
is exercised without a GPU.  The product's GPU executor under the same runner is covered by
tests/test_gpu_tnmpi.py.
"""

import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist

import arctn_b200 as A
from arctn_b200 import tnmpi as T
from oracle import oracle as O
from tests.helpers import random_arrays, spawn_ranks

# Dense networks (legs numbered in first-occurrence order), with their SSA paths and sliced legs.
CASES = {
    "internal": ([[0, 1], [1, 2], [2, 3]], [0, 3], {0: 2, 1: 3, 2: 5, 3: 2}, [(0, 1), (3, 2)], [1, 2]),
    "output_and_internal": ([[0, 1, 2], [1, 3, 2], [1, 4]], [4, 1, 0, 3], {0: 2, 1: 3, 2: 5, 3: 2, 4: 2},
                            [(0, 1), (3, 2)], [2, 0]),
    "two_slices": ([[0], [0]], [], {0: 2}, [(0, 1)], [0]),
}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _save_case(tmp, name, dtype=np.float64):
    inputs, output, size_dict, path, sliced = CASES[name]
    plan = A.ExecutionPlan.from_path(inputs, output, size_dict, path, sliced, name=name)
    plan_path = plan.save(os.path.join(tmp, f"{name}.json"))
    arrays = random_arrays(inputs, size_dict, dtype, 7)
    data_path = os.path.join(tmp, f"{name}.bin")
    A.save_tensors_bin(data_path, arrays)
    return plan_path, data_path, arrays


def oracle_executor(plan, arrays, args, begin, end, device):
    """Test executor: the oracle's slice-range contraction, as a wide-dtype tensor."""

    def call():
        part = O.contract_slice_range(plan.inputs, plan.output, plan.size_dict, plan.ssa_path, plan.sliced_legs,
                                      begin, end, O.promote(arrays))
        return torch.from_numpy(np.array(part, order="C"))

    return call


def failing_on_rank1(plan, arrays, args, begin, end, device):
    if dist.get_rank() == 1:
        raise RuntimeError("rank 1 cannot build its program")
    return oracle_executor(plan, arrays, args, begin, end, device)


def _worker(rank, world, port, argv, executor_name, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        args = T.parse_args(argv)
        executor = {"oracle": oracle_executor, "failing": failing_on_rank1}[executor_name]
        try:
            stats, total = T.run(args, device=torch.device("cpu"), executor=executor)
            q.put((rank, "ok", stats, total))
        except T.RankFailure as exc:
            q.put((rank, "failed", str(exc), None))
    finally:
        dist.destroy_process_group()


def _run_ranks(world, argv, executor="oracle"):
    return spawn_ranks(_worker, (world, _free_port(), argv, executor), world)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", sorted(CASES))
def test_ranks_sum_their_slice_ranges_to_the_single_process_result(tmp_path, name, world):
    plan_path, data_path, arrays = _save_case(str(tmp_path), name)
    inputs, output, size_dict, path, sliced = CASES[name]
    want = O.contract_sliced(inputs, output, size_dict, path, sliced, arrays)
    results = _run_ranks(world, ["--load-path", plan_path, "--data", data_path, "--check", "--backend", "gloo"])
    n_slices = int(np.prod([size_dict[l] for l in sliced]))
    for rank, status, stats, total in results:
        assert status == "ok"
        assert np.max(np.abs(total - want)) < 1e-12
        assert stats["ranks"] == world and stats["n_slices"] == n_slices
        assert stats["network"] == name and stats["mode"] == "saved-path" and stats["dtype"] == "f64"
        assert stats["sliced_indices"] == list(sliced)
        assert stats["output_shape"] == [size_dict[l] for l in output]
        assert stats["check"].startswith("PASS(")
        assert stats["execution_device_seconds_max"] is None  # no CUDA events on CPU ranks
        assert stats["execution_wall_seconds_max"] >= 0 and stats["load_wall_seconds_max"] >= 0
    # The stats line is the same on every rank (maxima over ranks, rank 0's --check).
    assert all(r[2] == results[0][2] for r in results)


def test_a_failure_on_one_rank_stops_every_rank(tmp_path):
    plan_path, data_path, _ = _save_case(str(tmp_path), "internal")
    results = _run_ranks(2, ["--load-path", plan_path, "--data", data_path, "--backend", "gloo"], "failing")
    assert [r[1] for r in results] == ["failed", "failed"]
    assert "rank 1 cannot build" in results[1][2]


def test_a_plan_that_fails_to_load_on_rank0_stops_every_rank(tmp_path):
    bad = tmp_path / "bad.json"
    bad.write_text('{"schema": "arctn-execution-plan", "schema_version": 1}')
    results = _run_ranks(2, ["--load-path", str(bad), "--backend", "gloo"])
    assert [r[1] for r in results] == ["failed", "failed"]
    assert all("version" in r[2] for r in results)


def test_a_data_file_of_the_wrong_size_stops_every_rank(tmp_path):
    plan_path, data_path, _ = _save_case(str(tmp_path), "internal")
    with open(data_path, "ab") as f:
        f.write(b"\0" * 8)
    results = _run_ranks(2, ["--load-path", plan_path, "--data", data_path, "--backend", "gloo"])
    assert [r[1] for r in results] == ["failed", "failed"]
    assert "bytes" in results[0][2]


def test_example_inputs_are_seeded_and_uniform(tmp_path):
    plan = A.ExecutionPlan.load(_save_case(str(tmp_path), "internal")[0])
    a = T.example_inputs(plan, "complex64", 1)
    b = T.example_inputs(plan, "complex64", 1)
    c = T.example_inputs(plan, "complex64", 2)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert not all(np.array_equal(x, y) for x, y in zip(a, c))
    for x, legs in zip(a, plan.inputs):
        assert x.dtype == np.complex64 and x.shape == tuple(plan.size_dict[l] for l in legs)
        assert np.all(np.abs(x.real) <= 1) and np.all(np.abs(x.imag) <= 1)


def test_options():
    assert T.parse_args(["--help"]) is None
    args = T.parse_args(["--load-path", "p.json", "--dtype", "complex64", "--precision", "tf32x3", "--seed", "9",
                         "--check", "--backend", "gloo", "--data", "t.bin", "--broadcast-inputs"])
    assert (args.load_path, args.dtype, args.precision, args.seed, args.check, args.backend, args.data_file,
            args.broadcast_inputs) == ("p.json", "complex64", "tf32x3", 9, True, "gloo", "t.bin", True)
    defaults = T.parse_args(["--load-path", "p.json"])
    assert (defaults.dtype, defaults.precision, defaults.seed, defaults.check, defaults.backend,
            defaults.broadcast_inputs) == ("f64", "fp32", 1, False, "nccl", False)
    for argv, msg in [([], "--load-path"), (["--load-path"], "requires a value"),
                      (["--load-path", "--check"], "requires a value"),
                      (["--load-path", "p", "--dtype", "c64"], "--dtype must be"),
                      (["--load-path", "p", "--seed", "-1"], "unsigned 64-bit"),
                      (["--load-path", "p", "--precision", "tf32"], "--precision must be"),
                      (["--load-path", "p", "--net", "n.json"], "version 2"),
                      (["--load-path", "p", "--bogus"], "unknown option")]:
        with pytest.raises(T.UsageError, match=msg):
            T.parse_args(argv)


def test_main_exit_codes(capsys):
    assert T.main(["--help"]) == 0
    assert "Usage" in capsys.readouterr().out
    assert T.main(["--dtype", "f64"]) == 2
    assert "--load-path" in capsys.readouterr().err


def test_command_line_failure_exits_3_on_every_rank(tmp_path):
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    plan_path, data_path, _ = _save_case(str(tmp_path), "output_and_internal")
    with open(data_path, "ab") as f:
        f.write(b"\0" * 16)
    env = dict(os.environ, PYTHONPATH=root + os.pathsep + os.environ.get("PYTHONPATH", ""))
    proc = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
                           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
                           "-m", "arctn_b200.tnmpi", "--load-path", plan_path, "--data", data_path,
                           "--backend", "gloo"],
                          capture_output=True, text=True, timeout=300, env=env, cwd=root)
    # Both ranks fail at the same step; the launcher may stop the second before it reports, so only the first
    # rank's exit code 3 and message are certain (every rank raising is shown by the in-process tests above).
    assert proc.returncode != 0
    assert "exitcode  : 3" in proc.stderr
    assert "tnmpi rank" in proc.stderr and "bytes" in proc.stderr


@pytest.mark.parametrize("dtype", ["f32", "f64", "complex64", "complex128"])
def test_check_passes_and_catches_a_wrong_total(tmp_path, dtype):
    # src/bin/tnmpi.rs:645-671: the single-process comparison passes on the right total and fails once one
    # element moves by one unit (the imaginary unit for complex dtypes).
    plan_path, data_path, _ = _save_case(str(tmp_path), "output_and_internal", T.DTYPES[dtype])
    plan = A.ExecutionPlan.load(plan_path)
    arrays = A.load_tensors_bin(data_path, plan.inputs, plan.size_dict, T.DTYPES[dtype])
    args = T.parse_args(["--load-path", plan_path, "--dtype", dtype, "--check"])
    n = int(np.prod([plan.size_dict[l] for l in plan.sliced_legs]))
    total = oracle_executor(plan, arrays, args, 0, n, None)().numpy()
    assert T._check_result(plan, arrays, args, total, n, oracle_executor, None).startswith("PASS(")
    bad = total.copy()
    bad.reshape(-1)[0] += 1j if np.iscomplexobj(bad) else 1.0
    with pytest.raises(RuntimeError, match="single-process comparison failed"):
        T._check_result(plan, arrays, args, bad, n, oracle_executor, None)


def test_check_is_skipped_above_the_size_limits():
    # src/bin/tnmpi.rs:386-388
    big = np.zeros(T.CHECK_MAX_NUMEL + 1)
    assert T._check_result(None, None, None, big, 1, None, None).startswith("skipped")
    assert T._check_result(None, None, None, np.zeros(1), T.CHECK_MAX_SLICES + 1, None, None).startswith("skipped")


def _worker_per_rank(rank, world, port, argvs, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        try:
            stats, total = T.run(T.parse_args(argvs[rank]), device=torch.device("cpu"), executor=oracle_executor)
            q.put((rank, "ok", stats, total))
        except T.RankFailure as exc:
            q.put((rank, "failed", str(exc), None))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("dtype", ["f32", "complex128"])
def test_broadcast_inputs_need_the_data_file_on_rank0_only(tmp_path, world, dtype):
    plan_path, data_path, arrays = _save_case(str(tmp_path), "output_and_internal", T.DTYPES[dtype])
    inputs, output, size_dict, path, sliced = CASES["output_and_internal"]
    want = O.contract_sliced(inputs, output, size_dict, path, sliced, O.promote(arrays))
    common = ["--load-path", plan_path, "--dtype", dtype, "--backend", "gloo", "--broadcast-inputs", "--check"]
    argvs = [common + ["--data", data_path if r == 0 else str(tmp_path / "absent.bin")] for r in range(world)]
    results = spawn_ranks(_worker_per_rank, (world, _free_port(), argvs), world)
    for rank, status, stats, total in results:
        assert status == "ok", stats
        assert np.max(np.abs(total - want)) < 1e-12
        assert stats["check"].startswith("PASS(")


def test_broadcast_inputs_stop_every_rank_when_rank0_cannot_read(tmp_path):
    plan_path, data_path, _ = _save_case(str(tmp_path), "internal")
    argv = ["--load-path", plan_path, "--data", str(tmp_path / "absent.bin"), "--backend", "gloo",
            "--broadcast-inputs"]
    results = spawn_ranks(_worker_per_rank, (2, _free_port(), [argv, argv]), 2)
    assert [r[1] for r in results] == ["failed", "failed"]
    assert "absent.bin" in results[0][2] and results[1][2] == "another rank failed"

"""Shared helpers for the test suite (network fixtures and comparisons)."""

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def known_answers():
    with open(os.path.join(HERE, "golden", "known_answers.json")) as f:
        return json.load(f)


def sd(d):
    return {int(k): int(v) for k, v in d.items()}


def case_arrays(case):
    dt = np.dtype(case["dtype"])
    out = []
    for a, shape in zip(case["arrays"], case["shapes"]):
        arr = np.asarray(a, dtype=np.float64)
        if np.issubdtype(dt, np.complexfloating):
            arr = arr[..., 0] + 1j * arr[..., 1]
        out.append(np.array(arr.reshape(shape), dtype=dt, order="C"))
    return out


def case_expected(case):
    exp = case["expected"]
    if exp is None:
        return None
    arr = np.asarray(exp, dtype=np.float64)
    if case["dtype"].startswith("complex"):
        arr = arr[..., 0] + 1j * arr[..., 1]
    return arr


def random_arrays(inputs, size_dict, dtype, seed, scale=1.0):
    """Reference-style test data: uniform(-1, 1) entries (src/tensor.rs:117-119, 310-312)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dt = np.dtype(dtype)
    out = []
    for t in inputs:
        shape = tuple(size_dict[l] for l in t)
        if np.issubdtype(dt, np.complexfloating):
            v = rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)
        else:
            v = rng.uniform(-1, 1, shape)
        out.append(np.array(np.asarray(v) * scale, dtype=dt, order="C"))
    return out


def rel_err(got, want):
    got = np.asarray(got, dtype=np.complex128)
    want = np.asarray(want, dtype=np.complex128)
    scale = max(1.0, float(np.max(np.abs(want)))) if want.size else 1.0
    return float(np.max(np.abs(got - want))) / scale if want.size else 0.0


def mixed_network():
    """A diagonal, a trace, a dangling leg, a batch leg and a hyperedge (tests/compiled_pair_steps.rs:67-93)."""
    inputs = [[0, 0, 1], [0, 2, 3, 3], [1, 2, 4, 5], [4, 6, 9], [6, 8, 9], [9, 10]]
    output = [8, 6, 10]
    size_dict = {0: 3, 1: 2, 2: 3, 3: 2, 4: 2, 5: 3, 6: 2, 8: 3, 9: 2, 10: 3}
    return inputs, output, size_dict


SMALL_NETWORKS = {
    "matmul": ([[0, 1], [1, 2]], [0, 2], {0: 3, 1: 4, 2: 5}),
    "chain3": ([[0, 1], [1, 2], [2, 3]], [0, 3], {0: 2, 1: 3, 2: 5, 3: 7}),
    "hyper": ([[0, 1], [0, 2], [0]], [], {0: 3, 1: 2, 2: 4}),
    "trace": ([[0, 0, 1], [1]], [], {0: 3, 1: 4}),
    "diag_shared": ([[0, 0, 1], [0, 2]], [1, 2], {0: 3, 1: 2, 2: 4}),
    "diag_output": ([[0, 0, 1], [1, 2]], [0, 2], {0: 4, 1: 3, 2: 5}),
    "trace_and_diag": ([[0, 0, 1, 1], [1, 2]], [2], {0: 3, 1: 2, 2: 4}),
    "single": ([[0, 1]], [0], {0: 3, 1: 5}),
    "single_perm": ([[0, 1, 2]], [2, 0], {0: 2, 1: 3, 2: 4}),
    "dangling": ([[0, 1], [1, 2]], [2], {0: 7, 1: 3, 2: 5}),
    "scalar_inputs": ([[], []], [], {}),
    "scalar_and_vec": ([[], [0]], [0], {0: 5}),
    "mixed": mixed_network(),
    "tiny6": ([[0, 1], [1, 2], [2, 3], [3, 4], [4, 5], [5, 0, 6]], [6], {0: 4, 1: 5, 2: 4, 3: 6, 4: 4, 5: 5, 6: 3}),
}


def spawn_ranks(fn, args, world, timeout=300):
    """Run fn(rank, *args, q) in ``world`` spawned processes and return the ``world`` items they put on q,
    sorted by their first field (the rank).  The queue is drained while the processes run: a child that has
    put more than a pipe buffer holds cannot exit until its data is read, so joining first would wait forever.
    A child that raises fails the call at once; a missing item fails it after ``timeout`` seconds."""
    import queue
    import time

    import torch.multiprocessing as mp

    q = mp.get_context("spawn").Queue()
    pc = mp.start_processes(fn, args=tuple(args) + (q,), nprocs=world, join=False, start_method="spawn")
    got, deadline = [], time.monotonic() + timeout
    while len(got) < world:
        try:
            got.append(q.get(timeout=1.0))
        except queue.Empty:
            pc.join(timeout=0)  # raises if a child failed
            if time.monotonic() > deadline:
                raise TimeoutError(f"{len(got)} of {world} ranks reported within {timeout} s")
    while not pc.join(timeout=1.0):
        if time.monotonic() > deadline:
            raise TimeoutError(f"ranks did not exit within {timeout} s")
    return sorted(got, key=lambda item: item[0])

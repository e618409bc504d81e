"""GPU: the captured graph runs independent steps concurrently (8 lanes, edges from memory footprints).

Every kernel computes the same values whatever runs beside it, so a graph replay must give the same bits as
the plain sequential launch of the same program, on its first capture and on later replays.
"""

import numpy as np
import pytest
import torch

import arctn_b200 as A
from arctn_b200 import networks as N

pytestmark = pytest.mark.gpu


def _cases():
    yield pytest.param("grid6_c128", *N.workload_grid6(np.complex128, seed=0), (), "fp32", id="grid6_c128")
    net, arrays = N.brickwork_circuit(30, 14, seed=0)
    yield pytest.param("brickwork", net, [a.astype(np.complex64) for a in arrays], (), "tf32x3", id="brickwork_tf32x3")
    net, arrays = N.workload_rand3reg(104, 2, 1, np.complex64, seed=0)
    sliced = A.find_slices_to_size(*net.as_tuple(), A.greedy(*net.as_tuple()), 2 ** 14)
    yield pytest.param("rand3reg104", net, arrays, sliced, "tf32x3", id="rand3reg104_sliced_tf32x3")
    net = N.grid_2d(5, 5, 6)
    yield pytest.param("grid5", net, N.gaussian_tensors(net, np.complex64, 3, scale_base=6), (), "fp32",
                       id="grid5_bond6_fp32")


@pytest.mark.parametrize("name,net,arrays,sliced,precision", list(_cases()))
def test_graph_replay_equals_sequential_launch(name, net, arrays, sliced, precision):
    path = A.greedy(*net.as_tuple())
    kw = dict(dtype=arrays[0].dtype, precision=precision, max_slices_per_group=4 if sliced else 0)
    seq = A.SlicedProgram(*net.as_tuple(), path, sliced, use_graph=False, **kw)
    dag = A.SlicedProgram(*net.as_tuple(), path, sliced, use_graph=True, **kw)
    st = torch.cuda.Stream()  # graphs are captured from a non-default stream
    with torch.cuda.stream(st):  # allocations, launches and the copies back all in stream order
        x = [torch.from_numpy(a).cuda() for a in arrays]
        want = seq.execute(x, stream=st).cpu()
        ws = torch.empty(max(dag.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
        for _ in range(3):  # first capture, then replays of the instantiated graph
            got = dag.execute(x, workspace=ws, stream=st).cpu()
            assert torch.equal(got, want), name
        assert dag.device_status(ws, st) == 0


def test_numpy_calls_reuse_buffers_and_see_new_inputs():
    # Repeated NumPy calls on one stream reuse the staged-input buffer, workspace and output (so the graph
    # replays); each call must still see its own inputs.  Doubling one input doubles the result exactly
    # (a power-of-two scale is exact through every product and the TF32 split).
    net, arrays = N.workload_rand3reg(64, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 8)
    prog = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3")
    first = prog.execute(arrays)
    again = prog.execute(arrays)
    doubled = [a * 2 if i == 3 else a for i, a in enumerate(arrays)]
    twice = prog.execute(doubled)
    assert np.array_equal(first, again)
    assert np.array_equal(twice, first * 2)
    st = torch.cuda.Stream()  # an explicit stream that is not the current one: copies follow it
    other = prog.execute(doubled, stream=st)
    assert np.array_equal(other, twice)


def test_profile_reports_one_entry_per_launch_unit():
    # A grouped launch of thin steps is one profiled launch; every other kernel one entry each.
    net, arrays = N.brickwork_circuit(30, 14, seed=0)
    arrays = [a.astype(np.complex64) for a in arrays]
    prog = A.SlicedProgram(*net.as_tuple(), A.greedy(*net.as_tuple()), (), dtype=np.complex64, precision="tf32x3")
    d = prog.describe()
    first_of_unit = {}
    for o in d["ops"]:
        first_of_unit.setdefault(o["unit"], o["kind"])
    want = sum(k != "memset" for k in first_of_unit.values())
    x = [torch.from_numpy(a).cuda() for a in arrays]
    ms, kinds, work = prog.profile(x)
    assert len(kinds) == len(ms) == len(work) == want < sum(o["kind"] != "memset" for o in d["ops"])
    assert all(t > 0 for t in ms)
    gemm = {1, 2, 3, 9, 10, 14}
    assert sum(w for k, w in zip(kinds, work) if k in gemm) == pytest.approx(prog.flops, rel=1e-12)

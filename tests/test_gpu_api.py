"""GPU tests of the high-level Python callers, mirroring the reference's public interface.

``arctn_contract(..., backend="b200")`` (pybind/python/arctn/__init__.py:903-1072) and
``ArcTNCompiledContraction.compile(..., backend="b200").execute`` (``__init__.py:776-807``) against the
oracle; arbitrary hashable leg labels are renumbered as the reference's ``_to_int_labels`` does.
"""

import numpy as np
import pytest
import torch

import arctn_b200 as A
from arctn_b200 import networks as N
from oracle import oracle as O
from tests.helpers import random_arrays, rel_err

pytestmark = pytest.mark.gpu


def labelled(net):
    """The network with string leg labels (the reference accepts any hashable label), and the integer form
    the binding numbers them into: ids in order of first appearance over the inputs, then the output."""
    name = {l: f"leg{l}" for l in net.size_dict}
    inputs = [[name[l] for l in t] for t in net.inputs]
    output = [name[l] for l in net.output]
    size = {name[l]: d for l, d in net.size_dict.items()}
    ids = {}
    for lab in [l for t in inputs for l in t] + output:
        ids.setdefault(lab, len(ids))
    internal = ([[ids[l] for l in t] for t in inputs], [ids[l] for l in output], {ids[l]: d for l, d in size.items()})
    return inputs, output, size, internal


@pytest.mark.parametrize("dtype,tol", [(np.complex128, 1e-12), (np.complex64, 1e-5), (np.float64, 1e-12)],
                         ids=["c128", "c64", "f64"])
def test_arctn_contract_plans_slices_and_matches_oracle(dtype, tol):
    net, arrays = N.workload_rand3reg(64, 2, 1, dtype, seed=1)
    inputs, output, size, internal = labelled(net)
    got, info = A.arctn_contract(inputs, output, size, [torch.from_numpy(a).cuda() for a in arrays],
                                 target_size=2 ** 8, backend="b200", return_info=True)
    assert info["execution_backend"] == "b200"
    path = O.greedy(*internal)
    assert [tuple(p) for p in info["path"]] == [tuple(p) for p in path]
    sliced = O.find_slices_to_size(*internal, path, 2 ** 8)
    assert list(info["sliced_legs"]) == list(sliced) and len(sliced) >= 1
    want = O.contract_sliced(*internal, path, sliced, O.promote(arrays), threads=4)
    assert abs(complex(got.item()) - complex(want)) <= tol * abs(complex(want))


def test_arctn_contract_numpy_inputs_and_rejections():
    net, arrays = N.workload_rand3reg(40, 2, 3, np.complex128, seed=2)
    inputs, output, size, internal = labelled(net)
    got = A.arctn_contract(inputs, output, size, arrays, backend="b200")
    path = O.greedy(*internal)
    want = complex(O.contract_sliced(*internal, path, [], arrays))
    assert abs(complex(np.asarray(got)) - want) <= 1e-12 * abs(want)
    with pytest.raises(ValueError):
        A.arctn_contract(inputs, output, size, arrays, backend="auto")
    with pytest.raises(ValueError):
        A.arctn_contract(inputs, output, size, arrays, backend="cpu")
    with pytest.raises(ValueError):
        A.arctn_contract(inputs, output, size, arrays, backend="b200", target_size=0)


@pytest.mark.parametrize("precision", ["fp32", "tf32x3"])
def test_compiled_contraction_facade_matches_oracle(precision):
    # A contraction with dense complex64 steps (the tensor-core path under tf32x3).
    inputs = [["a", "b", "c"], ["c", "d"], ["d", "e"], ["b", "e", "f"]]
    output = ["a", "f"]
    size = {"a": 192, "b": 8, "c": 160, "d": 144, "e": 8, "f": 176}
    ids = {l: i for i, l in enumerate(size)}
    ii = [[ids[l] for l in t] for t in inputs]
    oi = [ids[l] for l in output]
    si = {ids[l]: d for l, d in size.items()}
    arrays = random_arrays(ii, si, np.complex64, 8, scale=0.5)
    path = O.greedy(ii, oi, si)
    cc = A.ArcTNCompiledContraction.compile(inputs, output, size, ssa_path=path, backend="b200")
    assert cc.backend == "b200" and cc.stats()["n_steps"] == len(path)
    got = cc.execute([torch.from_numpy(a).cuda() for a in arrays], precision=precision)
    want = O.contract_sliced(ii, oi, si, path, [], O.promote(arrays))
    assert rel_err(got.cpu().numpy(), want) <= 1e-5
    assert cc.last_execute_wall_s is not None
    with pytest.raises(ValueError):
        A.ArcTNCompiledContraction.compile(inputs, output, size, ssa_path=path, backend="auto")


def test_arctn_contract_with_output_slicing_matches_oracle():
    # allow_output_slicing (pybind/python/arctn/__init__.py:903-1072): the slice search may pick output legs, and
    # the output is assembled from their blocks.
    net = N.random_connected(7, 2, [2, 3, 4], 2, 7301)
    arrays = random_arrays(net.inputs, net.size_dict, np.complex128, 5)
    inputs, output, size, internal = labelled(net)
    got, info = A.arctn_contract(inputs, output, size, arrays, target_size=4, allow_output_slicing=True,
                                 backend="b200", return_info=True)
    path = O.greedy(*internal)
    sliced = O.find_slices_to_size(*internal, path, 4, allow_output_slicing=True)
    assert list(info["sliced_legs"]) == list(sliced)
    assert any(l in internal[1] for l in sliced)  # at least one output leg is sliced
    want = O.execute(*internal, path, arrays)
    assert np.asarray(got).shape == want.shape
    assert np.max(np.abs(np.asarray(got) - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))

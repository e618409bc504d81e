"""Error propagation from the C ABI to Python, with failures injected on the host (no GPU needed).

``arctn_b200_debug_inject_failure`` makes the countdown-th next call of a site fail at its entry, before any
CUDA work, as a failed CUDA allocation would: the status is ARCTN_B200_ERR_CUDA, the message is readable through
``arctn_b200_last_error`` and Python raises ``ArcTNB200Error`` (a ``ValueError``, the reference's error type,
pybind/src/lib.rs:379,688) carrying that code.  The reference reports every failure as a ``Result`` error and
has no fault injection; these hooks stand in for the failures a GPU run could meet, without making any on the
GPU.  tests/test_gpu_failure.py checks that a program keeps working after an injected failure.
"""

import numpy as np
import pytest

import arctn_b200 as A
from arctn_b200 import _capi as C

NET = ([[0, 1], [1, 2]], [0, 2], {0: 2, 1: 3, 2: 2}, [(0, 1)])


@pytest.fixture(autouse=True)
def disarmed():
    yield
    for site in (0, 1):
        assert C.lib().arctn_b200_debug_inject_failure(site, 0) == 0


def program():
    inputs, output, size_dict, path = NET
    return A.SlicedProgram(inputs, output, size_dict, path, (), dtype=np.float64)


def test_an_injected_creation_failure_reaches_python_once():
    assert C.lib().arctn_b200_debug_inject_failure(1, 1) == 0
    with pytest.raises(ValueError, match="injected") as info:
        program()
    assert isinstance(info.value, A.ArcTNB200Error) and info.value.code == C.ERR_CUDA
    assert "cudaErrorMemoryAllocation" in str(info.value)
    assert program().describe()["ops"]  # the hook fired once; creation works again


def test_the_countdown_picks_the_call_that_fails():
    assert C.lib().arctn_b200_debug_inject_failure(1, 3) == 0
    program()
    program()
    with pytest.raises(A.ArcTNB200Error, match="injected"):
        program()
    program()


def test_batch_creation_failure():
    progs = [program(), program()]
    assert C.lib().arctn_b200_debug_inject_failure(1, 1) == 0
    with pytest.raises(A.ArcTNB200Error, match="injected"):
        A.ProgramBatch(progs)
    assert A.ProgramBatch(progs).describe()["programs"] == 2


def test_an_injected_execute_failure_comes_before_any_other_check():
    # The armed call fails at its entry, before the argument checks and before any CUDA work, so it can be
    # exercised with null arguments here; the next call reaches the checks again.
    p = program()
    L = C.lib()
    assert L.arctn_b200_debug_inject_failure(0, 1) == 0
    rc = L.arctn_b200_program_execute(p._h, None, None, None, 0, None)
    assert rc == C.ERR_CUDA and b"injected" in L.arctn_b200_last_error()
    rc = L.arctn_b200_program_execute(p._h, None, None, None, 0, None)
    assert rc == C.ERR_INVALID and b"null argument" in L.arctn_b200_last_error()
    for fn, args in ((L.arctn_b200_program_execute_f64out, (p._h, None, None, None, 0, None)),
                     (L.arctn_b200_program_gradient, (p._h, 0, None, None, None, None, None, 0, None))):
        assert L.arctn_b200_debug_inject_failure(0, 1) == 0
        assert fn(*args) == C.ERR_CUDA


def test_the_hook_checks_its_arguments():
    L = C.lib()
    assert L.arctn_b200_debug_inject_failure(2, 1) == C.ERR_INVALID
    assert b"site" in L.arctn_b200_last_error()
    assert L.arctn_b200_debug_inject_failure(0, -1) == C.ERR_INVALID
    assert L.arctn_b200_debug_inject_failure(0, 0) == 0

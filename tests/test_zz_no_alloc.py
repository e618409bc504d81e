"""The allocation-free batched complex GEMM entry point (arctn_b200_cgemm_tf32x3_noalloc).

This entry point exists for callers that cannot allocate device memory (a
framework that has reserved the whole memory pool, code inside a region where
an allocation would synchronise the device or break a stream capture).  Its
scratch lives in a fixed 64 MiB __device__ array.  The test checks it against
the existing stage entry point (arctn_b200_plan_step_execute on the same
pairwise step, split-TF32 tensor-core path) on two calls in a row, within the
1e-5 relative tolerance the GPU tests use, and checks that an oversized
problem is rejected.  The file name sorts last so a run that stops at the
first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

import arctn_b200 as A
from arctn_b200 import _capi as C
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


def _operands(bt, m, k, n, seed):
    import torch

    rng = np.random.default_rng(seed)
    a = (rng.uniform(-1, 1, (bt, m, k)) + 1j * rng.uniform(-1, 1, (bt, m, k))).astype(np.complex64)
    b = (rng.uniform(-1, 1, (bt, k, n)) + 1j * rng.uniform(-1, 1, (bt, k, n))).astype(np.complex64)
    return a, b, torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()


def test_noalloc_cgemm_matches_existing_entry_point_twice():
    import torch

    bt, m, k, n = 3, 200, 96, 136
    a, b, ta, tb = _operands(bt, m, k, n, 17)
    # Existing entry point: the same product as one pairwise step [b,i,l] . [b,l,j] -> [b,i,j].
    cc = A.CompiledContraction.compile([[0, 1, 2], [0, 2, 3]], [0, 1, 3], {0: bt, 1: m, 2: k, 3: n},
                                       ssa_path=[(0, 1)])
    assert cc.pair_steps()[0].gemm_dims() == (bt, m, k, n)
    want = cc.pair_steps()[0].execute(ta, tb, precision="tf32x3")
    exact = np.einsum("bik,bkj->bij", a.astype(np.complex128), b.astype(np.complex128))
    fn = C.lib().arctn_b200_cgemm_tf32x3_noalloc
    stream = torch.cuda.current_stream()
    for _ in range(2):
        out = torch.full((bt, m, n), float("nan"), dtype=torch.complex64, device="cuda")
        rc = fn(ta.data_ptr(), tb.data_ptr(), out.data_ptr(), bt, m, k, n, stream.cuda_stream)
        stream.synchronize()
        C.check(rc, "no-alloc GEMM")
        got = out.cpu().numpy()
        assert _status(stream) == 0
        assert np.all(np.isfinite(got))
        assert rel_err(got, want.cpu().numpy()) <= 1e-5
        assert rel_err(got, exact) <= 1e-5


def _status(stream):
    code = ctypes.c_int(-1)
    C.check(C.lib().arctn_b200_cgemm_noalloc_status(stream.cuda_stream, ctypes.byref(code)), "no-alloc status")
    return code.value


# Ragged shapes: K not a multiple of the 16-wide K tile (zero padding of the packs), m and n below one
# 32-row pack tile, n not a multiple of 32 on the strided B pack.
SMALL = [(1, 5, 7, 3), (2, 130, 17, 33), (4, 64, 1, 129)]


@pytest.mark.parametrize("shape", SMALL, ids=[str(s) for s in SMALL])
def test_noalloc_cgemm_ragged_shapes(shape):
    import torch

    bt, m, k, n = shape
    a, b, ta, tb = _operands(bt, m, k, n, 29 + m)
    exact = np.einsum("bik,bkj->bij", a.astype(np.complex128), b.astype(np.complex128))
    fn = C.lib().arctn_b200_cgemm_tf32x3_noalloc
    stream = torch.cuda.current_stream()
    for _ in range(2):
        out = torch.full((bt, m, n), float("nan"), dtype=torch.complex64, device="cuda")
        C.check(fn(ta.data_ptr(), tb.data_ptr(), out.data_ptr(), bt, m, k, n, stream.cuda_stream), "no-alloc GEMM")
        assert _status(stream) == 0
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_err(got, exact) <= 1e-5


def test_noalloc_cgemm_rejects_problems_beyond_its_scratch():
    import torch

    fn = C.lib().arctn_b200_cgemm_tf32x3_noalloc
    x = torch.zeros(1, dtype=torch.complex64, device="cuda")
    rc = fn(x.data_ptr(), x.data_ptr(), x.data_ptr(), 1, 1 << 16, 1024, 128, torch.cuda.current_stream().cuda_stream)
    assert rc == C.ERR_UNSUPPORTED
    assert b"fixed maximum" in C.lib().arctn_b200_last_error()

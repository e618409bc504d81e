"""GPU parity of the adjoint sweep (arctn_b200_program_gradient / arctn_b200.autograd).

Gradients follow PyTorch's complex convention (grad = dL/d conj(T)).  They are checked
against (1) the oracle's step-by-step torch replay of the same plan under torch.autograd
(oracle/torch_replay.py), within 1e-10 relative for f64/c128 and 1e-5 for c64, and
(2) central finite differences in FP64 along random complex directions V:
  (f(T + eps V) - f(T - eps V)) / (2 eps)  ~  sum_i <conj(g_i), V_i>,   eps = 1e-3.
"""

import numpy as np
import pytest
import torch

import arctn_b200 as A
from arctn_b200 import networks as N
from arctn_b200.autograd import Contraction
from oracle import oracle as O
from oracle.torch_replay import replay
from tests.helpers import SMALL_NETWORKS, random_arrays

pytestmark = pytest.mark.gpu


def reference_grads(inputs, output, size_dict, path, arrays, grad_out):
    ts = [torch.from_numpy(np.asarray(a).astype(np.complex128 if np.iscomplexobj(a) else np.float64)).requires_grad_()
          for a in arrays]
    out = replay(inputs, output, size_dict, path, ts)
    g = torch.from_numpy(np.asarray(grad_out).astype(out.detach().numpy().dtype))
    out.backward(g)
    return out.detach().numpy(), [t.grad.numpy() for t in ts]


def max_rel(a, b):
    a, b = np.asarray(a, dtype=np.complex128), np.asarray(b, dtype=np.complex128)
    return float(np.max(np.abs(a - b))) / max(1.0, float(np.max(np.abs(b)))) if b.size else 0.0


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-10), (np.complex128, 1e-10), (np.complex64, 1e-5)],
                         ids=["f64", "c128", "c64"])
@pytest.mark.parametrize("name", sorted(SMALL_NETWORKS))
def test_gradients_match_torch_replay(name, dtype, tol):
    inputs, output, size_dict = SMALL_NETWORKS[name]
    path = A.greedy(inputs, output, size_dict)
    arrays = random_arrays(inputs, size_dict, dtype, 13)
    shape = tuple(size_dict[l] for l in output)
    grad_out = random_arrays([output], size_dict, dtype, 14)[0].reshape(shape)
    want_out, want = reference_grads(inputs, output, size_dict, path, arrays, grad_out)
    prog = A.SlicedProgram(inputs, output, size_dict, path, (), dtype=dtype, gradient=True, use_graph=False)
    out, grads = prog.gradient(arrays, grad_out)
    assert max_rel(out, want_out) <= tol
    for g, w in zip(grads, want):
        assert g.shape == w.shape
        assert max_rel(g, w) <= tol, name


def test_forward_then_reverse_parts_match_single_call():
    inputs, output, size_dict = SMALL_NETWORKS["mixed"]
    path = A.greedy(inputs, output, size_dict)
    x = [torch.from_numpy(a).cuda() for a in random_arrays(inputs, size_dict, np.complex128, 3)]
    prog = A.SlicedProgram(inputs, output, size_dict, path, (), dtype=np.complex128, gradient=True, use_graph=False)
    g_out = torch.randn(tuple(size_dict[l] for l in output), dtype=torch.complex128, device="cuda")
    out0, grads0 = prog.gradient(x, g_out, part=0)
    ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
    out1, _ = prog.gradient(x, part=1, workspace=ws)
    _, grads2 = prog.gradient(x, g_out, part=2, workspace=ws)
    assert torch.equal(out0, out1)
    for a, b in zip(grads0, grads2):
        assert torch.equal(a, b)


def test_autograd_function_and_central_differences_grid():
    # 4x4 open grid, bond 3, c128; directional central differences in FP64, eps = 1e-3.
    net = N.grid_2d(4, 4, 3)
    arrays = N.gaussian_tensors(net, np.complex128, 5, scale_base=3)
    path = A.greedy(*net.as_tuple())
    con = Contraction(*net.as_tuple(), path)
    x = [torch.from_numpy(a).cuda().requires_grad_() for a in arrays]
    out = con(*x)
    out.real.backward()  # L = Re f  ->  grad = conj(df/dT) (PyTorch's convention for holomorphic f)
    g = [t.grad.cpu().numpy() for t in x]
    rng = np.random.default_rng(0)
    eps = 1e-3
    for _ in range(8):
        v = [(rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape)) for a in arrays]
        fp = complex(O.contract_sliced(*net.as_tuple(), path, [], [a + eps * d for a, d in zip(arrays, v)]))
        fm = complex(O.contract_sliced(*net.as_tuple(), path, [], [a - eps * d for a, d in zip(arrays, v)]))
        fd = (fp - fm) / (2 * eps)
        lin = sum(np.sum(np.conj(gi) * vi) for gi, vi in zip(g, v))
        # d Re f along V  =  Re(sum conj(g) V)
        assert abs(fd.real - lin.real) <= 1e-6 * max(1.0, abs(fd)), (fd, lin)


def test_grid8_bond6_c64_gradient_tf32x3_against_c128():
    # 8x8 open grid, bond 6, c64 N(0,1)/sqrt(6^rank): the adjoint on the tensor cores against the FP64 sweep.
    net, arrays = N.workload_grid8(6, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    x64 = [torch.from_numpy(a).cuda() for a in arrays]
    x128 = [t.to(torch.complex128) for t in x64]
    p32 = A.SlicedProgram(*net.as_tuple(), path, (), dtype=np.complex64, precision="tf32x3", gradient=True,
                          use_graph=False, workspace_budget=40 << 30)
    p64 = A.SlicedProgram(*net.as_tuple(), path, (), dtype=np.complex128, gradient=True, use_graph=False,
                          workspace_budget=40 << 30)
    o32, g32 = p32.gradient(x64)
    o64, g64 = p64.gradient(x128)
    assert abs(complex(o32.item()) - complex(o64.item())) / abs(complex(o64.item())) <= 1e-5
    for a, b in zip(g32, g64):
        assert max_rel(a.cpu().numpy(), b.cpu().numpy()) <= 1e-5 * max(1.0, 1.0)

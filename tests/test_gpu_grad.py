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

    def central(v, h):
        fp = complex(O.contract_sliced(*net.as_tuple(), path, [], [a + h * d for a, d in zip(arrays, v)]))
        fm = complex(O.contract_sliced(*net.as_tuple(), path, [], [a - h * d for a, d in zip(arrays, v)]))
        return (fp - fm) / (2 * h)

    for _ in range(8):
        # directions scaled like the tensors themselves (entries ~ N(0,1)/sqrt(3^rank))
        v = [(rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape)) / np.sqrt(3.0 ** a.ndim)
             for a in arrays]
        d1, d2 = central(v, eps), central(v, eps / 2)
        rich = (4 * d2 - d1) / 3  # removes the eps^2 term of the central difference
        lin = sum(np.sum(np.conj(gi) * vi) for gi, vi in zip(g, v))
        # d Re f along V  =  Re(sum conj(g) V)
        assert abs(d1.real - lin.real) <= 1e-3 * abs(d1), (d1, lin)
        assert abs(rich.real - lin.real) <= 1e-8 * abs(rich), (rich, lin)


def test_grid8_bond6_c64_gradient_tf32x3_against_c128():
    # 8x8 open grid, bond 6, c64 N(0,1)/sqrt(6^rank): the adjoint on the tensor cores against the FP64 sweep.
    # With that scaling the scalar is ~1e-35, at the bottom of FP32's range; every input is multiplied
    # by 4 (exact in binary floating point), which scales the result by 4^64 and every gradient by 4^63.
    # The contraction cancels heavily (the scalar is far below the norms of its intermediates), so even
    # exact-FP32 arithmetic misses the c128 value by ~3e-5 relative: the scalar must do as well as the FP32
    # SIMT path (1.7e-5 against 2.5e-5 measured).  Every gradient tensor meets 1e-5 normwise,
    # ||g - g_ref||_F / ||g_ref||_F (at most 7.9e-6 measured; the FP32 path 5.5e-6).
    net, arrays = N.workload_grid8(6, np.complex64, seed=0)
    arrays = [a * np.float32(4.0) for a in arrays]
    path = A.greedy(*net.as_tuple())
    x64 = [torch.from_numpy(a).cuda() for a in arrays]
    x128 = [t.to(torch.complex128) for t in x64]
    kw = dict(gradient=True, use_graph=False, workspace_budget=40 << 30)
    ptc = A.SlicedProgram(*net.as_tuple(), path, (), dtype=np.complex64, precision="tf32x3", **kw)
    pf32 = A.SlicedProgram(*net.as_tuple(), path, (), dtype=np.complex64, precision="fp32", **kw)
    p64 = A.SlicedProgram(*net.as_tuple(), path, (), dtype=np.complex128, **kw)
    otc, gtc = ptc.gradient(x64)
    of32, gf32 = pf32.gradient(x64)
    o64, g64 = p64.gradient(x128)
    ref = complex(o64.item())

    def rel(o):
        return abs(complex(o.item()) - ref) / abs(ref)

    assert rel(of32) <= 1e-4  # sanity of the comparison itself
    assert rel(otc) <= max(1e-5, rel(of32)), (rel(otc), rel(of32))
    for a, f, b in zip(gtc, gf32, g64):
        a, f, b = (t.cpu().numpy().astype(np.complex128) for t in (a, f, b))
        scale = np.linalg.norm(b)
        err_tc, err_f32 = np.linalg.norm(a - b) / scale, np.linalg.norm(f - b) / scale
        assert err_tc <= 1e-5, (err_tc, err_f32)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
def test_recompute_under_workspace_budget_is_bit_identical(dtype):
    # A budget far below what keeping every intermediate needs: the program drops step results from
    # what the adjoint keeps and recomputes them with the same kernels, so nothing changes bitwise.
    net = N.grid_2d(5, 5, 3)
    arrays = N.gaussian_tensors(net, dtype, 2, scale_base=3)
    path = A.greedy(*net.as_tuple())
    x = [torch.from_numpy(a).cuda() for a in arrays]
    full = A.SlicedProgram(*net.as_tuple(), path, (), dtype=dtype, gradient=True, use_graph=False)
    small = A.SlicedProgram(*net.as_tuple(), path, (), dtype=dtype, gradient=True, use_graph=False,
                            workspace_budget=1)
    assert full.recomputed_steps == 0
    assert small.recomputed_steps >= 1
    assert small.workspace_bytes < full.workspace_bytes
    o1, g1 = full.gradient(x)
    o2, g2 = small.gradient(x)
    assert torch.equal(o1, o2)
    for a, b in zip(g1, g2):
        assert torch.equal(a, b)
    # the forward part alone is unchanged by recompute
    assert torch.equal(small.execute(x), full.execute(x))


def _norm_rel(a, b):
    a = np.asarray(a.cpu() if hasattr(a, "cpu") else a, dtype=np.complex128)
    b = np.asarray(b.cpu() if hasattr(b, "cpu") else b, dtype=np.complex128)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# Sliced adjoint: every slice group runs its own reverse sweep; the per-slice input gradients add up in
# FP64.  "mixed" has a diagonal, a trace, a dangling leg, a hyperedge (leg 9) and open legs (8, 10).
@pytest.mark.parametrize("sliced", [[2], [2, 9], [8], [2, 8, 10]], ids=["internal", "internal2", "output", "mixed"])
def test_sliced_gradients_equal_unsliced(sliced):
    inputs, output, size_dict = SMALL_NETWORKS["mixed"]
    path = A.greedy(inputs, output, size_dict)
    x = [torch.from_numpy(a).cuda() for a in random_arrays(inputs, size_dict, np.complex128, 21)]
    shape = tuple(size_dict[l] for l in output)
    g_out = torch.from_numpy(random_arrays([output], size_dict, np.complex128, 22)[0].reshape(shape)).cuda()
    full = A.SlicedProgram(inputs, output, size_dict, path, (), dtype=np.complex128, gradient=True, use_graph=False)
    o1, g1 = full.gradient(x, g_out)
    for group in (1, 2):
        sl = A.SlicedProgram(inputs, output, size_dict, path, sliced, dtype=np.complex128, gradient=True,
                             use_graph=False, max_slices_per_group=group)
        assert sl.n_slices > 1
        ws = torch.empty(max(sl.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
        o2, g2 = sl.gradient(x, g_out, workspace=ws)
        assert _norm_rel(o2, o1) <= 1e-12
        for a, b in zip(g2, g1):
            assert a.shape == b.shape and _norm_rel(a, b) <= 1e-12, (sliced, group)
        assert sl.device_status(ws) == 0


def test_sliced_gradients_are_independent_of_the_group_size():
    # Accumulation runs in global slice order whatever the grouping, so the sums match bit for bit.
    net, arrays = N.workload_rand3reg(24, 2, 1, np.complex128, seed=3)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 3)  # 5 legs, 32 slices
    assert sliced
    x = [torch.from_numpy(a).cuda() for a in arrays]
    res = []
    for group in (1, 3, 0):
        p = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex128, gradient=True, use_graph=False,
                            max_slices_per_group=group)
        res.append(p.gradient(x))
    for o, g in res[1:]:
        assert torch.equal(o, res[0][0])
        for a, b in zip(g, res[0][1]):
            assert torch.equal(a, b)


def test_sliced_c64_gradients_through_autograd_match_c128():
    net, arrays = N.workload_rand3reg(32, 2, 1, np.complex64, seed=4)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 6)
    assert sliced
    con = Contraction(*net.as_tuple(), path, sliced_legs=sliced, precision="tf32x3")
    x = [torch.from_numpy(a).cuda().requires_grad_() for a in arrays]
    out = con(*x)
    out.real.backward()
    ref = A.SlicedProgram(*net.as_tuple(), path, (), dtype=np.complex128, gradient=True, use_graph=False)
    o64, g64 = ref.gradient([t.detach().to(torch.complex128) for t in x],
                            torch.ones((), dtype=torch.complex128, device="cuda"))
    assert abs(complex(out.item()) - complex(o64.item())) <= 1e-5 * abs(complex(o64.item()))
    for t, b in zip(x, g64):
        assert _norm_rel(t.grad, b) <= 1e-5


def test_sliced_gradient_parts_one_and_two_are_rejected():
    inputs, output, size_dict = SMALL_NETWORKS["mixed"]
    path = A.greedy(inputs, output, size_dict)
    x = [torch.from_numpy(a).cuda() for a in random_arrays(inputs, size_dict, np.complex128, 5)]
    sl = A.SlicedProgram(inputs, output, size_dict, path, [2], dtype=np.complex128, gradient=True, use_graph=False)
    with pytest.raises(ValueError, match="part 0"):
        sl.gradient(x, part=1)
    # a plain execute of the gradient program is the forward contraction
    plain = A.SlicedProgram(inputs, output, size_dict, path, [2], dtype=np.complex128, use_graph=False)
    assert torch.equal(sl.execute(x), plain.execute(x))

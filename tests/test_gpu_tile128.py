"""Large real float32 steps: the 128 x 128 FP32 tile GEMM (k_gemm_tile128, precision fp32) and the
complex tensor-core GEMM on half the K (precision tf32x3: A' = A1 + i A2, B' = conj(B1 + i B2),
Re(A'.B') = A.B).

Checked against an FP64 matmul of the same operands (normwise, FP32 tolerance), with operands stored in
both row orders (contiguous and transposed K) and odd K, the tile GEMM also against the batch
interpreter's run of the same body (bit for bit), and the tensor-core form's gradients against the FP32
form's.
"""

import numpy as np
import pytest
import torch

import arctn_b200 as A

pytestmark = pytest.mark.gpu


def two_tensor(m, k, n, transposed):
    # C[i, j] = sum_l A[i, l] B[l, j]; transposed stores A as [l, i] and B as [j, l]
    inputs = [[1, 0], [2, 1]] if transposed else [[0, 1], [1, 2]]
    return inputs, [0, 2], {0: m, 1: k, 2: n}


@pytest.mark.parametrize("transposed", [False, True])
@pytest.mark.parametrize("m,k,n", [(2048, 256, 2048), (2000, 300, 1900)])
def test_tile128_matches_fp64(m, k, n, transposed):
    inputs, output, size = two_tensor(m, k, n, transposed)
    prog = A.SlicedProgram(inputs, output, size, [(0, 1)], (), dtype=np.float32)
    assert [o["kind"] for o in prog.describe()["ops"] if o["kind"].startswith("gemm")] == ["gemm_tile128"]
    rng = np.random.default_rng(7)
    arrays = [rng.standard_normal([size[l] for l in legs]).astype(np.float32) for legs in inputs]
    got = prog.execute([torch.from_numpy(a).cuda() for a in arrays]).cpu().numpy().astype(np.float64)
    a64, b64 = (arrays[0].T, arrays[1].T) if transposed else (arrays[0], arrays[1])
    want = a64.astype(np.float64) @ b64.astype(np.float64)
    assert np.linalg.norm(got - want) <= 1e-6 * np.linalg.norm(want) * np.sqrt(k)


def test_tile128_interpreter_equals_launch():
    inputs, output, size = two_tensor(1024, 128, 1024, False)  # 64 tiles: picked in a batch only when sliced
    prog = A.SlicedProgram(inputs, output, size, [(0, 1)], (), dtype=np.float32, use_graph=False)
    kinds = [o["kind"] for o in prog.describe()["ops"] if o["kind"].startswith("gemm")]
    inputs2, output2, size2 = two_tensor(2048, 128, 2048, True)
    prog2 = A.SlicedProgram(inputs2, output2, size2, [(0, 1)], (), dtype=np.float32, use_graph=False)
    assert [o["kind"] for o in prog2.describe()["ops"] if o["kind"].startswith("gemm")] == ["gemm_tile128"]
    rng = np.random.default_rng(8)
    xs = [[torch.from_numpy(rng.standard_normal([s[l] for l in legs]).astype(np.float32)).cuda() for legs in ins]
          for ins, s in [(inputs, size), (inputs2, size2)]]
    batch = A.ProgramBatch([prog, prog2], max_lanes=2, mode="staged")  # both inside the interpreter
    ws = torch.empty(batch.workspace_bytes, dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        outs = batch.execute(xs, workspace=ws, stream=st)
        assert batch.device_status(ws, stream=st) == 0
    assert kinds  # the small one uses the 64 x 64 tile or a thinner kernel
    for p, x, o in zip([prog, prog2], xs, outs):
        assert torch.equal(o, p.execute(x))


@pytest.mark.parametrize("transposed", [False, True])
@pytest.mark.parametrize("m,k,n", [(1024, 512, 768), (700, 301, 650)])
def test_real_tensor_core_matches_fp64(m, k, n, transposed):
    inputs, output, size = two_tensor(m, k, n, transposed)
    prog = A.SlicedProgram(inputs, output, size, [(0, 1)], (), dtype=np.float32, precision="tf32x3")
    ops = prog.describe()["ops"]
    assert [o.get("real") for o in ops if o["kind"] == "gemm_tc"] == [1]
    rng = np.random.default_rng(9)
    arrays = [rng.standard_normal([size[l] for l in legs]).astype(np.float32) for legs in inputs]
    got = prog.execute([torch.from_numpy(a).cuda() for a in arrays]).cpu().numpy().astype(np.float64)
    a64, b64 = (arrays[0].T, arrays[1].T) if transposed else (arrays[0], arrays[1])
    want = a64.astype(np.float64) @ b64.astype(np.float64)
    assert np.linalg.norm(got - want) <= 1e-6 * np.linalg.norm(want) * np.sqrt(k)


def test_real_tensor_core_gradient_matches_fp32():
    inputs, output, size = two_tensor(512, 384, 640, False)
    rng = np.random.default_rng(10)
    arrays = [torch.from_numpy(rng.standard_normal([size[l] for l in legs]).astype(np.float32)).cuda()
              for legs in inputs]
    res = {}
    for precision in ("fp32", "tf32x3"):
        prog = A.SlicedProgram(inputs, output, size, [(0, 1)], (), dtype=np.float32, precision=precision,
                               gradient=True)
        kinds = [o["kind"] for o in prog.describe()["ops"]]
        assert ("gemm_tc" in kinds) == (precision == "tf32x3")
        out, grads = prog.gradient(arrays)
        res[precision] = (out.double(), [g.double() for g in grads])
    (o32, g32), (otc, gtc) = res["fp32"], res["tf32x3"]
    assert torch.linalg.norm(otc - o32) <= 1e-5 * torch.linalg.norm(o32)
    for a, b in zip(gtc, g32):
        assert torch.linalg.norm(a - b) <= 1e-5 * torch.linalg.norm(b)

"""torch.autograd integration of the B200 executor.

The reference makes each compiled stage callable so a caller can put pair
contractions on an autograd tape (``src/compiled.rs:7-10``, README
"step-by-step" API).  Here the whole contraction is one autograd node whose
backward is the executor's own adjoint sweep (``arctn_b200_program_gradient``):
the forward runs with its intermediates kept in a workspace saved on the
node, and the backward runs only the reverse sweep on that workspace.
"""

from __future__ import annotations

import numpy as np
import torch

from .api import SlicedProgram, _torch_code


class _Contract(torch.autograd.Function):
    @staticmethod
    def forward(ctx, prog, *tensors):
        ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device=tensors[0].device)
        out, _ = prog.gradient(list(tensors), part=1, workspace=ws)
        ctx.prog = prog
        ctx.ws = ws
        ctx.save_for_backward(*tensors)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        tensors = ctx.saved_tensors
        _, grads = ctx.prog.gradient(list(tensors), grad_out.contiguous(), part=2, workspace=ctx.ws)
        ctx.ws = None
        return (None, *grads)


class Contraction:
    """A differentiable contraction of CUDA tensors along a fixed SSA path.

    ``Contraction(inputs, output, size_dict, ssa_path)(*tensors)`` returns the
    output tensor; ``.backward()`` on anything computed from it yields
    ``tensor.grad`` for every input that requires gradients.
    """

    def __init__(self, inputs, output, size_dict, ssa_path, *, precision="fp32"):
        self.args = (inputs, output, size_dict, ssa_path)
        self.precision = precision
        self._programs = {}

    def program(self, dtype, device):
        key = (dtype, device)
        if key not in self._programs:
            self._programs[key] = SlicedProgram(*self.args, (), dtype=_torch_code(dtype), precision=self.precision,
                                                device=device, use_graph=False, gradient=True)
        return self._programs[key]

    def __call__(self, *tensors):
        t0 = tensors[0]
        return _Contract.apply(self.program(t0.dtype, t0.device.index), *tensors)


def contract(inputs, output, size_dict, ssa_path, *tensors, precision="fp32"):
    """One-shot differentiable contraction (builds the program on every call)."""
    return Contraction(inputs, output, size_dict, ssa_path, precision=precision)(*tensors)


__all__ = ["Contraction", "contract"]
_ = np  # numpy is imported for callers that pass host arrays to SlicedProgram directly

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
        ctx.prog = prog
        ctx.save_for_backward(*tensors)
        if prog.sliced_legs:
            # Sliced: each slice group's reverse sweep reuses that group's workspace, so the backward
            # reruns the forward with it (part 0); the forward here is a plain execute.
            ctx.ws = None
            return prog.execute(list(tensors))
        ws = torch.empty(max(prog.workspace_bytes, 1), dtype=torch.uint8, device=tensors[0].device)
        out, _ = prog.gradient(list(tensors), part=1, workspace=ws)
        ctx.ws = ws
        return out

    @staticmethod
    def backward(ctx, grad_out):
        tensors = ctx.saved_tensors
        if ctx.prog.sliced_legs:
            _, grads = ctx.prog.gradient(list(tensors), grad_out.contiguous(), part=0)
        else:
            _, grads = ctx.prog.gradient(list(tensors), grad_out.contiguous(), part=2, workspace=ctx.ws)
        ctx.ws = None
        return (None, *grads)


class Contraction:
    """A differentiable contraction of CUDA tensors along a fixed SSA path.

    ``Contraction(inputs, output, size_dict, ssa_path)(*tensors)`` returns the
    output tensor; ``.backward()`` on anything computed from it yields
    ``tensor.grad`` for every input that requires gradients.
    """

    def __init__(self, inputs, output, size_dict, ssa_path, *, sliced_legs=(), precision="fp32", **program_kw):
        self.args = (inputs, output, size_dict, ssa_path)
        self.sliced_legs = tuple(sliced_legs)
        self.precision = precision
        self.program_kw = program_kw
        self._programs = {}

    def program(self, dtype, device):
        key = (dtype, device)
        if key not in self._programs:
            self._programs[key] = SlicedProgram(*self.args, self.sliced_legs, dtype=_torch_code(dtype),
                                                precision=self.precision, device=device, use_graph=False,
                                                gradient=True, **self.program_kw)
        return self._programs[key]

    def __call__(self, *tensors):
        t0 = tensors[0]
        return _Contract.apply(self.program(t0.dtype, t0.device.index), *tensors)


def contract(inputs, output, size_dict, ssa_path, *tensors, sliced_legs=(), precision="fp32"):
    """One-shot differentiable contraction (builds the program on every call)."""
    return Contraction(inputs, output, size_dict, ssa_path, sliced_legs=sliced_legs, precision=precision)(*tensors)


__all__ = ["Contraction", "contract"]
_ = np  # numpy is imported for callers that pass host arrays to SlicedProgram directly

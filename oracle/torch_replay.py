"""Step-by-step torch replay of a compiled plan -- TEST INFRASTRUCTURE ONLY (gradient oracle).

The reference exposes its compiled stages so a caller can put every pair
contraction on an autograd tape (``src/compiled.rs:7-10``: input preps, pair
steps and finalize run in order give the same result as ``execute``).  This
module is that caller: it replays the oracle's plan (``oracle.plan_json``)
stage by stage with one ``torch.einsum`` per stage on CPU tensors, so
``torch.autograd`` yields the reference-path gradient of every input.
Only tests/ may import it.
"""

from __future__ import annotations

import torch

from . import oracle as O


def _einsum(*operands_and_legs):
    """torch.einsum in sublist form with the network's leg ids renumbered 0, 1, ... for this one stage
    (torch accepts sublist labels below 52 only; a stage names far fewer legs than that)."""
    local = {}
    args = []
    for i, x in enumerate(operands_and_legs):
        if i % 2 == 0 and i + 1 < len(operands_and_legs):
            args.append(x)
        else:
            args.append([local.setdefault(int(l), len(local)) for l in x])
    return torch.einsum(*args)


def replay(inputs, output, size_dict, ssa_path, tensors):
    """Contract CPU torch tensors along the plan; differentiable with torch.autograd."""
    plan = O.plan_json(inputs, output, size_dict, ssa_path)
    slots = []
    for legs, prep, t in zip(inputs, plan["preps"], tensors):
        # trace (leg dropped) / diagonal (leg kept once), src/compiled.rs:60-75
        slots.append(_einsum(t, list(legs), list(prep["legs"])) if prep["traces"] else t)
    for st in plan["steps"]:
        a, b = slots[st["left_slot"]], slots[st["right_slot"]]
        slots[st["left_slot"]] = slots[st["right_slot"]] = None
        # dangling legs are summed, the result is laid out [batch, free_a, free_b] (src/compiled.rs:155-171)
        slots.append(_einsum(a, list(st["left_legs"]), b, list(st["right_legs"]), list(st["result_legs"])))
    fin = plan["finalize"]
    return _einsum(slots[fin["slot"]], list(fin["input_legs"]), list(output))

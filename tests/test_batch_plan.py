"""Host-side plan of the persistent batch interpreter, checked without a GPU (arctn_b200_batch_describe).

The interpreter's correctness rests on its queue: every step of every program appears once, its waits
name exactly its same-stage interpreter dependencies, those sit earlier in the queue (so the claim order
can always make progress), and every dependency across a stage boundary is ordered by the launches
between stages.  These tests rebuild the dependency relation from each program's own description and
check the batch plan against it.
"""

import numpy as np
import pytest

import arctn_b200 as A
from arctn_b200 import networks as N

EXTERNAL = {"gemm_tc", "pack", "pack_tiled", "maxabs", "strip"}


def programs(count, seed, precision, gradient, sliced_target=None):
    out = []
    for net, arrays in N.workload_batch(count, seed=seed):
        path = A.greedy(*net.as_tuple())
        sliced = ()
        if sliced_target is not None:
            sliced = A.find_slices_to_size(*net.as_tuple(), path, sliced_target)
        out.append(A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=arrays[0].dtype, precision=precision,
                                   gradient=gradient, use_graph=False, device=0, max_slices_per_group=2))
    return out


def in_part(op, part):
    return part == 0 or not op.get("bwd")


def part_deps(ops, part):
    """Dependencies restricted to the part: a skipped op is replaced by its own dependencies."""
    deps = []
    for i, op in enumerate(ops):
        d = set()
        for x in op["deps"]:
            d |= {x} if in_part(ops[x], part) else deps[x]
        deps.append(d)
    return deps


def check_plan(progs, batch):
    desc = batch.describe(detail=True)
    assert desc["mode"] in ("persistent", "staged")
    interpreted = set(desc["interpreted"])
    offs = desc["program_offsets"]
    for j in range(1, len(progs)):  # disjoint workspace regions
        assert offs[j] >= offs[j - 1] + progs[j - 1].workspace_bytes
    assert desc["workspace_bytes"] >= offs[-1] + progs[-1].workspace_bytes
    for part in desc["parts"]:
        p = part["part"]
        steps = part["step_list"]
        staged = part["staged_launches"]
        stage_of, pos_of, step_of, first_of = {}, {}, {}, {}
        for q, (j, i, sub, st, lv, nvb, deps) in enumerate(steps):
            assert nvb >= 1
            assert all(d < q for d in deps), "a wait must name an earlier queue entry"
            assert all(steps[d][3] == st for d in deps), "waits stay within a stage"
            if sub == 0:
                assert (j, i) not in first_of, "one entry per op"
                stage_of[(j, i)] = st
                first_of[(j, i)] = q
            step_of[(j, i)] = q  # the op's last descriptor
        assert [s[3] for s in steps] == sorted(s[3] for s in steps), "stages are contiguous in the queue"
        for k, (st, j, i) in enumerate(staged):
            assert (j, i) not in stage_of
            stage_of[(j, i)] = st
            pos_of[(j, i)] = k
        assert part["tasks"] == sum(s[5] for s in steps)
        assert sum(part["stage_tasks"]) == part["tasks"]
        assert sum(part["stage_launches"]) == len(staged)
        for j, prog in enumerate(progs):
            ops = prog.describe()["ops"]
            if j not in interpreted:  # a lane program: launched on its own
                assert all((j, i) not in stage_of for i in range(len(ops)))
                continue
            deps = part_deps(ops, p)
            for i, op in enumerate(ops):
                if not in_part(op, p):
                    assert (j, i) not in stage_of
                    continue
                assert (j, i) in stage_of, (j, i, op["kind"])
                ext = op["kind"] in EXTERNAL
                assert ext == ((j, i) not in first_of)
                for d in deps[i]:
                    dext = ops[d]["kind"] in EXTERNAL
                    si, sd = stage_of[(j, i)], stage_of[(j, d)]
                    if ext and dext:  # same lane, in op order
                        assert sd < si or (sd == si and pos_of[(j, d)] < pos_of[(j, i)])
                    elif ext:  # an interpreter step before a staged launch: an earlier interpreter launch
                        assert sd < si
                    elif dext:  # a staged launch before an interpreter step: launched before its stage
                        assert sd <= si
                    elif sd == si:
                        assert step_of[(j, d)] in steps[first_of[(j, i)]][6]
                    else:
                        assert sd < si
    return desc


@pytest.mark.parametrize("mode", ["persistent", "staged"])
@pytest.mark.parametrize("precision", ["fp32", "tf32x3"])
def test_gradient_batch_plan(precision, mode):
    progs = programs(8, 0, precision, True)  # networks 5 and 7 have tensor-core steps under tf32x3
    desc = check_plan(progs, A.ProgramBatch(progs, max_lanes=4, mode=mode))
    parts = {p["part"]: p for p in desc["parts"]}
    assert set(parts) == {-1, 0}
    tc = {j for j, p in enumerate(progs) if any(o["kind"] == "gemm_tc" for o in p.describe()["ops"])}
    assert (precision == "tf32x3") == bool(tc)
    if mode == "staged":  # every program interpreted; tensor-core steps between interpreter launches
        assert desc["interpreted"] == list(range(len(progs)))
        assert (sum(parts[0]["stage_launches"]) > 0) == bool(tc)
    else:  # programs with tensor-core steps (or large ones) run on the lanes alongside one launch
        assert not tc & set(desc["interpreted"])
        assert parts[0]["stages"] == 1 and sum(parts[0]["stage_launches"]) == 0
        assert all(progs[j].flops <= 5e8 for j in desc["interpreted"])


def test_sliced_gradient_batch_plan():
    # the reverse sweep runs inside every slice group, so the forward part skips interleaved reverse steps
    progs = []
    for rows, cols, bond, target in [(4, 4, 2, 2 ** 3), (4, 5, 2, 2 ** 4), (3, 3, 4, 2 ** 4)]:
        net = N.grid_2d(rows, cols, bond)
        path = A.greedy(*net.as_tuple())
        sliced = A.find_slices_to_size(*net.as_tuple(), path, target)
        progs.append(A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3",
                                     gradient=True, use_graph=False, device=0, max_slices_per_group=2))
    assert all(p.n_slices >= 8 for p in progs)
    check_plan(progs, A.ProgramBatch(progs, max_lanes=2, mode="staged"))


def test_plain_batch_plan_and_lanes_mode():
    progs = programs(6, 6, "fp32", False)
    desc = check_plan(progs, A.ProgramBatch(progs))
    assert [p["part"] for p in desc["parts"]] == [-1]
    lanes = A.ProgramBatch(progs, max_lanes=2, mode="lanes").describe()
    assert lanes["mode"] == "lanes" and lanes["parts"] == [] and lanes["lanes"] == 2
    assert lanes["workspace_bytes"] <= desc["workspace_bytes"]

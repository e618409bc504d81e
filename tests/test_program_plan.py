"""Host-side program planning, checked without a GPU through arctn_b200_program_describe.

A program builds its whole launch sequence and workspace layout on the host; these tests read that
plan back: launch counts, the tensor-core / pack geometry, the adjoint's checkpoint recompute under a
workspace budget, and option validation.
"""

import numpy as np
import pytest

import arctn_b200 as A
from arctn_b200 import networks as N

GEMM_KINDS = {"gemm_small", "gemm_tile64", "gemm_tile32", "gemm_tile128", "gemm_dot", "gemm_tc", "gemm_warp"}


def program(net, path, sliced=(), **kw):
    return A.SlicedProgram(*net.as_tuple(), path, sliced, device=0, **kw)


def test_describe_matches_counters_and_plan():
    net = N.grid_2d(4, 4, 3)
    path = A.greedy(*net.as_tuple())
    p = program(net, path, dtype=np.complex128)
    d = p.describe()
    assert d["workspace_bytes"] == p.workspace_bytes
    # one launch per launch unit (independent thin GEMMs of one DAG level share one grouped launch)
    units = {o["unit"] for o in d["ops"] if o["kind"] != "memset"}
    assert d["launches"] == p.launches == len(units) <= sum(o["kind"] != "memset" for o in d["ops"])
    assert d["groups"] == 1 and d["n_slices"] == 1
    gemms = [o for o in d["ops"] if o["kind"] in GEMM_KINDS]
    assert len(gemms) == len(path)  # one GEMM per pairwise step
    cc = A.CompiledContraction.compile(*net.as_tuple(), ssa_path=path)
    dims = sorted(tuple(s.gemm_dims()) for s in cc.pair_steps())
    assert sorted((o["bt"], o["m"], o["k"], o["n"]) for o in gemms) == dims


def test_sliced_program_groups_and_flops():
    net, _ = N.workload_rand3reg(64, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 8)
    p = program(net, path, sliced, dtype=np.complex64, max_slices_per_group=16)
    d = p.describe()
    assert d["n_slices"] == 2 ** len(sliced)
    assert d["slices_per_group"] == 16
    assert d["groups"] == -(-d["n_slices"] // 16)
    cc = A.CompiledContraction.compile(net.inputs, net.output,
                                       {l: (1 if l in sliced else s) for l, s in net.size_dict.items()},
                                       ssa_path=path)
    per_slice = 8.0 * sum(a * b * c * e for a, b, c, e in (s.gemm_dims() for s in cc.pair_steps()))
    assert p.flops == pytest.approx(per_slice * d["n_slices"], rel=1e-12)


def test_tf32x3_packs_use_full_tiles_and_split_long_k():
    net, _ = N.workload_rand3reg(172, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 24)
    p = program(net, path, sliced, dtype=np.complex64, precision="tf32x3", max_slices_per_group=4)
    ops = p.describe()["ops"]
    tc = [o for o in ops if o["kind"] == "gemm_tc"]
    packs = [o for o in ops if o["kind"] == "pack_tiled"]
    assert tc and len(packs) + sum("pack_into" in o for o in tc) == 2 * len(tc)
    for o in tc:
        assert (o["k"] >= 32 and ((o["m"] >= 96 and o["n"] >= 96) or (min(o["m"], o["n"]) >= 16 and o["k"] >= 256))
                or (o["k"] >= 16 and o["m"] >= 96 and o["n"] >= 96))
        assert o["splits"] == 1  # slice-batched GEMMs fill the GPU without splitting K
    for o in packs:
        assert o["rpad"] % 128 == 0 and o["kpad"] % 16 == 0 and 32 <= o["tile"] <= 1024
    assert all(o["tile"] == 1024 for o in packs)  # dimension-2 legs always fill a tile
    p256 = program(net, path, sliced, dtype=np.complex64, precision="tf32x3", max_slices_per_group=4, tc_k_chunk=256)
    for o in (o for o in p256.describe()["ops"] if o["kind"] == "gemm_tc"):
        assert o["splits"] == max(1, -(-o["k"] // 256))
    fp32 = program(net, path, sliced, dtype=np.complex64, precision="fp32", max_slices_per_group=4)
    assert not any(o["kind"] in ("gemm_tc", "pack_tiled", "pack") for o in fp32.describe()["ops"])


def test_bf16x3_programs_pack_bf16_planes_on_32_wide_k_rows():
    # Split-BF16 runs the same steps on the tensor cores as split-TF32, with 2-byte planes whose packed K
    # is a multiple of 32 (a 64-byte row), and no epilogue packs.
    net, _ = N.workload_rand3reg(172, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 24)
    tf = program(net, path, sliced, dtype=np.complex64, precision="tf32x3", max_slices_per_group=4).describe()["ops"]
    bf = program(net, path, sliced, dtype=np.complex64, precision="bf16x3", max_slices_per_group=4).describe()["ops"]
    tf_tc = [(o["bt"], o["m"], o["k"], o["n"]) for o in tf if o["kind"] == "gemm_tc"]
    bf_tc = [(o["bt"], o["m"], o["k"], o["n"]) for o in bf if o["kind"] == "gemm_tc"]
    assert bf_tc and sorted(bf_tc) == sorted(tf_tc)
    assert all(o["bf16"] == 1 for o in bf if o["kind"] in ("gemm_tc", "pack", "pack_tiled"))
    assert all(o["kpad"] % 32 == 0 for o in bf if o["kind"] in ("pack", "pack_tiled"))
    assert not any("pack_into" in o for o in bf)
    assert all(o["bf16"] == 0 for o in tf if o["kind"] == "gemm_tc")
    with pytest.raises(A.ArcTNB200Error, match="multiple of 32"):
        program(net, path, sliced, dtype=np.complex64, precision="bf16x3", tc_k_chunk=16)


def test_bf16x6_programs_pack_six_bf16_planes():
    # Three-piece split-BF16: the same tensor-core steps, 2-byte planes on 32-wide K rows, six planes per operand
    # (so each pack holds 1.5x the bytes of a split-BF16 pair pack), no epilogue packs.
    net, _ = N.workload_rand3reg(172, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 24)
    b3 = program(net, path, sliced, dtype=np.complex64, precision="bf16x3", max_slices_per_group=4).describe()["ops"]
    b6 = program(net, path, sliced, dtype=np.complex64, precision="bf16x6", max_slices_per_group=4).describe()["ops"]
    tc3 = [(o["bt"], o["m"], o["k"], o["n"]) for o in b3 if o["kind"] == "gemm_tc"]
    tc6 = [(o["bt"], o["m"], o["k"], o["n"]) for o in b6 if o["kind"] == "gemm_tc"]
    assert tc6 and tc6 == tc3
    assert all(o["bf16"] == 1 and o["bf16x6"] == 1 for o in b6 if o["kind"] in ("gemm_tc", "pack", "pack_tiled"))
    assert all(o["bf16x6"] == 0 for o in b3 if o["kind"] in ("gemm_tc", "pack", "pack_tiled"))
    assert all(o["kpad"] % 32 == 0 for o in b6 if o["kind"] in ("pack", "pack_tiled"))
    assert not any("pack_into" in o for o in b6)
    with pytest.raises(A.ArcTNB200Error, match="multiple of 32"):
        program(net, path, sliced, dtype=np.complex64, precision="bf16x6", tc_k_chunk=16)
    with pytest.raises(A.ArcTNB200Error, match="precision"):
        program(net, path, sliced, dtype=np.complex64, precision=4)


def test_tensor_core_epilogues_pack_the_next_gemm_operand():
    # rand3reg n=172: the producer's epilogue writes the packed operand of the GEMM that reads its result,
    # so no separate pack reads that result; gradient programs keep separate packs.
    net, _ = N.workload_rand3reg(172, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 24)
    p = program(net, path, sliced, dtype=np.complex64, precision="tf32x3", max_slices_per_group=4)
    d = p.describe()
    ops = d["ops"]
    per_group = [i for i, o in enumerate(ops) if "pack_into" in o]
    assert len(per_group) >= 2 * d["groups"]
    for i in per_group:
        prod, dst = ops[i], ops[i]["pack_into"]
        assert prod["kind"] == "gemm_tc" and prod["splits"] == 1
        # the next op touching the packed buffer is the consuming GEMM, reading it as an operand
        nxt = next(o for o in ops[i + 1:] if dst in (o.get("a"), o.get("b"), o.get("c"), o.get("pack_into")))
        assert nxt["kind"] == "gemm_tc" and dst in (nxt["a"], nxt["b"]) and nxt["c"] != dst
    g = program(net, path, sliced, dtype=np.complex64, precision="tf32x3", max_slices_per_group=4, gradient=True)
    assert not any("pack_into" in o for o in g.describe()["ops"])
    fp32 = program(net, path, sliced, dtype=np.complex64, precision="fp32", max_slices_per_group=4)
    assert not any("pack_into" in o for o in fp32.describe()["ops"])


def test_unsliced_small_tile_gemms_split_k_to_fill_the_gpu():
    net, _ = N.workload_grid8(6, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    p = program(net, path, dtype=np.complex64, precision="tf32x3", gradient=True)
    tc = [o for o in p.describe()["ops"] if o["kind"] == "gemm_tc"]
    assert tc
    for o in tc:
        tiles = -(-o["m"] // 128) * -(-o["n"] // 128) * o["bt"]
        k_tiles = -(-o["k"] // 16)
        want = min(-(-2 * 148 // tiles), k_tiles // 8)
        splits = -(-k_tiles // -(-k_tiles // want)) if want >= 2 else 1  # chunk = ceil(k_tiles / want)
        assert o["splits"] == splits, o
    assert any(o["splits"] > 1 for o in tc)  # the adjoint's 1296 x 1296 x 46656 GEMM


def test_tc_k_chunk_must_be_a_multiple_of_16():
    net = N.grid_2d(3, 3, 2)
    path = A.greedy(*net.as_tuple())
    with pytest.raises(ValueError, match="multiple of 16"):
        program(net, path, dtype=np.complex64, precision="tf32x3", tc_k_chunk=100)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64, np.float64])
def test_adjoint_recompute_under_budget(dtype):
    net = N.grid_2d(5, 5, 3)
    path = A.greedy(*net.as_tuple())
    full = program(net, path, dtype=dtype, gradient=True)
    small = program(net, path, dtype=dtype, gradient=True, workspace_budget=1)
    df, ds = full.describe(), small.describe()
    assert df["recomputed_steps"] == [] and full.recomputed_steps == 0
    assert len(ds["recomputed_steps"]) == small.recomputed_steps >= 1
    assert small.workspace_bytes < full.workspace_bytes
    # the forward sweeps are identical; the reverse sweep re-runs each dropped step exactly once
    fwd_f = [o for o in df["ops"][: df["backward_begin"]]]
    fwd_s = [o for o in ds["ops"][: ds["backward_begin"]]]
    assert [o["kind"] for o in fwd_f] == [o["kind"] for o in fwd_s]
    n_gemm = lambda ops: sum(o["kind"] in GEMM_KINDS for o in ops)  # noqa: E731
    bwd_f, bwd_s = df["ops"][df["backward_begin"]:], ds["ops"][ds["backward_begin"]:]
    assert n_gemm(bwd_f) == 2 * len(path)
    assert n_gemm(bwd_s) == 2 * len(path) + small.recomputed_steps
    # a budget the full layout meets recomputes nothing
    roomy = program(net, path, dtype=dtype, gradient=True, workspace_budget=full.workspace_bytes)
    assert roomy.recomputed_steps == 0 and roomy.workspace_bytes == full.workspace_bytes


def test_sliced_gradient_program_interleaves_reverse_sweeps_per_group():
    net, _ = N.workload_rand3reg(64, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 8)
    p = program(net, path, sliced, dtype=np.complex64, gradient=True, max_slices_per_group=32)
    d = p.describe()
    ops, groups, n_in = d["ops"], d["groups"], len(net.inputs)
    assert groups == -(-d["n_slices"] // 32)
    kinds = [o["kind"] for o in ops]
    assert kinds.count("grad_accum") == n_in * groups  # every group folds its slices' input gradients
    assert kinds.count("narrow") == n_in  # once, after the last group
    assert all(o.get("bwd") for o in ops if o["kind"] in ("grad_accum", "narrow"))
    last_output = max(i for i, k in enumerate(kinds) if k == "slice_output")
    assert min(i for i, k in enumerate(kinds) if k == "narrow") > last_output
    # reverse work sits inside the groups: a backward GEMM precedes the next group's forward GEMMs
    first_bwd = min(i for i, o in enumerate(ops) if o.get("bwd") and o["kind"].startswith("gemm"))
    assert any(o["kind"].startswith("gemm") and not o.get("bwd") for o in ops[first_bwd:])
    # a plain execute runs only the forward ops; its GEMM count is the forward program's
    plain = program(net, path, sliced, dtype=np.complex64, max_slices_per_group=32)
    n_gemm = sum(o["kind"].startswith("gemm") for o in plain.describe()["ops"])
    assert sum(o["kind"].startswith("gemm") and not o.get("bwd") for o in ops) == n_gemm


def test_batch_workload_generator():
    nets = N.workload_batch(16, seed=3)
    assert len(nets) == 16
    for j, (net, arrays) in enumerate(nets):
        n = len(net.inputs)
        assert 20 <= n <= 50 and n % 2 == 0
        bond = next(iter(net.size_dict.values()))
        assert bond in (2, 3, 4) and all(v == bond for v in net.size_dict.values())
        assert arrays[0].dtype == (np.float32 if j % 2 == 0 else np.complex64)
        assert all(len(t) == 3 for t in net.inputs)


def _dag_orders_every_overlap(ops):
    # anc[j]: bitset of the ops j follows through its dependency edges.
    anc = []
    for j, o in enumerate(ops):
        a = 0
        for d in o["deps"]:
            assert d < j
            a |= anc[d] | (1 << d)
        anc.append(a)
    # grouped launches: thin GEMMs only, none an ancestor of another
    groups = {}
    for j, o in enumerate(ops):
        groups.setdefault(o["unit"], []).append(j)
    for members in groups.values():
        if len(members) > 1:
            assert all(ops[j]["kind"] == "gemm_small" for j in members)
            assert not any(anc[j] >> i & 1 for i in members for j in members)
    spans = [[(sp, lo, (1 << 64) if hi == -1 else hi) for sp, lo, hi in o["foot"]] for o in ops]
    for j in range(len(ops)):
        for i in range(j):
            if any(si == sj and li < hj and lj < hi_ for si, li, hi_ in spans[i] for sj, lj, hj in spans[j]):
                assert anc[j] >> i & 1, (i, j, ops[i]["kind"], ops[j]["kind"])


@pytest.mark.parametrize("case", ["grid6", "brickwork", "sliced_fused"])
def test_graph_dag_orders_every_pair_of_ops_sharing_memory(case):
    # The captured graph runs independent steps concurrently on 8 lanes; two ops whose memory footprints
    # overlap (a step and its consumer, or two buffers the arena places on the same bytes) must stay ordered.
    if case == "grid6":
        net, _ = N.workload_grid6(np.complex128, seed=0)
        p = program(net, A.greedy(*net.as_tuple()), dtype=np.complex128)
    elif case == "brickwork":
        net, _ = N.brickwork_circuit(30, 14, seed=0)
        p = program(net, A.greedy(*net.as_tuple()), dtype=np.complex64, precision="tf32x3")
    else:
        net, _ = N.workload_rand3reg(104, 2, 1, np.complex64, seed=0)
        path = A.greedy(*net.as_tuple())
        sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 14)
        p = program(net, path, sliced, dtype=np.complex64, precision="tf32x3", max_slices_per_group=4)
    ops = p.describe()["ops"]
    assert all("deps" in o and "foot" in o for o in ops)
    _dag_orders_every_overlap(ops)
    if case != "sliced_fused":
        assert len({o["lane"] for o in ops}) > 1  # independent steps do run on several lanes
        assert len({o["unit"] for o in ops}) < len(ops)  # and thin steps of one level share a launch


def _two_tensor(m, k, n):
    return [[0, 1], [1, 2]], [0, 2], {0: m, 1: k, 2: n}


def test_large_float32_steps_pick_the_128_tile_or_the_folded_tensor_core_gemm():
    inputs, output, size = _two_tensor(2048, 301, 2048)
    ops = A.SlicedProgram(inputs, output, size, [(0, 1)], (), dtype=np.float32, device=0).describe()["ops"]
    assert [o["kind"] for o in ops if o["kind"].startswith("gemm")] == ["gemm_tile128"]
    ops = A.SlicedProgram(inputs, output, size, [(0, 1)], (), dtype=np.float32, precision="tf32x3",
                          device=0).describe()["ops"]
    packs = [o for o in ops if o["kind"] == "pack"]
    gemm = [o for o in ops if o["kind"] == "gemm_tc"]
    assert len(packs) == 2 and len(gemm) == 1 and gemm[0]["real"] == 1
    assert all(p["real"] == 1 and p["cols"] == 151 and p["kpad"] % 16 == 0 for p in packs)  # K = 301 folds to 151
    # the complex product lands in scratch; one gather keeps its real part, into the output
    last = ops[ops.index(gemm[0]) + 1]
    assert last["kind"] == "gather" and last["a"] == gemm[0]["c"] and last["n_out"] == 2048 * 2048
    # complex64 keeps the unfolded K
    ops = A.SlicedProgram(inputs, output, size, [(0, 1)], (), dtype=np.complex64, precision="tf32x3",
                          device=0).describe()["ops"]
    assert [o["real"] for o in ops if o["kind"] == "gemm_tc"] == [0]


def test_adjoint_reads_gradients_through_strides_without_permute_copies():
    # each intermediate's gradient is the adjoint GEMM's output seen through strides: the reverse sweep
    # copies only into the callers' gradient buffers (one gather per input) besides the incoming gradient
    net = N.grid_2d(4, 4, 3)
    p = program(net, A.greedy(*net.as_tuple()), dtype=np.float32, gradient=True)
    bwd = [o for o in p.describe()["ops"] if o.get("bwd")]
    gathers = sum(o["kind"] == "gather" for o in bwd)
    gemms = sum(o["kind"].startswith("gemm") for o in bwd)
    assert gemms == 2 * (len(net.inputs) - 1)
    assert gathers <= len(net.inputs) + 1


@pytest.mark.parametrize("precision", ["fp32", "tf32x3"])
def test_gradient_program_dag_orders_every_pair_of_ops_sharing_memory(precision):
    # the batch interpreter runs a gradient program's steps from these dependencies
    nets = N.workload_batch(8, seed=0)
    for j in (5, 6):
        net, arrays = nets[j]
        p = program(net, A.greedy(*net.as_tuple()), dtype=arrays[0].dtype, precision=precision, gradient=True)
        _dag_orders_every_overlap(p.describe()["ops"])


def test_tmem_chain_defaults_and_setter():
    # Forward split-TF32 programs sum 64 of K per TMEM chain, gradient programs 32; the setter changes every
    # split-TF32 GEMM and rejects other lengths; BF16 formats keep theirs.
    from arctn_b200 import _capi as C

    net, _ = N.workload_rand3reg(104, 2, 1, np.complex64, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 14)
    chains = lambda p: {o["tmem_chunk_k"] for o in p.describe()["ops"] if o["kind"] == "gemm_tc"}  # noqa: E731
    fwd = program(net, path, sliced, dtype=np.complex64, precision="tf32x3")
    grad = program(net, path, sliced, dtype=np.complex64, precision="tf32x3", gradient=True)
    assert chains(fwd) == {64} and chains(grad) == {32}
    assert chains(program(net, path, sliced, dtype=np.complex64, precision="tf32x3", tc_chain_k=128)) == {128}
    assert chains(program(net, path, sliced, dtype=np.complex64, precision="bf16x3")) == {64}
    assert chains(program(net, path, sliced, dtype=np.complex64, precision="bf16x6")) == {32}
    assert C.lib().arctn_b200_program_set_tc_chain(fwd._h, 48) == C.ERR_INVALID

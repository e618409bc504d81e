"""GEMM autotuner, host side: the tuning table's JSON round trip, the candidate sets, and that a table pins
exactly the GEMMs whose key it holds (read back through arctn_b200_program_gemms and describe, which also
ties every pack to the GEMM it serves), all without a GPU.  The timed search itself runs in
tests/test_gpu_tuning.py.
"""

import json

import numpy as np
import pytest

import arctn_b200 as A
from arctn_b200 import _capi as C
from arctn_b200 import networks as N
from arctn_b200 import tuning as T


def rand3reg(n=64, dtype=np.complex64):
    net, _ = N.workload_rand3reg(n, 2, 1, dtype, seed=0)
    path = A.greedy(*net.as_tuple())
    sliced = A.find_slices_to_size(*net.as_tuple(), path, 2 ** 8)
    return net, path, sliced


def test_table_json_round_trip(tmp_path):
    t = T.TuneTable({"device": "test"})
    t.set((C.C64, C.PREC_TF32X3, 2, 1, 0, 1, 512, 16384, 1024), "tc_nfast", {"tc_mfast": 1.5, "tc_nfast": 1.25}, 37)
    t.set((C.F64, C.PREC_FP32, 1, 0, 0, 4, 3, 5, 7), "simt_warp")
    path = tmp_path / "table.json"
    t.save(path)
    u = T.TuneTable.load(path)
    assert sorted(u.keys()) == sorted(t.keys())
    for k in t.keys():
        assert u.get(k) == t.get(k) and u.timings(k) == t.timings(k)
    assert u.meta == {"device": "test"}
    assert json.loads(u.to_json()) == json.loads(t.to_json())
    with pytest.raises(ValueError):
        T.TuneTable.from_json(json.dumps({"format": "other", "version": 1, "entries": []}))
    with pytest.raises(ValueError):
        t.set((1, 2, 3), "simt_warp")
    with pytest.raises(ValueError):
        t.set((C.C64, C.PREC_FP32, 1, 0, 0, 1, 2, 3, 4), "auto")


def test_entries_follow_the_abi_field_order():
    t = T.TuneTable()
    key = (C.C64, C.PREC_TF32X3, 2, 1, 0, 3, 5, 7, 9)
    t.set(key, "tc_splitk")
    t.set((C.C128, C.PREC_FP32, 1, 0, 0, 1, 2, 2, 2), "simt_dot")
    (e,) = t.entries_for(C.C64, C.PREC_TF32X3)
    g = C.GemmChoice(*e)
    assert (g.dtype, g.precision, g.phase, g.a_var, g.b_var, g.bt, g.m, g.k, g.n) == key
    assert T.VARIANT_NAMES[g.variant] == "tc_splitk"
    assert t.entries_for(C.C64, C.PREC_FP32) == []


def test_candidates_respect_dtype_and_precision():
    big = (C.C64, C.PREC_TF32X3, 2, 1, 1, 1, 1024, 64, 16384)
    c = T.candidates(big, 37)
    assert c[:2] == ["tc_mfast", "tc_nfast"] and "simt_dot" not in c and "simt_tile128" not in c
    assert all(not v.startswith("tc_") for v in T.candidates((C.C64, C.PREC_FP32, 1, 0, 0, 1, 512, 512, 512)))
    assert all(not v.startswith("tc_") for v in T.candidates((C.C128, C.PREC_TF32X3, 1, 0, 0, 1, 512, 512, 512)))
    assert "simt_tile128" in T.candidates((C.F32, C.PREC_FP32, 1, 0, 0, 1, 512, 512, 512))
    # a long K over few output tiles may split K; a batch of slices that already fills the GPU does not
    assert "tc_splitk" in T.candidates((C.C64, C.PREC_TF32X3, 1, 0, 0, 1, 128, 65536, 128))
    assert "tc_splitk" not in T.candidates((C.C64, C.PREC_TF32X3, 2, 1, 1, 1, 512, 16384, 1024), 37)
    # the streaming epilogue: split-TF32 only, and only where K is short enough for the epilogue to matter
    assert "tc_stream" in c and "tc_stream" not in T.candidates((C.C64, C.PREC_TF32X3, 2, 1, 1, 1, 512, 16384, 1024), 37)
    assert "tc_stream" not in T.candidates((C.C64, C.PREC_BF16X6, 2, 1, 1, 1, 1024, 64, 16384), 37)
    # the deep ring: split-TF32 only, for K of at least 8 tiles
    assert "tc_deep" in T.candidates((C.C64, C.PREC_TF32X3, 2, 1, 1, 1, 512, 16384, 1024), 37)
    assert "tc_deep" not in T.candidates((C.C64, C.PREC_TF32X3, 2, 1, 1, 1, 1024, 16, 8192), 37)
    # CTA pairs: split-TF32 only, for outputs of more than one 128-row tile
    assert "tc_pair" in T.candidates((C.C64, C.PREC_TF32X3, 2, 1, 1, 1, 512, 16384, 1024), 37)
    assert "tc_pair" not in T.candidates((C.C64, C.PREC_TF32X3, 2, 1, 1, 1, 128, 64, 16384), 37)
    assert "tc_pair" not in T.candidates((C.C64, C.PREC_BF16X6, 2, 1, 1, 1, 512, 16384, 1024), 37)
    assert "tc_pair_stream" in T.candidates((C.C64, C.PREC_TF32X3, 2, 1, 1, 1, 512, 512, 32768), 37)
    assert "tc_pair_stream" not in T.candidates((C.C64, C.PREC_TF32X3, 2, 1, 1, 1, 512, 16384, 1024), 37)


def test_table_pins_only_matching_gemms():
    net, path, sliced = rand3reg()
    base = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3")
    gs = base.gemms()
    assert gs and not any(g["tuned"] for g in gs) and all(g["variant"] != "auto" for g in gs)
    keys = sorted({T.key_of(g) for g in gs})
    pick = keys[len(keys) // 2]
    t = T.TuneTable()
    t.set(pick, "simt_warp")
    p = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3", tuning=t)
    for g0, g1 in zip(gs, p.gemms()):
        assert T.key_of(g0) == T.key_of(g1)
        if T.key_of(g1) == pick:
            assert g1["tuned"] and g1["variant"] == "simt_warp"
        else:
            assert not g1["tuned"] and g1["variant"] == g0["variant"]
    ops = p.describe()["ops"]
    gemm_ops = [o for o in ops if "variant" in o]
    assert [o["variant"] for o in gemm_ops] == [g["variant"] for g in p.gemms()]
    # every pack serves exactly one GEMM, which runs on the tensor cores
    ids = {o["gemm"]: o for o in gemm_ops}
    for o in ops:
        if o["kind"] in ("pack", "pack_tiled"):
            assert ids[o["gemm"]]["kind"] == "gemm_tc"
    # a table for another dtype / precision leaves the program alone
    q = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="fp32", tuning=t)
    assert not any(g["tuned"] for g in q.gemms())


def test_tensor_core_pin_builds_packs_and_rejects_wrong_dtypes():
    net, path, sliced = rand3reg()
    gs = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3").gemms()
    key = next(T.key_of(g) for g in gs if g["variant"].startswith("simt"))
    t = T.TuneTable()
    t.set(key, "tc_nfast")
    p = A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3", tuning=t)
    ops = p.describe()["ops"]
    tc = [o for o in ops if o.get("variant") == "tc_nfast"]
    assert tc and all(o["kind"] == "gemm_tc" for o in tc)
    assert any(o["kind"] in ("pack", "pack_tiled") for o in ops)
    bad = T.TuneTable()
    bad.set((C.C128, C.PREC_FP32) + key[2:], "tc_mfast")
    with pytest.raises(A.ArcTNB200Error, match="tensor-core"):
        A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex128, precision="fp32", tuning=bad)
    bad = T.TuneTable()
    bad.set((C.C64, C.PREC_BF16X3) + key[2:], "tc_stream")
    with pytest.raises(A.ArcTNB200Error, match="split-TF32 only"):
        A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="bf16x3", tuning=bad)
    bad = T.TuneTable()
    bad.set((C.C64, C.PREC_BF16X6) + key[2:], "tc_deep")
    with pytest.raises(A.ArcTNB200Error, match="split-TF32 only"):
        A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="bf16x6", tuning=bad)
    bad = T.TuneTable()
    bad.set((C.C64, C.PREC_BF16X3) + key[2:], "tc_pair")
    with pytest.raises(A.ArcTNB200Error, match="split-TF32 only"):
        A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="bf16x3", tuning=bad)
    bad = T.TuneTable()
    bad.set(key, "simt_tile128")
    with pytest.raises(A.ArcTNB200Error, match="float32"):
        A.SlicedProgram(*net.as_tuple(), path, sliced, dtype=np.complex64, precision="tf32x3", tuning=bad)


def test_abi_rejects_unknown_variant_and_phase():
    import ctypes

    net, path, sliced = rand3reg()
    args = C.NetworkArgs(*net.as_tuple())
    n, p = C.path_array(path)
    sl = np.asarray(sliced, dtype=np.uint32)
    opts = C.ProgramOptions(C.C64, C.PREC_TF32X3, 0, 1, 0, 0, 0, 0, 0, 0)
    for fields, msg in [((C.C64, C.PREC_TF32X3, 1, 0, 0, 42, 1, 2, 2, 2), "unknown variant"),
                        ((C.C64, C.PREC_TF32X3, 3, 0, 0, 1, 1, 2, 2, 2), "phase")]:
        table = (C.GemmChoice * 1)(C.GemmChoice(*fields))
        h = C.vp()
        rc = C.lib().arctn_b200_program_create_tuned(args.ptr, n, p.ctypes.data_as(C.u64p), len(sliced),
                                                     sl.ctypes.data_as(C.u32p), ctypes.byref(opts), table, 1,
                                                     ctypes.byref(h))
        assert rc == C.ERR_INVALID and msg in C.lib().arctn_b200_last_error().decode()

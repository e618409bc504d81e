"""arctn_contract's keyword checks, on CPU: the reference's options with the reference's exception types.

``arctn_contract`` (pybind/python/arctn/__init__.py:903-1072) validates its planning options before it looks
at the arrays (``_validate_auto_preset``, ``_validate_slicing_mode``, ``_validate_max_time``,
``_validate_planner_weights``, ``_validate_bool``, ``_validate_target_size``: ``__init__.py:70-150``), so
every rejection here happens without a GPU.  The accepted forms run on the GPU in tests/test_gpu_api.py.
"""

import pytest

import arctn_b200 as A

NET = ([["a", "b"], ["b", "c"]], ["a", "c"], {"a": 2, "b": 3, "c": 2})


def call(**kw):
    return A.arctn_contract(*NET, None, **kw)


@pytest.mark.parametrize("kw,exc,msg", [
    (dict(preset="medium"), ValueError, "preset"),
    (dict(preset=None), ValueError, "preset"),
    (dict(seed=True), TypeError, "seed"),
    (dict(seed="1"), TypeError, None),
    (dict(target_size=0), ValueError, "target_size"),
    (dict(target_size=True), TypeError, "target_size"),
    (dict(target_size=2.5), TypeError, "target_size"),
    (dict(target_size=2 ** 80), OverflowError, "target_size"),
    (dict(slicing_mode="greedy"), ValueError, "slicing_mode"),
    (dict(slicing_mode="dynamic"), ValueError, "requires target_size"),
    (dict(max_time="soon"), TypeError, "max_time"),
    (dict(max_time=0), ValueError, "max_time"),
    (dict(max_time=float("inf")), ValueError, "max_time"),
    (dict(flops_weight=True), TypeError, "flops_weight"),
    (dict(read_write_weight=-1.0), ValueError, "read_write_weight"),
    (dict(flops_weight="x"), TypeError, "flops_weight"),
    (dict(flops_weight=0, read_write_weight=0.0), ValueError, "both be 0"),
    (dict(allow_output_slicing=1), TypeError, "allow_output_slicing"),
    (dict(backend="native"), ValueError, "backend"),
    (dict(backend="auto"), ValueError, "backend"),
    (dict(backend=" b200"), ValueError, "backend"),
])
def test_rejections_match_the_reference_types(kw, exc, msg):
    with pytest.raises(exc, match=msg):
        call(**kw)


def test_unreachable_target_is_reported_before_execution():
    # Every leg of a 1x1 product is an output leg: without output slicing nothing meets target 1.
    with pytest.raises(ValueError, match="unreachable"):
        A.arctn_contract([["a"], ["b"]], ["a", "b"], {"a": 2, "b": 2}, None, target_size=1, backend="b200")


def test_build_info_reports_the_loaded_library():
    # pybind/src/lib.rs:470-493: the loaded extension's identity.
    import os
    import re

    info = A.build_info()
    header = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                               "arctn_b200.h")).read()
    assert info["abi_version"] == int(re.search(r"#define ARCTN_B200_ABI_VERSION (\d+)u", header).group(1))
    assert os.path.basename(info["library"]) == "libarctn_b200.so" and os.path.exists(info["library"])
    assert info["version"] == A.__version__ and info["target_gpu_arch"] == "sm_100a"
    assert info["target_pointer_width"] == 64 and "tf32x3" in info["features"]["precisions"]


def test_the_reference_public_names_for_the_path_exist():
    # pybind/python/arctn/__init__.py:171-183: the names on the contraction path (the planner-only ones --
    # ArcTNOptimizer, arctn_path, arctn_tree, arctn_schedule, arctn_simplify -- are not part of this executor).
    for name in ("__version__", "ArcTNExecutionPlan", "ArcTNCompiledContraction", "PlanValidationError",
                 "arctn_plan", "arctn_contract"):
        assert name in A.__all__ and hasattr(A, name)
    assert issubclass(A.PlanValidationError, ValueError)

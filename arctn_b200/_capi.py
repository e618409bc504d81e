"""ctypes bindings of the C ABI in ``include/arctn_b200.h``.

The shared library is the product path.  Loading fails loudly when it is
missing -- there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libarctn_b200.so")

OK, ERR_INVALID, ERR_CUDA, ERR_UNSUPPORTED, ERR_DEVICE_TIMEOUT, ERR_WORKSPACE = range(6)
F32, F64, C64, C128 = range(4)
PREC_FP32, PREC_TF32X3, PREC_BF16X3, PREC_BF16X6 = 0, 1, 2, 3

u64 = ctypes.c_uint64
u32 = ctypes.c_uint32
u64p = ctypes.POINTER(ctypes.c_uint64)
u32p = ctypes.POINTER(ctypes.c_uint32)
vp = ctypes.c_void_p
vpp = ctypes.POINTER(ctypes.c_void_p)
c_int = ctypes.c_int
c_double = ctypes.c_double


class Network(ctypes.Structure):
    _fields_ = [("n_inputs", u64), ("input_offsets", u64p), ("input_legs", u32p), ("n_output", u64),
                ("output", u32p), ("n_sizes", u64), ("size_legs", u32p), ("size_dims", u64p)]


class StepInfo(ctypes.Structure):
    _fields_ = [("left_slot", u64), ("right_slot", u64), ("result_slot", u64), ("n_left", u64), ("n_right", u64),
                ("n_result", u64), ("left_legs", u32p), ("right_legs", u32p), ("result_legs", u32p),
                ("left_shape", u64p), ("right_shape", u64p), ("result_shape", u64p), ("n_sum_a", u64),
                ("n_sum_b", u64), ("sum_a", u64p), ("sum_b", u64p), ("a_perm", u64p), ("b_perm", u64p),
                ("bt", u64), ("m", u64), ("k", u64), ("n", u64)]


class PrepInfo(ctypes.Structure):
    _fields_ = [("n_input_shape", u64), ("input_shape", u64p), ("n_traces", u64), ("traces", u64p),
                ("n_legs", u64), ("legs", u32p), ("shape", u64p)]


class FinalizeInfo(ctypes.Structure):
    _fields_ = [("slot", u64), ("n_input", u64), ("input_legs", u32p), ("input_shape", u64p), ("n_sum", u64),
                ("sum", u64p), ("n_output", u64), ("perm", u64p), ("output_shape", u64p)]


class ProgramOptions(ctypes.Structure):
    _fields_ = [("dtype", c_int), ("precision", c_int), ("device", c_int), ("use_graph", c_int),
                ("max_slices_per_group", u64), ("workspace_budget", u64), ("slice_begin", u64),
                ("slice_end", u64), ("gradient", c_int), ("tc_k_chunk", u64)]


class GemmChoice(ctypes.Structure):
    _fields_ = [("dtype", c_int), ("precision", c_int), ("phase", c_int), ("a_var", c_int), ("b_var", c_int),
                ("variant", c_int), ("bt", u64), ("m", u64), ("k", u64), ("n", u64)]


# (name, restype, argtypes) for every symbol the header declares.
NETP = ctypes.POINTER(Network)
SIGNATURES = [
    ("arctn_b200_debug_inject_failure", c_int, [c_int, c_int]),
    ("arctn_b200_abi_version", u32, []),
    ("arctn_b200_last_error", ctypes.c_char_p, []),
    ("arctn_b200_simulate_path", c_int, [NETP, u64, u64p, ctypes.POINTER(c_double)]),
    ("arctn_b200_greedy", c_int, [NETP, u64p, u64p]),
    ("arctn_b200_find_slices_to_size", c_int, [NETP, u64, u64p, u64, u32p, u64p, ctypes.POINTER(c_int)]),
    ("arctn_b200_find_slices_with_output", c_int,
     [NETP, u64, u64p, u64, c_int, u32p, u64p, ctypes.POINTER(c_int)]),
    ("arctn_b200_slice_parallel_chunks", u64, [u64, u64]),
    ("arctn_b200_slice_plan_check", c_int, [NETP, u64, u64p, u64, u32p, u64, ctypes.POINTER(c_double),
                                            ctypes.POINTER(c_int)]),
    ("arctn_b200_plan_compile", c_int, [NETP, u64, u64p, ctypes.POINTER(vp)]),
    ("arctn_b200_plan_destroy", None, [vp]),
    ("arctn_b200_plan_n_inputs", u64, [vp]),
    ("arctn_b200_plan_n_steps", u64, [vp]),
    ("arctn_b200_plan_log10_flops", c_double, [vp]),
    ("arctn_b200_plan_log2_peak_size", c_double, [vp]),
    ("arctn_b200_plan_step_info", c_int, [vp, u64, ctypes.POINTER(StepInfo)]),
    ("arctn_b200_plan_prep_info", c_int, [vp, u64, ctypes.POINTER(PrepInfo)]),
    ("arctn_b200_plan_finalize_info", c_int, [vp, ctypes.POINTER(FinalizeInfo)]),
    ("arctn_b200_plan_prep_workspace_size", u64, [vp, c_int, u64]),
    ("arctn_b200_plan_step_workspace_size", u64, [vp, c_int, c_int, u64]),
    ("arctn_b200_plan_finalize_workspace_size", u64, [vp, c_int]),
    ("arctn_b200_plan_prep_execute", c_int, [vp, c_int, u64, vp, vp, vp, u64, vp]),
    ("arctn_b200_plan_step_execute", c_int, [vp, c_int, c_int, u64, vp, vp, vp, vp, u64, vp]),
    ("arctn_b200_plan_finalize_execute", c_int, [vp, c_int, vp, vp, vp, u64, vp]),
    ("arctn_b200_program_create", c_int, [NETP, u64, u64p, u64, u32p, ctypes.POINTER(ProgramOptions),
                                          ctypes.POINTER(vp)]),
    ("arctn_b200_program_create_tuned", c_int, [NETP, u64, u64p, u64, u32p, ctypes.POINTER(ProgramOptions),
                                                ctypes.POINTER(GemmChoice), u64, ctypes.POINTER(vp)]),
    ("arctn_b200_program_gemms", c_int, [vp, ctypes.POINTER(GemmChoice), ctypes.POINTER(c_int), u64, u64p]),
    ("arctn_b200_program_set_tc_chain", c_int, [vp, u64]),
    ("arctn_b200_program_destroy", None, [vp]),
    ("arctn_b200_program_workspace_size", u64, [vp]),
    ("arctn_b200_program_n_slices", u64, [vp]),
    ("arctn_b200_program_slices_per_group", u64, [vp]),
    ("arctn_b200_program_flops", c_double, [vp]),
    ("arctn_b200_program_launches", u64, [vp]),
    ("arctn_b200_program_recomputed_steps", u64, [vp]),
    ("arctn_b200_program_describe", c_int, [vp, ctypes.c_char_p, u64, u64p]),
    ("arctn_b200_batch_create", c_int, [ctypes.POINTER(vp), u64, c_int, ctypes.POINTER(vp)]),
    ("arctn_b200_batch_create_mode", c_int, [ctypes.POINTER(vp), u64, c_int, c_int, ctypes.POINTER(vp)]),
    ("arctn_b200_batch_describe", c_int, [vp, c_int, ctypes.c_char_p, u64, ctypes.POINTER(u64)]),
    ("arctn_b200_batch_wait_selftest", c_int, [vp, ctypes.POINTER(c_int)]),
    ("arctn_b200_batch_destroy", None, [vp]),
    ("arctn_b200_batch_workspace_size", u64, [vp]),
    ("arctn_b200_batch_lanes", u64, [vp]),
    ("arctn_b200_batch_execute", c_int, [vp, ctypes.POINTER(vpp), vpp, vp, u64, vp]),
    ("arctn_b200_batch_gradient", c_int, [vp, ctypes.POINTER(vpp), vpp, ctypes.POINTER(vpp), vpp, vp, u64, vp]),
    ("arctn_b200_batch_device_status", c_int, [vp, vp, vp, ctypes.POINTER(c_int)]),
    ("arctn_b200_program_execute", c_int, [vp, vpp, vp, vp, u64, vp]),
    ("arctn_b200_program_execute_f64out", c_int, [vp, vpp, vp, vp, u64, vp]),
    ("arctn_b200_program_execute_stripped", c_int, [vp, vpp, vp, vp, u64, vp, ctypes.POINTER(c_double)]),
    ("arctn_b200_program_gradient", c_int, [vp, c_int, vpp, vp, vpp, vp, vp, u64, vp]),
    ("arctn_b200_program_device_status", c_int, [vp, vp, vp, ctypes.POINTER(c_int)]),
    ("arctn_b200_program_profile", c_int, [vp, vpp, vp, vp, u64, vp, ctypes.POINTER(ctypes.c_float),
                                           ctypes.POINTER(c_int), ctypes.POINTER(c_double)]),
    ("arctn_b200_program_profile_gradient", c_int, [vp, vpp, vp, vpp, vp, vp, u64, vp,
                                                    ctypes.POINTER(ctypes.c_float), ctypes.POINTER(c_int),
                                                    ctypes.POINTER(c_double)]),
    ("arctn_b200_cgemm_tf32x3_noalloc", c_int, [vp, vp, vp, u64, u64, u64, u64, vp]),
    ("arctn_b200_cgemm_noalloc_status", c_int, [vp, ctypes.POINTER(c_int)]),
    ("arctn_b200_tc_peak", c_int, [c_int, c_int, u64, vp, vp, ctypes.POINTER(c_double)]),
    ("arctn_b200_contract_sliced_host", c_int, [NETP, u64, u64p, u64, u32p, ctypes.POINTER(ProgramOptions), vpp,
                                                vp]),
]

_lib = None


def lib():
    """Load the extension (building it first when this checkout has no build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _build

            _build.build()
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class ArcTNB200Error(ValueError):
    """Raised for every non-zero status; ``code`` is the ABI status."""

    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


def check(rc, context=""):
    if rc != OK:
        msg = lib().arctn_b200_last_error().decode(errors="replace")
        raise ArcTNB200Error(rc, f"{context}: {msg}" if context else msg)


class NetworkArgs:
    """Keeps the flat arrays of one network alive while a call uses them."""

    def __init__(self, inputs, output, size_dict):
        import numpy as np

        self.inputs = [[int(l) for l in t] for t in inputs]
        self.output = [int(l) for l in output]
        self.size_dict = {int(k): int(v) for k, v in size_dict.items()}
        offs = [0]
        for t in self.inputs:
            offs.append(offs[-1] + len(t))
        self._offs = np.asarray(offs, dtype=np.uint64)
        self._legs = np.asarray([l for t in self.inputs for l in t] or [0], dtype=np.uint32)
        self._out = np.asarray(self.output or [0], dtype=np.uint32)
        keys = sorted(self.size_dict)
        self._sl = np.asarray(keys or [0], dtype=np.uint32)
        self._sd = np.asarray([self.size_dict[k] for k in keys] or [0], dtype=np.uint64)
        self.struct = Network(len(self.inputs), self._offs.ctypes.data_as(u64p), self._legs.ctypes.data_as(u32p),
                              len(self.output), self._out.ctypes.data_as(u32p), len(keys),
                              self._sl.ctypes.data_as(u32p), self._sd.ctypes.data_as(u64p))

    @property
    def ptr(self):
        return ctypes.byref(self.struct)


def path_array(path):
    import numpy as np

    arr = np.asarray([int(x) for p in path for x in p] or [0], dtype=np.uint64)
    return len(path), arr

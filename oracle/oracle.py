"""ctypes wrapper around the C++ oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (``oracle/arctn_oracle.cpp``) restates the reference ArcTN CPU
executor.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may import this module, and only as the checker or the
timed CPU baseline -- never as the product path.

A network is passed as ``(inputs, output, size_dict)`` with integer leg ids,
exactly as the reference Python binding's ``CompiledContraction.compile``
(``pybind/src/lib.rs:384-398``) receives it.
"""

from __future__ import annotations

import ctypes
import json
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "liboracle.so")

DTYPE_CODES = {
    np.dtype(np.float32): 0,
    np.dtype(np.float64): 1,
    np.dtype(np.complex64): 2,
    np.dtype(np.complex128): 3,
}

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_NET_ARGS = [ctypes.c_uint64, _u64p, _u32p, ctypes.c_uint64, _u32p, ctypes.c_uint64, _u32p, _u64p]


def build() -> str:
    """Compile the oracle library with its Makefile (idempotent)."""
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run(["make", "-s", "-C", _HERE, f"CXX={cxx}"], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_plan_json.argtypes = _NET_ARGS + [ctypes.c_uint64, _u64p, ctypes.POINTER(ctypes.c_char_p)]
        L.oracle_simulate_path.argtypes = _NET_ARGS + [ctypes.c_uint64, _u64p, ctypes.POINTER(ctypes.c_double)]
        L.oracle_execute.argtypes = _NET_ARGS + [
            ctypes.c_uint64, _u64p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_int,
            ctypes.POINTER(ctypes.c_double)]
        L.oracle_contract_sliced.argtypes = _NET_ARGS + [
            ctypes.c_uint64, _u64p, ctypes.c_uint64, _u32p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
            ctypes.c_void_p, ctypes.c_int]
        L.oracle_contract_slice_range.argtypes = _NET_ARGS + [
            ctypes.c_uint64, _u64p, ctypes.c_uint64, _u32p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
            ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_int]
        L.oracle_naive_einsum.argtypes = _NET_ARGS + [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]
        L.oracle_greedy.argtypes = _NET_ARGS + [_u64p, _u64p]
        L.oracle_find_slices_to_size.argtypes = _NET_ARGS + [
            ctypes.c_uint64, _u64p, ctypes.c_uint64, _u32p, _u64p, ctypes.POINTER(ctypes.c_int)]
        L.oracle_find_slices_with_output.argtypes = _NET_ARGS + [
            ctypes.c_uint64, _u64p, ctypes.c_uint64, ctypes.c_int, _u32p, _u64p, ctypes.POINTER(ctypes.c_int)]
        L.oracle_slice_parallel_chunks.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.oracle_slice_parallel_chunks.restype = ctypes.c_uint64
        _lib = L
    return _lib


class OracleError(ValueError):
    pass


def _check(rc):
    if rc != 0:
        raise OracleError(lib().oracle_last_error().decode())


class _Net:
    """Flat CSR form of ``(inputs, output, size_dict)`` kept alive for a call."""

    def __init__(self, inputs, output, size_dict):
        self.inputs = [list(map(int, t)) for t in inputs]
        self.output = list(map(int, output))
        self.size_dict = {int(k): int(v) for k, v in size_dict.items()}
        offs = [0]
        for t in self.inputs:
            offs.append(offs[-1] + len(t))
        self.offs = np.asarray(offs, dtype=np.uint64)
        self.legs = np.asarray([l for t in self.inputs for l in t] or [0], dtype=np.uint32)
        self.out = np.asarray(self.output or [0], dtype=np.uint32)
        keys = sorted(self.size_dict)
        self.sl = np.asarray(keys or [0], dtype=np.uint32)
        self.sd = np.asarray([self.size_dict[k] for k in keys] or [0], dtype=np.uint64)
        self.n_sizes = len(keys)

    def args(self):
        return [len(self.inputs), self.offs.ctypes.data_as(_u64p), self.legs.ctypes.data_as(_u32p),
                len(self.output), self.out.ctypes.data_as(_u32p), self.n_sizes,
                self.sl.ctypes.data_as(_u32p), self.sd.ctypes.data_as(_u64p)]

    def output_shape(self):
        return tuple(self.size_dict[l] for l in self.output)


def _path_arr(path):
    arr = np.asarray([x for p in path for x in p] or [0], dtype=np.uint64)
    return len(path), arr


def _inputs(net: _Net, arrays):
    arrays = [np.array(a, order="C", copy=None) for a in arrays]  # keeps 0-d shapes
    dt = arrays[0].dtype
    if dt not in DTYPE_CODES:
        raise OracleError(f"unsupported dtype {dt}")
    if any(a.dtype != dt for a in arrays):
        raise OracleError("mixed dtypes")
    ptrs = (ctypes.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
    return arrays, dt, ptrs


def plan_json(inputs, output, size_dict, ssa_path):
    net = _Net(inputs, output, size_dict)
    n, p = _path_arr(ssa_path)
    out = ctypes.c_char_p()
    _check(lib().oracle_plan_json(*net.args(), n, p.ctypes.data_as(_u64p), ctypes.byref(out)))
    return json.loads(out.value.decode())


STAT_KEYS = ("log10_flops", "log2_max_size", "log2_max_contraction_size", "log2_total_size",
             "log2_read_write", "log2_peak_size")


def simulate_path(inputs, output, size_dict, ssa_path):
    net = _Net(inputs, output, size_dict)
    n, p = _path_arr(ssa_path)
    st = (ctypes.c_double * 6)()
    _check(lib().oracle_simulate_path(*net.args(), n, p.ctypes.data_as(_u64p), st))
    return dict(zip(STAT_KEYS, list(st)))


def execute(inputs, output, size_dict, ssa_path, arrays, strip=False):
    """Compiled execution; returns the result (and the log10 exponent when ``strip``)."""
    net = _Net(inputs, output, size_dict)
    n, p = _path_arr(ssa_path)
    arrays, dt, ptrs = _inputs(net, arrays)
    res = np.zeros(net.output_shape(), dtype=dt)
    e = ctypes.c_double(0.0)
    _check(lib().oracle_execute(*net.args(), n, p.ctypes.data_as(_u64p), DTYPE_CODES[dt], ptrs,
                                res.ctypes.data, 1 if strip else 0, ctypes.byref(e)))
    return (res, e.value) if strip else res


def contract_sliced(inputs, output, size_dict, ssa_path, sliced_legs, arrays, threads=1):
    net = _Net(inputs, output, size_dict)
    n, p = _path_arr(ssa_path)
    arrays, dt, ptrs = _inputs(net, arrays)
    sl = np.asarray(list(sliced_legs) or [0], dtype=np.uint32)
    res = np.zeros(net.output_shape(), dtype=dt)
    _check(lib().oracle_contract_sliced(*net.args(), n, p.ctypes.data_as(_u64p), len(sliced_legs),
                                        sl.ctypes.data_as(_u32p), DTYPE_CODES[dt], ptrs, res.ctypes.data,
                                        int(threads)))
    return res


def contract_slice_range(inputs, output, size_dict, ssa_path, sliced_legs, begin, end, arrays, threads=1):
    """Slices [begin, end) summed into a zeroed full output (the reference's tnmpi contract_slice_range)."""
    net = _Net(inputs, output, size_dict)
    n, p = _path_arr(ssa_path)
    arrays, dt, ptrs = _inputs(net, arrays)
    sl = np.asarray(list(sliced_legs) or [0], dtype=np.uint32)
    res = np.zeros(net.output_shape(), dtype=dt)
    _check(lib().oracle_contract_slice_range(*net.args(), n, p.ctypes.data_as(_u64p), len(sliced_legs),
                                             sl.ctypes.data_as(_u32p), int(begin), int(end), DTYPE_CODES[dt], ptrs,
                                             res.ctypes.data, int(threads)))
    return res


def naive_einsum(inputs, output, size_dict, arrays):
    net = _Net(inputs, output, size_dict)
    arrays, dt, ptrs = _inputs(net, arrays)
    res = np.zeros(net.output_shape(), dtype=dt)
    _check(lib().oracle_naive_einsum(*net.args(), DTYPE_CODES[dt], ptrs, res.ctypes.data))
    return res


def greedy(inputs, output, size_dict):
    net = _Net(inputs, output, size_dict)
    buf = np.zeros(2 * max(1, len(net.inputs)), dtype=np.uint64)
    ns = ctypes.c_uint64(0)
    _check(lib().oracle_greedy(*net.args(), buf.ctypes.data_as(_u64p), ctypes.byref(ns)))
    return [(int(buf[2 * s]), int(buf[2 * s + 1])) for s in range(ns.value)]


def find_slices_to_size(inputs, output, size_dict, ssa_path, target_size, allow_output_slicing=False):
    """Returns the sliced legs, or ``None`` where the reference returns ``None``.  ``allow_output_slicing``
    lets output legs be chosen too (src/slice.rs:254-289)."""
    net = _Net(inputs, output, size_dict)
    n, p = _path_arr(ssa_path)
    buf = np.zeros(max(1, net.n_sizes), dtype=np.uint32)
    nl = ctypes.c_uint64(0)
    found = ctypes.c_int(0)
    _check(lib().oracle_find_slices_with_output(*net.args(), n, p.ctypes.data_as(_u64p), int(target_size),
                                                1 if allow_output_slicing else 0, buf.ctypes.data_as(_u32p),
                                                ctypes.byref(nl), ctypes.byref(found)))
    return [int(x) for x in buf[: nl.value]] if found.value else None


def slice_parallel_chunks(n_slices, out_numel):
    return int(lib().oracle_slice_parallel_chunks(int(n_slices), int(out_numel)))


def promote(arrays):
    """FP64 oracle inputs: f32 -> f64, c64 -> c128 (the ``tnexec --check`` promotion)."""
    out = []
    for a in arrays:
        a = np.asarray(a)
        out.append(a.astype(np.complex128 if np.iscomplexobj(a) else np.float64))
    return out

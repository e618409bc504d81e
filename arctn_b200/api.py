"""Python surface of the B200 executor, mirroring ArcTN's execution entry points.

Reference surfaces mirrored (paths inside the ArcTN repository):

* ``CompiledContraction.compile(inputs, output, size_dict, *, ssa_path)`` /
  ``.execute(arrays)`` / ``.stats()`` -- ``pybind/src/lib.rs:355-454``;
  the stage API ``input_preps()`` / ``pair_steps()`` / ``finalize()`` with
  their accessors -- ``src/compiled.rs:33-250``.
* ``contract_sliced(inputs, output, size_dict, arrays, sliced_legs, path=None,
  ssa_path=None)`` -- ``pybind/src/lib.rs:667-765``.
* ``ArcTNCompiledContraction.compile(..., backend=)`` and
  ``arctn_contract(..., backend=)`` -- ``pybind/python/arctn/__init__.py:749-1072``,
  with ``backend="b200"`` selecting this executor explicitly.

Arrays may be NumPy arrays (copied to the GPU and the result copied back) or
CUDA ``torch`` tensors (used in place; the result stays on the device).  Every
error is raised as ``ValueError`` before anything is launched, as the
reference raises ``ValueError`` from its preflight (``pybind/src/lib.rs:246-330``).
"""

from __future__ import annotations

import ctypes
import math
import operator
import sys
import threading
import time

import numpy as np

from . import _capi as C

_NP_CODES = {np.dtype(np.float32): C.F32, np.dtype(np.float64): C.F64, np.dtype(np.complex64): C.C64,
             np.dtype(np.complex128): C.C128}
_PRECISIONS = {"fp32": C.PREC_FP32, "tf32x3": C.PREC_TF32X3, "bf16x3": C.PREC_BF16X3, "bf16x6": C.PREC_BF16X6}


def _torch():
    import torch

    return torch


def _torch_code(dtype):
    torch = _torch()
    table = {torch.float32: C.F32, torch.float64: C.F64, torch.complex64: C.C64, torch.complex128: C.C128}
    if dtype not in table:
        raise ValueError(f"dtype {dtype} is not supported; use float32, float64, complex64 or complex128")
    return table[dtype]


def _torch_dtype(code, wide=False):
    torch = _torch()
    if wide:
        return torch.complex128 if code in (C.C64, C.C128) else torch.float64
    return {C.F32: torch.float32, C.F64: torch.float64, C.C64: torch.complex64, C.C128: torch.complex128}[code]


def _precision(p):
    if isinstance(p, int):
        return p
    if p not in _PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}, got {p!r}")
    return _PRECISIONS[p]


def _is_torch(x):
    try:
        import torch
    except ImportError:  # pragma: no cover
        return False
    return isinstance(x, torch.Tensor)


def _expected_shapes(inputs, size_dict):
    return [tuple(int(size_dict[l]) for l in t) for t in inputs]


def _preflight(arrays, inputs, size_dict, context, shapes=None):
    """Validate count, dtype, layout and every shape before any copy (pybind/src/lib.rs:246-330)."""
    try:
        arrays = list(arrays)
    except TypeError as exc:
        raise TypeError("arrays must be a sequence of tensors") from exc
    if len(arrays) != len(inputs):
        raise ValueError(f"{context}: {len(arrays)} arrays given for {len(inputs)} input tensors")
    if not arrays:
        raise ValueError(f"{context}: arrays is empty")
    shapes = shapes if shapes is not None else _expected_shapes(inputs, size_dict)
    torch_mode = _is_torch(arrays[0])
    # Fast path: NumPy arrays of one supported dtype whose shapes all match (the checks below, in one pass).
    if not torch_mode and all(type(a) is np.ndarray for a in arrays):
        dt = arrays[0].dtype
        if dt in _NP_CODES and all(a.dtype == dt and a.shape == sh for a, sh in zip(arrays, shapes)):
            return arrays, _NP_CODES[dt], False
    code = None
    for i, (a, shape) in enumerate(zip(arrays, shapes)):
        if torch_mode != _is_torch(a):
            raise ValueError(f"{context}: arrays[{i}] mixes torch tensors and NumPy arrays")
        if torch_mode:
            c = _torch_code(a.dtype)
            if not a.is_cuda:
                raise ValueError(f"{context}: arrays[{i}] is a CPU torch tensor; pass CUDA tensors or NumPy arrays")
            if not a.is_contiguous():
                raise ValueError(f"{context}: arrays[{i}] must be contiguous (call .contiguous())")
        else:
            a = np.asarray(a)
            if a.dtype not in _NP_CODES:
                raise ValueError(f"{context}: arrays[{i}] dtype {a.dtype} is not supported; "
                                 "use float32, float64, complex64 or complex128")
            c = _NP_CODES[a.dtype]
        if code is None:
            code = c
        elif c != code:
            raise ValueError(f"{context}: arrays[{i}] dtype differs from the first tensor's")
        if tuple(int(d) for d in a.shape) != shape:
            raise ValueError(f"{context}: arrays[{i}] shape {tuple(a.shape)} does not match the network's {shape} "
                             "(invalid input layout)")
    return arrays, code, torch_mode


class _DeviceCall:
    """Moves NumPy inputs to the GPU (via pinned staging) or passes CUDA tensors through."""

    def __init__(self, arrays, torch_mode, device=None, stream=None, reuse=None):
        """``stream``: where the staging copy runs (the caller's execution stream; default: current).
        ``reuse``: a device byte buffer from an earlier call on the same stream to copy the inputs into."""
        torch = _torch()
        self._views = None
        if torch_mode:
            self.device = arrays[0].device
            for a in arrays:
                if a.device != self.device:
                    raise ValueError("all arrays must live on one CUDA device")
            self._views = list(arrays)
            ptrs = [t.data_ptr() for t in arrays]
        else:
            if not torch.cuda.is_available():
                raise ValueError("the B200 executor needs a CUDA device; none is visible")
            self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
            # One pinned staging buffer and one host-to-device copy for all inputs (a network can have hundreds
            # of small tensors); input i sits 256-byte aligned at offset offs[i] of the device copy.
            arrs = [np.array(a, order="C", copy=None) for a in arrays]
            offs, total = [], 0
            for a in arrs:
                offs.append(total)
                total += (a.nbytes + 255) // 256 * 256
            host = torch.empty(max(total, 1), dtype=torch.uint8, pin_memory=True)
            hv = host.numpy()
            for a, o in zip(arrs, offs):
                hv[o:o + a.nbytes] = a.reshape(-1).view(np.uint8)
            with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream(self.device)):
                if reuse is not None and reuse.device == self.device and reuse.numel() >= host.numel():
                    reuse[:host.numel()].copy_(host, non_blocking=True)
                    self._dev = reuse
                else:
                    self._dev = host.to(self.device, non_blocking=True)
            self._layout = [(o, a.nbytes, a.dtype, a.shape) for a, o in zip(arrs, offs)]
            base = self._dev.data_ptr()
            ptrs = [base + o for o in offs]
        self.stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        self.ptrs = (ctypes.c_void_p * len(ptrs))(*ptrs)

    @property
    def tensors(self):
        """The inputs as CUDA tensors (views of the staged copy for NumPy inputs), built on first use."""
        if self._views is None:
            torch = _torch()
            kinds = {}
            self._views = []
            for o, nb, dt, shape in self._layout:
                if dt not in kinds:
                    kinds[dt] = torch.from_numpy(np.empty(0, dt)).dtype
                self._views.append(self._dev[o:o + nb].view(kinds[dt]).view(shape))
        return self._views

    def empty(self, shape, dtype):
        return _torch().empty(shape, dtype=dtype, device=self.device)

    def workspace(self, nbytes):
        return _torch().empty(max(int(nbytes), 1), dtype=_torch().uint8, device=self.device)


def _to_output(t, torch_mode, stream=None):
    """CUDA tensors are returned as they are; NumPy callers get a host copy made on ``stream`` (the stream the
    result was computed on), after the work queued there."""
    if torch_mode:
        return t
    if stream is None:
        return t.cpu().numpy()
    with _torch().cuda.stream(stream):
        return t.cpu().numpy()


# ---------------------------------------------------------------------------- planning support


def simulate_path(inputs, output, size_dict, ssa_path):
    """Path metrics (``simulate_path_full``, src/path.rs:239-434) as a dict."""
    net = C.NetworkArgs(inputs, output, size_dict)
    n, p = C.path_array(ssa_path)
    st = (ctypes.c_double * 6)()
    C.check(C.lib().arctn_b200_simulate_path(net.ptr, n, p.ctypes.data_as(C.u64p), st), "invalid path")
    keys = ("log10_flops", "log2_max_size", "log2_max_contraction_size", "log2_total_size", "log2_read_write",
            "log2_peak_size")
    return dict(zip(keys, list(st)))


def greedy(inputs, output, size_dict):
    """Deterministic greedy SSA path (src/paths/greedy.rs:307-320)."""
    net = C.NetworkArgs(inputs, output, size_dict)
    buf = np.zeros(2 * max(1, len(net.inputs)), dtype=np.uint64)
    ns = C.u64(0)
    C.check(C.lib().arctn_b200_greedy(net.ptr, buf.ctypes.data_as(C.u64p), ctypes.byref(ns)), "invalid network")
    return [(int(buf[2 * s]), int(buf[2 * s + 1])) for s in range(ns.value)]


def find_slices_to_size(inputs, output, size_dict, ssa_path, target_size, allow_output_slicing=False):
    """Sliced legs meeting ``target_size`` elements per intermediate, or None (src/slice.rs:209-215).  With
    ``allow_output_slicing`` output legs may be chosen too, the reference's opt-in output-index slicing
    (src/slice.rs:254-289)."""
    net = C.NetworkArgs(inputs, output, size_dict)
    n, p = C.path_array(ssa_path)
    buf = np.zeros(max(1, len(net.size_dict)), dtype=np.uint32)
    nl = C.u64(0)
    found = ctypes.c_int(0)
    if allow_output_slicing:
        rc = C.lib().arctn_b200_find_slices_with_output(net.ptr, n, p.ctypes.data_as(C.u64p), int(target_size), 1,
                                                        buf.ctypes.data_as(C.u32p), ctypes.byref(nl),
                                                        ctypes.byref(found))
    else:
        rc = C.lib().arctn_b200_find_slices_to_size(net.ptr, n, p.ctypes.data_as(C.u64p), int(target_size),
                                                    buf.ctypes.data_as(C.u32p), ctypes.byref(nl),
                                                    ctypes.byref(found))
    C.check(rc, "slice search")
    return [int(x) for x in buf[: nl.value]] if found.value else None


def build_info():
    """Identity of the loaded library, the counterpart of the reference's ``build_info`` (pybind/src/lib.rs:
    470-493): the package version, the C-ABI version of ``libarctn_b200.so``, where it was loaded from, the GPU
    architecture it was compiled for, the host platform and the executor's features.  Host-only."""
    import platform

    return {"version": __import__("arctn_b200").__version__, "abi_version": int(C.lib().arctn_b200_abi_version()),
            "library": C.lib()._name, "target_gpu_arch": "sm_100a", "target_arch": platform.machine(),
            "target_os": platform.system().lower(), "target_pointer_width": ctypes.sizeof(ctypes.c_void_p) * 8,
            "features": {"dtypes": ["f32", "f64", "complex64", "complex128"],
                         "precisions": ["fp32", "tf32x3", "bf16x3", "bf16x6"], "tensor_cores": "tcgen05",
                         "adjoint": True, "output_slicing": True, "batch": True, "autotuner": True}}


def slice_range(count, ranks, rank):
    """Contiguous slice range [begin, end) of one rank (src/bin/tnmpi.rs:278-284); empty when ranks > count."""
    if ranks < 1 or not 0 <= rank < ranks:
        raise ValueError(f"rank {rank} outside [0, {ranks})")
    chunk, extra = divmod(int(count), int(ranks))
    begin = rank * chunk + min(rank, extra)
    return begin, begin + chunk + (1 if rank < extra else 0)


def slice_parallel_chunks(n_slices, out_numel):
    """Deterministic chunk count of the sliced sum (src/slice.rs:893-905)."""
    return int(C.lib().arctn_b200_slice_parallel_chunks(int(n_slices), int(out_numel)))


# ---------------------------------------------------------------------------- programs


def tensor_pipe_peak(kind="tf32", n=256, iters=1 << 16, device=None, repeats=3):
    """Measured dense tensor-pipe rate of a GPU in TFLOP/s (``arctn_b200_tc_peak``): tcgen05 MMAs with M = 128,
    N = ``n`` (128 or 256) over operands resident in shared memory, ``kind`` "tf32" or "bf16"; or
    "tf32_gemm_stream" (n = 128): the split-TF32 GEMM's own MMA sequence over operands streaming through its
    three-stage ring layout, every operand 1.0; "tf32_gemm_stream_random": the same over random TF32 hi / lo
    operands; "bf16x6_gemm_stream_random": the three-piece split-BF16 GEMM's 24-MMA sequence over random BF16
    pieces (BF16 MMA work); "tf32_3m_stream_random": a 3M split-TF32 product's 9 MMAs per K step over random
    operands (TF32 MMA work).  Best of ``repeats`` launches after one warm-up."""
    torch = _torch()
    code = {"tf32": 0, "bf16": 1, "tf32_gemm_stream": 2, "tf32_gemm_stream_random": 3,
            "bf16x6_gemm_stream_random": 4, "tf32_3m_stream_random": 5}[kind]
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    with torch.cuda.device(dev):
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev)
        best = 0.0
        for r in range(repeats + 1):
            out = ctypes.c_double(0.0)
            C.check(C.lib().arctn_b200_tc_peak(code, int(n), int(iters), status.data_ptr(), stream.cuda_stream,
                                               ctypes.byref(out)), "tensor-pipe peak")
            if r:
                best = max(best, out.value)
        if int(status.item()) != 0:
            raise C.ArcTNB200Error(C.ERR_DEVICE_TIMEOUT, "tensor-pipe peak probe: a bounded wait expired")
    return best


class SlicedProgram:
    """A network + SSA path + sliced legs bound to a dtype, precision and GPU.

    ``execute`` runs all slices (slices batched, slice-invariant subtrees run
    once, FP64 cross-slice sum in the reference's chunk order) and returns the
    full output, like ``contract_network_sliced`` (src/slice.rs:960-1173).
    """

    def __init__(self, inputs, output, size_dict, ssa_path, sliced_legs=(), *, dtype="complex64",
                 precision="fp32", device=None, use_graph=True, max_slices_per_group=0, workspace_budget=0,
                 slice_begin=0, slice_end=0, gradient=False, tc_k_chunk=0, tuning=None, tc_chain_k=None):
        torch = _torch()
        self.inputs = [[int(l) for l in t] for t in inputs]
        self.output = [int(l) for l in output]
        self.size_dict = {int(k): int(v) for k, v in size_dict.items()}
        self.ssa_path = [(int(a), int(b)) for a, b in ssa_path]
        self.sliced_legs = [int(l) for l in sliced_legs]
        if isinstance(dtype, int):
            self.code = dtype
        else:
            self.code = _NP_CODES.get(np.dtype(dtype)) if not _is_torch_dtype(dtype) else _torch_code(dtype)
            if self.code is None:
                raise ValueError(f"unsupported dtype {dtype}")
        self.precision = _precision(precision)
        if device is None:
            device = torch.cuda.current_device() if torch.cuda.is_available() else 0
        self.device = int(device)
        net = C.NetworkArgs(self.inputs, self.output, self.size_dict)
        n, p = C.path_array(self.ssa_path)
        sl = np.asarray(self.sliced_legs or [0], dtype=np.uint32)
        self.has_gradient = bool(gradient)
        opts = C.ProgramOptions(self.code, self.precision, self.device, 1 if use_graph else 0,
                                int(max_slices_per_group), int(workspace_budget), int(slice_begin), int(slice_end),
                                1 if gradient else 0, int(tc_k_chunk))
        h = C.vp()
        entries = tuning.entries_for(self.code, self.precision) if tuning is not None else []
        self.tuning = tuning
        if entries:
            table = (C.GemmChoice * len(entries))(*[C.GemmChoice(*e) for e in entries])
            C.check(C.lib().arctn_b200_program_create_tuned(net.ptr, n, p.ctypes.data_as(C.u64p),
                                                            len(self.sliced_legs), sl.ctypes.data_as(C.u32p),
                                                            ctypes.byref(opts), table, len(entries),
                                                            ctypes.byref(h)), "sliced contraction failed")
        else:
            C.check(C.lib().arctn_b200_program_create(net.ptr, n, p.ctypes.data_as(C.u64p), len(self.sliced_legs),
                                                      sl.ctypes.data_as(C.u32p), ctypes.byref(opts),
                                                      ctypes.byref(h)), "sliced contraction failed")
        self._h = h
        self._lock = threading.Lock()
        L = C.lib()
        if tc_chain_k is not None:  # K per TMEM chain of the split-TF32 GEMMs (default 64; gradient programs 32)
            C.check(L.arctn_b200_program_set_tc_chain(h, int(tc_chain_k)), "sliced contraction failed")
        self.workspace_bytes = int(L.arctn_b200_program_workspace_size(h))
        self.n_slices = int(L.arctn_b200_program_n_slices(h))
        self.slices_per_group = int(L.arctn_b200_program_slices_per_group(h))
        self.flops = float(L.arctn_b200_program_flops(h))
        self.launches = int(L.arctn_b200_program_launches(h))
        self.recomputed_steps = int(L.arctn_b200_program_recomputed_steps(h))
        self.output_shape = tuple(self.size_dict[l] for l in self.output)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                C.lib().arctn_b200_program_destroy(h)
            except Exception:  # interpreter shutdown: the module globals may already be gone
                pass
            self._h = None

    def describe(self):
        """Launch sequence and workspace layout as a dict (host-only; works without a GPU)."""
        import json

        need = C.u64(0)
        C.check(C.lib().arctn_b200_program_describe(self._h, None, 0, ctypes.byref(need)), "describe")
        buf = ctypes.create_string_buffer(int(need.value))
        C.check(C.lib().arctn_b200_program_describe(self._h, buf, need.value, ctypes.byref(need)), "describe")
        return json.loads(buf.value.decode())

    def gemms(self):
        """The program's GEMMs in launch order (a per-slice GEMM once per slice group), as dicts: the shape key
        (dtype, precision, phase, a_var, b_var, bt, m, k, n), the variant that runs and whether a tuning
        table chose it.  Host-only."""
        from .tuning import VARIANT_NAMES

        n = C.u64(0)
        C.check(C.lib().arctn_b200_program_gemms(self._h, None, None, 0, ctypes.byref(n)), "gemms")
        out = (C.GemmChoice * max(1, n.value))()
        tuned = (ctypes.c_int * max(1, n.value))()
        C.check(C.lib().arctn_b200_program_gemms(self._h, out, tuned, n.value, ctypes.byref(n)), "gemms")
        return [dict(dtype=e.dtype, precision=e.precision, phase=e.phase, a_var=e.a_var, b_var=e.b_var, bt=e.bt,
                     m=e.m, k=e.k, n=e.n, variant=VARIANT_NAMES[e.variant], tuned=bool(tuned[i]))
                for i, e in enumerate(out[:n.value])]

    def _shapes(self):
        """The input shapes the network expects, computed once."""
        if getattr(self, "_shape_cache", None) is None:
            self._shape_cache = _expected_shapes(self.inputs, self.size_dict)
        return self._shape_cache

    def execute(self, arrays, *, f64_out=False, workspace=None, stream=None, out=None):
        """Full output of the contraction.  ``out`` (a CUDA tensor of the output's shape and dtype -- the
        wide dtype with ``f64_out``) receives it in place, which keeps a captured graph's pointers fixed."""
        arrays, code, torch_mode = _preflight(arrays, self.inputs, self.size_dict, "sliced contraction failed",
                                              self._shapes())
        if code != self.code:
            raise ValueError("sliced contraction failed: arrays dtype differs from the program's dtype")
        torch = _torch()
        dev = arrays[0].device if torch_mode else torch.device(
            "cuda", torch.cuda.current_device() if self.device is None else self.device)
        st = stream if stream is not None else torch.cuda.current_stream(dev)
        # Buffers of the previous call on the same stream are reused in stream order (inputs staged into the
        # same device buffer, the same workspace and scalar-or-array output): the pointers stay fixed, so the
        # captured graph replays without a new capture.
        prev = getattr(self, "_reuse", None)
        prev = prev if prev is not None and prev["stream"] == st.cuda_stream else None
        sig = None if torch_mode else tuple((a.shape, a.dtype.str) for a in arrays)
        call = _DeviceCall(arrays, torch_mode, self.device, stream=st,
                           reuse=prev["stage"] if prev is not None and sig is not None and prev["sig"] == sig else None)
        want = _torch_dtype(code, wide=f64_out)
        own_out = out is None
        if out is not None:
            if tuple(out.shape) != tuple(self.output_shape) or out.dtype != want or not out.is_contiguous():
                raise ValueError(f"sliced contraction failed: out must be a contiguous {want} tensor of shape "
                                 f"{tuple(self.output_shape)}")
        elif not torch_mode and prev is not None and prev["out"] is not None and prev["out"].dtype == want:
            out = prev["out"]  # NumPy callers get a host copy, so the device buffer is free again
        else:
            out = call.empty(self.output_shape, want)
        if workspace is not None:
            ws = workspace
        elif prev is not None and prev["ws"] is not None and prev["ws"].numel() >= self.workspace_bytes:
            ws = prev["ws"]
        else:
            ws = call.workspace(self.workspace_bytes)
        fn = C.lib().arctn_b200_program_execute_f64out if f64_out else C.lib().arctn_b200_program_execute
        with torch.cuda.device(call.device):
            C.check(fn(self._h, call.ptrs, out.data_ptr(), ws.data_ptr(), ws.numel(), st.cuda_stream),
                    "sliced contraction failed")
        self._keep = (call, ws)  # keep device buffers alive until the next call on this stream
        self._reuse = {"stream": st.cuda_stream, "sig": sig, "stage": None if torch_mode else call._dev,
                       "ws": ws if workspace is None else (prev["ws"] if prev is not None else None),
                       "out": out if (own_out and not torch_mode) else None}
        return _to_output(out, torch_mode, st)

    def bind(self, arrays, out, workspace, stream=None, *, f64_out=False):
        """A zero-argument callable that re-runs this program on fixed CUDA buffers.

        All validation and pointer marshalling happen here, once; each call is one C-ABI call
        (graph replay when ``use_graph``), for latency-bound callers that execute the same buffers
        repeatedly.  The caller keeps ``arrays``, ``out`` and ``workspace`` alive.
        """
        arrays, code, torch_mode = _preflight(arrays, self.inputs, self.size_dict, "bind failed",
                                              self._shapes())
        if not torch_mode:
            raise ValueError("bind failed: arrays must be CUDA torch tensors")
        if code != self.code:
            raise ValueError("bind failed: arrays dtype differs from the program's dtype")
        want = _torch_dtype(code, wide=f64_out)
        if tuple(out.shape) != tuple(self.output_shape) or out.dtype != want or not out.is_contiguous():
            raise ValueError(f"bind failed: out must be a contiguous {want} tensor of shape {tuple(self.output_shape)}")
        if workspace.numel() < self.workspace_bytes:
            raise ValueError("bind failed: workspace is smaller than workspace_bytes")
        torch = _torch()
        st = stream if stream is not None else torch.cuda.current_stream(arrays[0].device)
        ptrs = (ctypes.c_void_p * len(arrays))(*[t.data_ptr() for t in arrays])
        fn = C.lib().arctn_b200_program_execute_f64out if f64_out else C.lib().arctn_b200_program_execute
        h, o, w, nb, s = self._h, out.data_ptr(), workspace.data_ptr(), workspace.numel(), st.cuda_stream

        def launch():
            rc = fn(h, ptrs, o, w, nb, s)
            if rc:
                C.check(rc, "execute failed")

        launch.keep = (arrays, out, workspace, ptrs, self)
        return launch

    def gradient(self, arrays, grad_output=None, *, part=0, workspace=None, output=None, stream=None):
        """Adjoint sweep (programs built with ``gradient=True``).

        Returns ``(output, [dL/d conj(T_i)])`` for part 0 (forward + reverse), ``(output, None)`` for
        part 1 (forward, intermediates kept in ``workspace``) and ``(None, grads)`` for part 2 (reverse
        only, with the workspace of a preceding part-1 call).  ``grad_output`` defaults to ones.
        """
        if not self.has_gradient:
            raise ValueError("program was built without gradient=True")
        arrays, code, torch_mode = _preflight(arrays, self.inputs, self.size_dict, "gradient failed",
                                              self._shapes())
        torch = _torch()
        call = _DeviceCall(arrays, torch_mode, self.device)
        out = output if output is not None else call.empty(self.output_shape, _torch_dtype(code))
        ws = workspace if workspace is not None else call.workspace(self.workspace_bytes)
        st = stream if stream is not None else call.stream
        grads, gptr, g = None, None, None
        if part != 1:
            if grad_output is None:
                g = torch.ones(self.output_shape, dtype=_torch_dtype(code), device=call.device)
            elif _is_torch(grad_output):
                g = grad_output.to(call.device, _torch_dtype(code)).contiguous()
            else:
                np_dt = {C.F32: np.float32, C.F64: np.float64, C.C64: np.complex64, C.C128: np.complex128}[code]
                g = torch.from_numpy(np.array(grad_output, dtype=np_dt, order="C")).to(call.device)
            grads = [torch.empty_like(t) for t in call.tensors]
            gptr = (ctypes.c_void_p * len(grads))(*[t.data_ptr() for t in grads])
        with torch.cuda.device(call.device):
            C.check(C.lib().arctn_b200_program_gradient(self._h, int(part), call.ptrs,
                                                        g.data_ptr() if g is not None else None, gptr,
                                                        out.data_ptr() if part != 2 else None, ws.data_ptr(),
                                                        ws.numel(), st.cuda_stream), "gradient failed")
        self._keep = (call, ws, g)
        if torch_mode:
            return (out if part != 2 else None), grads
        return (_to_output(out, False) if part != 2 else None), ([_to_output(x, False) for x in grads]
                                                                 if grads is not None else None)

    def device_status(self, workspace, stream=None):
        """Synchronise and return 0, or raise when a bounded device-side wait expired in the last execute."""
        torch = _torch()
        st = stream if stream is not None else torch.cuda.current_stream(torch.device("cuda", self.device))
        code = ctypes.c_int(0)
        C.check(C.lib().arctn_b200_program_device_status(self._h, workspace.data_ptr(), st.cuda_stream,
                                                         ctypes.byref(code)), "device status")
        return code.value

    def profile(self, arrays, *, workspace=None):
        """Launch-by-launch run with CUDA events between launches: (ms, kind, algorithmic work) per launch."""
        arrays, code, torch_mode = _preflight(arrays, self.inputs, self.size_dict, "profile failed",
                                              self._shapes())
        call = _DeviceCall(arrays, torch_mode, self.device)
        out = call.empty(self.output_shape, _torch_dtype(code))
        ws = workspace if workspace is not None else call.workspace(self.workspace_bytes)
        n = self.launches
        ms = (ctypes.c_float * n)()
        kind = (ctypes.c_int * n)(*([-1] * n))  # one entry per launch unit; a split op's two kernels share one
        work = (ctypes.c_double * n)()
        torch = _torch()
        with torch.cuda.device(call.device):
            if self.has_gradient:  # forward + reverse sweep, with ones as the incoming gradient
                g = torch.ones(self.output_shape, dtype=_torch_dtype(code), device=call.device)
                grads = [torch.empty_like(t) for t in call.tensors]
                gptr = (ctypes.c_void_p * len(grads))(*[t.data_ptr() for t in grads])
                C.check(C.lib().arctn_b200_program_profile_gradient(
                    self._h, call.ptrs, g.data_ptr(), gptr, out.data_ptr(), ws.data_ptr(), ws.numel(),
                    call.stream.cuda_stream, ms, kind, work), "profile failed")
            else:
                C.check(C.lib().arctn_b200_program_profile(self._h, call.ptrs, out.data_ptr(), ws.data_ptr(),
                                                           ws.numel(), call.stream.cuda_stream, ms, kind, work),
                        "profile failed")
        used = [i for i in range(n) if kind[i] >= 0]
        return [ms[i] for i in used], [kind[i] for i in used], [work[i] for i in used]

    def execute_stripped(self, arrays):
        """Mantissa tensor and decimal exponent (src/compiled.rs:376-441); unsliced programs only."""
        arrays, code, torch_mode = _preflight(arrays, self.inputs, self.size_dict, "compiled contraction failed")
        call = _DeviceCall(arrays, torch_mode, self.device)
        out = call.empty(self.output_shape, _torch_dtype(code))
        ws = call.workspace(self.workspace_bytes)
        e = ctypes.c_double(0.0)
        with _torch().cuda.device(call.device):
            C.check(C.lib().arctn_b200_program_execute_stripped(self._h, call.ptrs, out.data_ptr(), ws.data_ptr(),
                                                                ws.numel(), call.stream.cuda_stream,
                                                                ctypes.byref(e)), "compiled contraction failed")
        return _to_output(out, torch_mode), e.value


class ProgramBatch:
    """Many independent programs (uneven networks, mixed dtypes) run as one CUDA graph launch.

    ``mode="persistent"`` (the default): the small programs made of SIMT steps only run inside one
    persistent interpreter launch that follows the steps' dependencies on the device, while the others
    (tensor-core steps, large SIMT GEMMs) run launch by launch on up to ``max_lanes`` streams alongside it.
    ``mode="staged"``: every program inside the interpreter, tensor-core GEMMs and their operand packs
    launched between interpreter launches.  ``mode="lanes"``: every program launch by launch, spread over
    the streams longest first onto the least-loaded lane.  All modes give the same bits.  No reference
    counterpart: ArcTN contracts one network per call.
    """

    _MODES = {"lanes": 0, "persistent": 1, "staged": 2}

    def __init__(self, programs, *, max_lanes=32, mode="persistent"):
        self.programs = list(programs)
        if not self.programs:
            raise ValueError("a batch needs at least one program")
        arr = (C.vp * len(self.programs))(*[p._h for p in self.programs])
        h = C.vp()
        if mode not in self._MODES:
            raise ValueError(f"batch mode must be one of {sorted(self._MODES)}")
        C.check(C.lib().arctn_b200_batch_create_mode(arr, len(self.programs), int(max_lanes), self._MODES[mode],
                                                     ctypes.byref(h)), "batch")
        self._h = h
        self.mode = mode
        self.workspace_bytes = int(C.lib().arctn_b200_batch_workspace_size(h))
        self.lanes = int(C.lib().arctn_b200_batch_lanes(h))

    def describe(self, detail=False):
        """Mode, lanes, workspace regions and the interpreter's stages, steps and tasks per part, as a dict
        (host-only; works without a GPU).  ``detail=True`` adds every interpreter step and staged launch."""
        import json

        need = C.u64(0)
        C.check(C.lib().arctn_b200_batch_describe(self._h, int(bool(detail)), None, 0, ctypes.byref(need)),
                "batch describe")
        buf = ctypes.create_string_buffer(int(need.value))
        C.check(C.lib().arctn_b200_batch_describe(self._h, int(bool(detail)), buf, need.value,
                                                  ctypes.byref(need)), "batch describe")
        return json.loads(buf.value.decode())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                C.lib().arctn_b200_batch_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self._h = None

    def _bind(self, arrays_list, context):
        if len(arrays_list) != len(self.programs):
            raise ValueError(f"{context}: {len(arrays_list)} input lists for {len(self.programs)} programs")
        calls = []
        for j, (p, arrays) in enumerate(zip(self.programs, arrays_list)):
            arrays, code, torch_mode = _preflight(arrays, p.inputs, p.size_dict, f"{context} (program {j})",
                                                  p._shapes())
            if code != p.code:
                raise ValueError(f"{context}: program {j} arrays dtype differs from the program's dtype")
            calls.append((_DeviceCall(arrays, torch_mode, p.device), code, torch_mode))
        return calls

    def _host_run(self, arrays_list, gradient, grad_outputs, workspace, stream, context):
        """NumPy inputs: every program's inputs (and grad_outputs) go to the GPU through one pinned staging
        buffer and one copy, every output and gradient comes back in one copy.  The device buffers of the
        previous call on the same stream with the same shapes are reused, so the captured graph replays."""
        torch = _torch()
        if len(arrays_list) != len(self.programs):
            raise ValueError(f"{context}: {len(arrays_list)} input lists for {len(self.programs)} programs")
        checked = []
        for j, (p, arrays) in enumerate(zip(self.programs, arrays_list)):
            arrays, code, torch_mode = _preflight(arrays, p.inputs, p.size_dict, f"{context} (program {j})",
                                                  p._shapes())
            if torch_mode:
                raise ValueError(f"{context}: program {j} mixes CUDA tensors with the NumPy arrays of program 0")
            if code != p.code:
                raise ValueError(f"{context}: program {j} arrays dtype differs from the program's dtype")
            if gradient and not p.has_gradient:
                raise ValueError(f"{context}: program {j} was built without gradient=True")
            checked.append([np.array(a, order="C", copy=None) for a in arrays])
        dev = torch.device("cuda", torch.cuda.current_device() if self.programs[0].device is None
                           else self.programs[0].device)
        st = stream if stream is not None else torch.cuda.current_stream(dev)
        np_dt = {C.F32: np.float32, C.F64: np.float64, C.C64: np.complex64, C.C128: np.complex128}
        gouts = []
        if gradient:
            for j, p in enumerate(self.programs):
                g = None if grad_outputs is None else grad_outputs[j]
                g = np.ones(p.output_shape, np_dt[p.code]) if g is None else np.array(g, np_dt[p.code], order="C")
                if g.shape != tuple(p.output_shape):
                    raise ValueError(f"{context}: grad_outputs[{j}] shape {g.shape} is not {tuple(p.output_shape)}")
                gouts.append(g)
        # The layout depends only on the programs' shapes and dtypes, which the preflight has enforced.
        sig = (st.cuda_stream, gradient)
        cache = getattr(self, "_host_cache", None)
        if cache is None or cache["sig"] != sig or (workspace is not None and cache["ws"] is not workspace):
            def place(tensors, total):
                # element-aligned (the kernels load whole elements): tight packing lets one copy fill a run
                # of tensors of one dtype
                offs = []
                for shape, dt in tensors:
                    isz = np.dtype(dt).itemsize
                    total = (total + isz - 1) // isz * isz
                    offs.append(total)
                    total += int(np.prod(shape, dtype=np.int64)) * isz
                return offs, total
            ins = [(a.shape, a.dtype) for arrs in checked for a in arrs]
            in_offs, n_in = place(ins + [(g.shape, g.dtype) for g in gouts], 0)
            outs = [(tuple(p.output_shape), np_dt[p.code]) for p in self.programs]
            out_offs, n_out = place(outs + (ins if gradient else []), 0)
            d_in = torch.empty(max(n_in, 1), dtype=torch.uint8, device=dev)
            d_out = torch.empty(max(n_out, 1), dtype=torch.uint8, device=dev)
            base_in, base_out = d_in.data_ptr(), d_out.data_ptr()
            k, inp = 0, []
            for arrs in checked:
                inp.append((C.vp * len(arrs))(*[base_in + in_offs[k + q] for q in range(len(arrs))]))
                k += len(arrs)
            n_prog = len(self.programs)
            cache = {
                "sig": sig, "d_in": d_in, "d_out": d_out, "in_offs": in_offs, "out_offs": out_offs,
                "h_in": torch.empty(max(n_in, 1), dtype=torch.uint8, pin_memory=True),
                "h_out": torch.empty(max(n_out, 1), dtype=torch.uint8, pin_memory=True),
                "ws": workspace if workspace is not None else torch.empty(
                    max(self.workspace_bytes, 1), dtype=torch.uint8, device=dev),
                "inp_arrays": inp, "inp": (C.vpp * n_prog)(*[ctypes.cast(a, C.vpp) for a in inp]),
                "optr": (C.vp * n_prog)(*[base_out + out_offs[j] for j in range(n_prog)]),
                "outs": outs, "ins": ins,
            }
            if gradient:
                cache["gptr"] = (C.vp * n_prog)(*[base_in + in_offs[k + j] for j in range(n_prog)])
                garrs, q = [], n_prog
                for arrs in checked:
                    garrs.append((C.vp * len(arrs))(*[base_out + out_offs[q + r] for r in range(len(arrs))]))
                    q += len(arrs)
                cache["garrs"] = garrs
                cache["gpp"] = (C.vpp * n_prog)(*[ctypes.cast(a, C.vpp) for a in garrs])
            self._host_cache = cache
        if "in_runs" not in cache:  # runs of consecutive tensors without alignment padding between them
            runs, k = [], 0
            flat = [a.nbytes for arrs in checked for a in arrs] + [g.nbytes for g in gouts]
            offs = cache["in_offs"]
            while k < len(flat):
                e = k + 1
                while e < len(flat) and offs[e] == offs[e - 1] + flat[e - 1]:
                    e += 1
                runs.append((k, e, offs[k]))
                k = e
            cache["in_runs"] = runs
        hv = cache["h_in"].numpy()
        flat = [a for arrs in checked for a in arrs] + gouts
        for k, e, o in cache["in_runs"]:
            chunk = np.concatenate([a.reshape(-1).view(np.uint8) for a in flat[k:e]]) if e - k > 1 else \
                flat[k].reshape(-1).view(np.uint8)
            hv[o:o + chunk.nbytes] = chunk
        ws = cache["ws"]
        with torch.cuda.device(dev), torch.cuda.stream(st):
            cache["d_in"].copy_(cache["h_in"], non_blocking=True)
            if gradient:
                C.check(C.lib().arctn_b200_batch_gradient(self._h, cache["inp"], cache["gptr"], cache["gpp"],
                                                          cache["optr"], ws.data_ptr(), ws.numel(), st.cuda_stream),
                        context)
            else:
                C.check(C.lib().arctn_b200_batch_execute(self._h, cache["inp"], cache["optr"], ws.data_ptr(),
                                                         ws.numel(), st.cuda_stream), context)
            cache["h_out"].copy_(cache["d_out"], non_blocking=True)
        st.synchronize()
        host = cache["h_out"].numpy().copy()  # one copy; the results are views of it
        views = [host[o:o + int(np.prod(shape, dtype=np.int64)) * np.dtype(dt).itemsize].view(dt).reshape(shape)
                 for (shape, dt), o in zip(cache["outs"] + (cache["ins"] if gradient else []), cache["out_offs"])]
        n_prog = len(self.programs)
        outs = views[:n_prog]
        if not gradient:
            return outs
        grads, q = [], n_prog
        for arrs in checked:
            grads.append(views[q:q + len(arrs)])
            q += len(arrs)
        return outs, grads

    @staticmethod
    def _numpy_inputs(arrays_list):
        try:
            return len(arrays_list) > 0 and len(arrays_list[0]) > 0 and not _is_torch(arrays_list[0][0])
        except TypeError:
            return False

    def execute(self, arrays_list, *, workspace=None, stream=None):
        """Every program's output, in program order."""
        if self._numpy_inputs(arrays_list):
            return self._host_run(arrays_list, False, None, workspace, stream, "batch execute")
        calls = self._bind(arrays_list, "batch execute")
        torch = _torch()
        outs = [c.empty(p.output_shape, _torch_dtype(code)) for p, (c, code, _) in zip(self.programs, calls)]
        c0 = calls[0][0]
        ws = workspace if workspace is not None else c0.workspace(self.workspace_bytes)
        st = stream if stream is not None else c0.stream
        inp = (C.vpp * len(calls))(*[ctypes.cast(c.ptrs, C.vpp) for c, _, _ in calls])
        optr = (C.vp * len(outs))(*[o.data_ptr() for o in outs])
        with torch.cuda.device(c0.device):
            C.check(C.lib().arctn_b200_batch_execute(self._h, inp, optr, ws.data_ptr(), ws.numel(), st.cuda_stream),
                    "batch execute")
        self._keep = (calls, ws, outs)
        return [_to_output(o, tm) for o, (_, _, tm) in zip(outs, calls)]

    def gradient(self, arrays_list, grad_outputs=None, *, workspace=None, stream=None):
        """(outputs, grads) of every program (built with ``gradient=True``); grad_outputs default to ones."""
        if self._numpy_inputs(arrays_list):
            return self._host_run(arrays_list, True, grad_outputs, workspace, stream, "batch gradient")
        calls = self._bind(arrays_list, "batch gradient")
        torch = _torch()
        outs, gouts, grads = [], [], []
        for j, (p, (c, code, _)) in enumerate(zip(self.programs, calls)):
            if not p.has_gradient:
                raise ValueError(f"batch gradient: program {j} was built without gradient=True")
            outs.append(c.empty(p.output_shape, _torch_dtype(code)))
            g = None if grad_outputs is None else grad_outputs[j]
            if g is None:
                g = torch.ones(p.output_shape, dtype=_torch_dtype(code), device=c.device)
            elif _is_torch(g):
                g = g.to(c.device, _torch_dtype(code)).contiguous()
            else:
                np_dt = {C.F32: np.float32, C.F64: np.float64, C.C64: np.complex64, C.C128: np.complex128}[code]
                g = torch.from_numpy(np.array(g, dtype=np_dt, order="C")).to(c.device)
            gouts.append(g)
            grads.append([torch.empty_like(t) for t in c.tensors])
        c0 = calls[0][0]
        ws = workspace if workspace is not None else c0.workspace(self.workspace_bytes)
        st = stream if stream is not None else c0.stream
        inp = (C.vpp * len(calls))(*[ctypes.cast(c.ptrs, C.vpp) for c, _, _ in calls])
        optr = (C.vp * len(outs))(*[o.data_ptr() for o in outs])
        gptr = (C.vp * len(gouts))(*[g.data_ptr() for g in gouts])
        garrs = [(C.vp * len(gl))(*[t.data_ptr() for t in gl]) for gl in grads]
        gpp = (C.vpp * len(garrs))(*[ctypes.cast(a, C.vpp) for a in garrs])
        with torch.cuda.device(c0.device):
            C.check(C.lib().arctn_b200_batch_gradient(self._h, inp, gptr, gpp, optr, ws.data_ptr(), ws.numel(),
                                                      st.cuda_stream), "batch gradient")
        self._keep = (calls, ws, outs, gouts, grads, garrs)
        outs_r = [_to_output(o, tm) for o, (_, _, tm) in zip(outs, calls)]
        grads_r = [[_to_output(t, tm) for t in gl] for gl, (_, _, tm) in zip(grads, calls)]
        return outs_r, grads_r

    def bind(self, arrays_list, *, gradient=False, grad_outputs=None, workspace=None, stream=None):
        """A zero-argument callable that re-runs the batch on fixed CUDA buffers.

        Validation, every output / gradient allocation and the pointer arrays happen here, once; each call
        is then one C-ABI call (a graph replay on a side stream).  ``arrays_list`` holds CUDA tensors; the
        returned callable has ``outputs``, ``grads`` (gradient runs) and ``workspace`` attributes, which
        every call overwrites.
        """
        calls = self._bind(arrays_list, "batch bind")
        torch = _torch()
        if any(tm is False for _, _, tm in calls):
            raise ValueError("batch bind: arrays must be CUDA torch tensors")
        c0 = calls[0][0]
        st = stream if stream is not None else c0.stream
        ws = workspace if workspace is not None else c0.workspace(self.workspace_bytes)
        outs = [c.empty(p.output_shape, _torch_dtype(code)) for p, (c, code, _) in zip(self.programs, calls)]
        inp = (C.vpp * len(calls))(*[ctypes.cast(c.ptrs, C.vpp) for c, _, _ in calls])
        optr = (C.vp * len(outs))(*[o.data_ptr() for o in outs])
        lib, h, dev = C.lib(), self._h, c0.device
        if gradient:
            gouts, grads = [], []
            for j, (p, (c, code, _)) in enumerate(zip(self.programs, calls)):
                if not p.has_gradient:
                    raise ValueError(f"batch bind: program {j} was built without gradient=True")
                g = None if grad_outputs is None else grad_outputs[j]
                g = torch.ones(p.output_shape, dtype=_torch_dtype(code), device=c.device) if g is None else \
                    g.to(c.device, _torch_dtype(code)).contiguous()
                gouts.append(g)
                grads.append([torch.empty_like(t) for t in c.tensors])
            gptr = (C.vp * len(gouts))(*[g.data_ptr() for g in gouts])
            garrs = [(C.vp * len(gl))(*[t.data_ptr() for t in gl]) for gl in grads]
            gpp = (C.vpp * len(garrs))(*[ctypes.cast(a, C.vpp) for a in garrs])

            def run():
                with torch.cuda.device(dev):
                    C.check(lib.arctn_b200_batch_gradient(h, inp, gptr, gpp, optr, ws.data_ptr(), ws.numel(),
                                                          st.cuda_stream), "batch gradient")
            run.grads = grads
            run._keep = (calls, gouts, garrs)
        else:
            def run():
                with torch.cuda.device(dev):
                    C.check(lib.arctn_b200_batch_execute(h, inp, optr, ws.data_ptr(), ws.numel(), st.cuda_stream),
                            "batch execute")
            run._keep = (calls,)
        run.outputs = outs
        run.workspace = ws
        return run

    def device_status(self, workspace, stream=None):
        torch = _torch()
        st = stream if stream is not None else torch.cuda.current_stream(
            torch.device("cuda", self.programs[0].device))
        code = ctypes.c_int(0)
        C.check(C.lib().arctn_b200_batch_device_status(self._h, workspace.data_ptr(), st.cuda_stream,
                                                       ctypes.byref(code)), "batch device status")
        return code.value


def _is_torch_dtype(d):
    try:
        import torch
    except ImportError:  # pragma: no cover
        return False
    return isinstance(d, torch.dtype)


# ---------------------------------------------------------------------------- CompiledContraction


class InputPrep:
    """CompiledInputPrep (src/compiled.rs:33-75)."""

    def __init__(self, owner, index, info):
        self._owner, self._i = owner, index
        self._input_shape = tuple(info.input_shape[j] for j in range(info.n_input_shape))
        self._traces = [tuple(info.traces[3 * t + j] for j in range(3)) for t in range(info.n_traces)]
        self._legs = tuple(int(info.legs[j]) for j in range(info.n_legs))
        self._shape = tuple(int(info.shape[j]) for j in range(info.n_legs))

    def is_identity(self):
        return not self._traces

    def input_shape(self):
        return self._input_shape

    def traces(self):
        return list(self._traces)

    def legs(self):
        return self._legs

    def shape(self):
        return self._shape

    def execute(self, tensor):
        return self._owner._stage("prep", self._i, [tensor], self._input_shape, self._shape)


class PairStep:
    """CompiledPairContraction (src/compiled.rs:77-172)."""

    def __init__(self, owner, index, s):
        self._owner, self._i = owner, index
        rng = lambda p, n: tuple(int(p[j]) for j in range(n))  # noqa: E731
        self._left_slot, self._right_slot, self._result_slot = int(s.left_slot), int(s.right_slot), int(s.result_slot)
        self._left_legs = rng(s.left_legs, s.n_left)
        self._right_legs = rng(s.right_legs, s.n_right)
        self._result_legs = rng(s.result_legs, s.n_result)
        self._left_shape = rng(s.left_shape, s.n_left)
        self._right_shape = rng(s.right_shape, s.n_right)
        self._result_shape = rng(s.result_shape, s.n_result)
        self._sum_a = rng(s.sum_a, s.n_sum_a)
        self._sum_b = rng(s.sum_b, s.n_sum_b)
        self._a_perm = rng(s.a_perm, s.n_left - s.n_sum_a)
        self._b_perm = rng(s.b_perm, s.n_right - s.n_sum_b)
        self._dims = (int(s.bt), int(s.m), int(s.k), int(s.n))

    def left_slot(self):
        return self._left_slot

    def right_slot(self):
        return self._right_slot

    def result_slot(self):
        return self._result_slot

    def left_legs(self):
        return self._left_legs

    def right_legs(self):
        return self._right_legs

    def result_legs(self):
        return self._result_legs

    def left_shape(self):
        return self._left_shape

    def right_shape(self):
        return self._right_shape

    def result_shape(self):
        return self._result_shape

    def sum_a(self):
        return self._sum_a

    def sum_b(self):
        return self._sum_b

    def a_perm(self):
        return self._a_perm

    def b_perm(self):
        return self._b_perm

    def gemm_dims(self):
        return self._dims

    def execute(self, left, right, *, precision="fp32"):
        return self._owner._stage("step", self._i, [left, right], None, self._result_shape, precision=precision)


class Finalize:
    """CompiledFinalize (src/compiled.rs:174-219)."""

    def __init__(self, owner, f):
        self._owner = owner
        self._slot = int(f.slot)
        self._input_legs = tuple(int(f.input_legs[j]) for j in range(f.n_input))
        self._input_shape = tuple(int(f.input_shape[j]) for j in range(f.n_input))
        self._sum = tuple(int(f.sum[j]) for j in range(f.n_sum))
        self._perm = tuple(int(f.perm[j]) for j in range(f.n_output))
        self._output_shape = tuple(int(f.output_shape[j]) for j in range(f.n_output))

    def slot(self):
        return self._slot

    def input_legs(self):
        return self._input_legs

    def input_shape(self):
        return self._input_shape

    def output_shape(self):
        return self._output_shape

    def sum_axes(self):
        return self._sum

    def perm(self):
        return self._perm

    def is_identity(self):
        return not self._sum and all(i == p for i, p in enumerate(self._perm))

    def execute(self, tensor):
        return self._owner._stage("finalize", 0, [tensor], self._input_shape, self._output_shape)


class CompiledContraction:
    """A reusable exact contraction compiled from an SSA path (pybind/src/lib.rs:355-454)."""

    def __init__(self, inputs, output, size_dict, ssa_path, handle):
        self.inputs = [[int(l) for l in t] for t in inputs]
        self.output = [int(l) for l in output]
        self.size_dict = {int(k): int(v) for k, v in size_dict.items()}
        self.ssa_path = [(int(a), int(b)) for a, b in ssa_path]
        self._h = handle
        self._programs = {}
        self._lock = threading.Lock()
        L = C.lib()
        self._n_inputs = int(L.arctn_b200_plan_n_inputs(handle))
        self._n_steps = int(L.arctn_b200_plan_n_steps(handle))
        self.log10_flops = float(L.arctn_b200_plan_log10_flops(handle))
        self.log2_peak_size = float(L.arctn_b200_plan_log2_peak_size(handle))
        self._preps = []
        for i in range(self._n_inputs):
            info = C.PrepInfo()
            C.check(L.arctn_b200_plan_prep_info(handle, i, ctypes.byref(info)))
            self._preps.append(InputPrep(self, i, info))
        self._steps = []
        for s in range(self._n_steps):
            info = C.StepInfo()
            C.check(L.arctn_b200_plan_step_info(handle, s, ctypes.byref(info)))
            self._steps.append(PairStep(self, s, info))
        fi = C.FinalizeInfo()
        C.check(L.arctn_b200_plan_finalize_info(handle, ctypes.byref(fi)))
        self._finalize = Finalize(self, fi)

    @staticmethod
    def compile(inputs, output, size_dict, *, ssa_path):
        """Compile a reusable contraction from an **SSA** path (keyword required, as the reference)."""
        net = C.NetworkArgs(inputs, output, size_dict)
        n, p = C.path_array(ssa_path)
        h = C.vp()
        C.check(C.lib().arctn_b200_plan_compile(net.ptr, n, p.ctypes.data_as(C.u64p), ctypes.byref(h)),
                "invalid compiled path")
        return CompiledContraction(inputs, output, size_dict, ssa_path, h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            C.lib().arctn_b200_plan_destroy(h)
            self._h = None

    def n_inputs(self):
        return self._n_inputs

    def n_steps(self):
        return self._n_steps

    def input_preps(self):
        return list(self._preps)

    def pair_steps(self):
        return list(self._steps)

    def finalize(self):
        return self._finalize

    def program(self, code, precision="fp32", device=None):
        key = (code, _precision(precision), device)
        with self._lock:
            prog = self._programs.get(key)
            if prog is None:
                prog = SlicedProgram(self.inputs, self.output, self.size_dict, self.ssa_path, (), dtype=code,
                                     precision=precision, device=device)
                self._programs[key] = prog
        return prog

    def execute(self, arrays, *, precision="fp32", f64_out=False):
        """Execute on arrays with the frozen shapes; one dtype for all inputs."""
        if len(list(arrays)) != self._n_inputs:
            raise ValueError(f"{len(list(arrays))} arrays given for a plan with {self._n_inputs} inputs")
        arrays, code, torch_mode = _preflight(arrays, self.inputs, self.size_dict, "compiled contraction failed")
        dev = arrays[0].device.index if torch_mode else None
        return self.program(code, precision, dev).execute(arrays, f64_out=f64_out)

    __call__ = execute

    def execute_stripped(self, arrays):
        arrays, code, torch_mode = _preflight(arrays, self.inputs, self.size_dict, "compiled contraction failed")
        dev = arrays[0].device.index if torch_mode else None
        return self.program(code, "fp32", dev).execute_stripped(arrays)

    def stats(self):
        return {"path_format": "ssa-v1", "n_inputs": self._n_inputs, "n_steps": self._n_steps,
                "log10_flops": self.log10_flops, "log2_peak_size": self.log2_peak_size}

    def __repr__(self):
        return f"CompiledContraction(path_format='ssa-v1', n_inputs={self._n_inputs}, n_steps={self._n_steps})"

    # Stage execution ---------------------------------------------------------------------------
    def _stage(self, kind, idx, tensors, want_shape, out_shape, precision="fp32"):
        torch = _torch()
        torch_mode = _is_torch(tensors[0])
        code = None
        for t in tensors:
            c = _torch_code(t.dtype) if _is_torch(t) else _NP_CODES.get(np.asarray(t).dtype)
            if c is None:
                raise ValueError("unsupported dtype")
            if code is None:
                code = c
            elif c != code:
                raise ValueError("stage operands differ in dtype")
        if kind == "step":
            st = self._steps[idx]
            shapes = [st.left_shape(), st.right_shape()]
            labels = ["left operand", "right operand"]
        elif kind == "prep":
            shapes, labels = [want_shape], ["input tensor"]
        else:
            shapes, labels = [want_shape], ["finalize tensor"]
        for t, shp, lab in zip(tensors, shapes, labels):
            if tuple(int(d) for d in t.shape) != tuple(shp):
                raise ValueError(f"{lab} shape {tuple(t.shape)} does not match the compiled plan's {tuple(shp)}")
            if _is_torch(t) and not t.is_contiguous():
                raise ValueError(f"{lab} must be contiguous")
        call = _DeviceCall(tensors, torch_mode)
        out = call.empty(tuple(out_shape), _torch_dtype(code))
        L = C.lib()
        with torch.cuda.device(call.device):
            if kind == "step":
                p = _precision(precision)
                nbytes = int(L.arctn_b200_plan_step_workspace_size(self._h, code, p, idx))
                ws = call.workspace(nbytes)
                rc = L.arctn_b200_plan_step_execute(self._h, code, p, idx, call.ptrs[0], call.ptrs[1],
                                                    out.data_ptr(), ws.data_ptr(), ws.numel(),
                                                    call.stream.cuda_stream)
            elif kind == "prep":
                nbytes = int(L.arctn_b200_plan_prep_workspace_size(self._h, code, idx))
                ws = call.workspace(nbytes)
                rc = L.arctn_b200_plan_prep_execute(self._h, code, idx, call.ptrs[0], out.data_ptr(), ws.data_ptr(),
                                                    ws.numel(), call.stream.cuda_stream)
            else:
                nbytes = int(L.arctn_b200_plan_finalize_workspace_size(self._h, code))
                ws = call.workspace(nbytes)
                rc = L.arctn_b200_plan_finalize_execute(self._h, code, call.ptrs[0], out.data_ptr(), ws.data_ptr(),
                                                        ws.numel(), call.stream.cuda_stream)
        C.check(rc, f"{kind} stage failed")
        return _to_output(out, torch_mode)


# ---------------------------------------------------------------------------- functional API


def linear_to_ssa(linear_path, n):
    """Inverse of ssa_to_linear (pybind/src/lib.rs:153-175)."""
    ids = list(range(n))
    out = []
    for nxt, (a, b) in enumerate(linear_path, start=n):
        lo, hi = (a, b) if a < b else (b, a)
        if hi >= len(ids) or lo == hi:
            raise ValueError(f"linear path index out of range or self-contraction: ({a},{b}); "
                             f"{len(ids)} tensors are alive (pass SSA paths through ssa_path=)")
        out.append((ids[lo], ids[hi]))
        del ids[hi]
        del ids[lo]
        ids.append(nxt)
    return out


def ssa_to_linear(ssa_path, n):
    """Recycled linear form of an SSA path (pybind/src/lib.rs:137-151)."""
    ids = list(range(n))
    out = []
    for nxt, (a, b) in enumerate(ssa_path, start=n):
        ia, ib = ids.index(a), ids.index(b)
        lo, hi = (ia, ib) if ia < ib else (ib, ia)
        out.append((lo, hi))
        del ids[hi]
        del ids[lo]
        ids.append(nxt)
    return out


def contract_sliced(inputs, output, size_dict, arrays, sliced_legs, path=None, ssa_path=None, *,
                    precision="fp32", f64_out=False):
    """Execute a supplied path over every slice assignment (pybind/src/lib.rs:692-765)."""
    n = len(inputs)
    arrays = list(arrays)
    if len(arrays) != n:
        raise ValueError(f"{len(arrays)} arrays given for {n} inputs")
    if path is not None and ssa_path is not None:
        raise ValueError("path and ssa_path are mutually exclusive (path = linear form, ssa_path = SSA form)")
    for leg in sliced_legs:
        if int(leg) not in {int(k) for k in size_dict}:
            raise ValueError(f"sliced leg {leg} is not in the network's size_dict")
    arrays, code, torch_mode = _preflight(arrays, inputs, size_dict, "sliced contraction failed")
    if ssa_path is not None:
        ssa = [tuple(p) for p in ssa_path]
    elif path is not None:
        ssa = linear_to_ssa(path, n)
    else:
        raise ValueError("give path= (linear form) or ssa_path= (SSA form)")
    dev = arrays[0].device.index if torch_mode else None
    prog = SlicedProgram(inputs, output, size_dict, ssa, sliced_legs, dtype=code, precision=precision, device=dev,
                         use_graph=False)
    return prog.execute(arrays, f64_out=f64_out)


def _to_int_labels(inputs, output, size_dict):
    """Arbitrary hashable labels -> dense u32 ids (pybind/python/arctn/__init__.py:186-235)."""
    if not hasattr(size_dict, "items"):
        raise TypeError("size_dict must be a mapping from leg label to positive integer dimension")
    label_of = {}

    def idx(lab):
        i = label_of.get(lab)
        if i is None:
            i = len(label_of)
            label_of[lab] = i
        return i

    inputs_i = [[idx(l) for l in term] for term in inputs]
    output_i = [idx(l) for l in output]
    missing = [lab for lab in label_of if lab not in size_dict]
    if missing:
        raise ValueError(f"size_dict lacks dimensions of used legs: {missing!r}")
    unused = [lab for lab in size_dict if lab not in label_of]
    if unused:
        raise ValueError(f"size_dict holds legs not used in inputs/output: {unused!r}")
    size_i = {}
    for lab, i in label_of.items():
        raw = size_dict[lab]
        if isinstance(raw, bool):
            raise ValueError(f"dimension of leg {lab!r} must be a positive integer, not bool")
        dim = operator.index(raw)
        if dim <= 0:
            raise ValueError(f"dimension of leg {lab!r} must be positive, got {dim}")
        size_i[i] = dim
    return inputs_i, output_i, size_i, label_of


def _validate_backend(backend):
    if not isinstance(backend, str) or not backend or backend != backend.strip():
        raise ValueError(f"backend must be a non-empty string without surrounding spaces, got {backend!r}")
    if backend == "auto":
        raise ValueError("backend must be chosen explicitly; this package executes backend='b200'")
    if backend != "b200":
        raise ValueError(f"backend {backend!r} is not provided by arctn_b200; use backend='b200'")
    return backend


class ArcTNCompiledContraction:
    """``ArcTNCompiledContraction`` with ``backend='b200'`` (pybind/python/arctn/__init__.py:749-853)."""

    def __init__(self, backend, inputs, output, size_dict, ssa_path, implementation, compile_wall_s):
        self.backend = backend
        self.inputs = tuple(tuple(t) for t in inputs)
        self.output = tuple(output)
        self.size_dict = dict(size_dict)
        self.ssa_path = tuple(tuple(p) for p in ssa_path)
        self._implementation = implementation
        self.compile_wall_s = float(compile_wall_s)
        self.last_execute_wall_s = None
        self.last_dispatch_wall_s = None

    @classmethod
    def compile(cls, inputs, output, size_dict, *, ssa_path, backend="b200"):
        backend = _validate_backend(backend)
        inputs_i, output_i, size_i, _ = _to_int_labels(inputs, output, size_dict)
        ssa_path = [tuple(p) for p in ssa_path]
        t0 = time.perf_counter()
        impl = CompiledContraction.compile(inputs_i, output_i, size_i, ssa_path=ssa_path)
        return cls(backend, inputs_i, output_i, size_i, ssa_path, impl, time.perf_counter() - t0)

    def execute(self, arrays, *, precision="fp32"):
        t0 = time.perf_counter()
        result = self._implementation.execute(arrays, precision=precision)
        self.last_dispatch_wall_s = time.perf_counter() - t0
        self.last_execute_wall_s = self.last_dispatch_wall_s
        return result

    __call__ = execute

    def stats(self):
        out = {"backend": self.backend, "path_format": "ssa-v1", "n_inputs": len(self.inputs),
               "n_steps": len(self.ssa_path), "compile_wall_s": self.compile_wall_s,
               "last_execute_wall_s": self.last_execute_wall_s, "last_dispatch_wall_s": self.last_dispatch_wall_s}
        out.update(self._implementation.stats())
        return out

    def __repr__(self):
        return (f"ArcTNCompiledContraction(backend={self.backend!r}, n_inputs={len(self.inputs)}, "
                f"n_steps={len(self.ssa_path)})")


_AUTO_PRESETS = ("light", "heavy")
_SLICING_MODES = ("fixed", "dynamic")


def _validate_planning_options(preset, seed, target_size, slicing_mode, max_time, flops_weight, read_write_weight,
                               allow_output_slicing):
    """The reference's argument checks for ``arctn_contract`` (pybind/python/arctn/__init__.py:70-150), with the
    same exception types; returns the normalised (target_size, max_time, weights)."""
    if not isinstance(preset, str) or preset not in _AUTO_PRESETS:
        raise ValueError(f"preset must be 'light' or 'heavy', got {preset!r}")
    if isinstance(seed, bool):
        raise TypeError("seed must be an integer, not bool")
    operator.index(seed)
    if target_size is not None:
        if isinstance(target_size, bool):
            raise TypeError("target_size must be an integer, not bool")
        try:
            target_size = operator.index(target_size)
        except TypeError as exc:
            raise TypeError(f"target_size must be an integer, got {target_size!r}") from exc
        if target_size < 1:
            raise ValueError(f"target_size must be >= 1, got {target_size}")
        if target_size > sys.maxsize:
            raise OverflowError(f"target_size={target_size} exceeds this platform's usize range {sys.maxsize}")
    if not isinstance(slicing_mode, str) or slicing_mode not in _SLICING_MODES:
        raise ValueError(f"slicing_mode must be 'fixed' or 'dynamic', got {slicing_mode!r}")
    if slicing_mode == "dynamic" and target_size is None:
        raise ValueError("slicing_mode='dynamic' requires target_size")
    if max_time is not None:
        try:
            max_time = float(max_time)
        except (TypeError, ValueError) as exc:
            raise TypeError("max_time must be a finite number of seconds greater than 0") from exc
        if not math.isfinite(max_time) or max_time <= 0.0:
            raise ValueError("max_time must be a finite number of seconds greater than 0")
    weights = []
    for name, value in (("flops_weight", flops_weight), ("read_write_weight", read_write_weight)):
        if isinstance(value, bool):
            raise TypeError(f"{name} must be a finite non-negative number, not bool")
        try:
            value = float(value)
        except (TypeError, ValueError) as exc:
            raise TypeError(f"{name} must be a finite non-negative number") from exc
        if not math.isfinite(value) or value < 0.0:
            raise ValueError(f"{name} must be a finite non-negative number")
        weights.append(value)
    if weights == [0.0, 0.0]:
        raise ValueError("flops_weight and read_write_weight cannot both be 0")
    if not isinstance(allow_output_slicing, bool):
        raise TypeError("allow_output_slicing must be a bool")
    return target_size, max_time, tuple(weights)


def arctn_contract(inputs, output, size_dict, arrays, *, preset="heavy", seed=0, target_size=None,
                   slicing_mode="fixed", max_time=None, backend="b200", flops_weight=1.0, read_write_weight=64.0,
                   return_info=False, allow_output_slicing=False, ssa_path=None, sliced_legs=None,
                   precision="fp32"):
    """Plan (when no path is given), optionally slice, and execute on the B200 executor.

    Mirrors ``arctn_contract`` (pybind/python/arctn/__init__.py:903-1072): the same keywords, checked the same
    way.  The reference plans with its closed-source engine, which ``preset``, ``seed``, ``max_time`` and the
    weights steer; here the public greedy planner (src/paths/greedy.rs:317-320) and the slice search
    (src/slice.rs:209-289) produce the path and slices unless ``ssa_path`` / ``sliced_legs`` are given, so
    those planner options are validated and reported but do not change the plan.  ``slicing_mode="dynamic"``
    lets the reference change the path while slicing; this planner keeps it, which that mode allows.
    ``allow_output_slicing`` lets the slice search pick output legs; the output is then assembled from blocks.
    """
    target_size, max_time, (flops_weight, read_write_weight) = _validate_planning_options(
        preset, seed, target_size, slicing_mode, max_time, flops_weight, read_write_weight, allow_output_slicing)
    backend = _validate_backend(backend)
    inputs_i, output_i, size_i, _ = _to_int_labels(inputs, output, size_dict)
    t0 = time.perf_counter()
    ssa = [tuple(p) for p in ssa_path] if ssa_path is not None else greedy(inputs_i, output_i, size_i)
    if sliced_legs is None:
        sliced_legs = []
        if target_size is not None:
            found = find_slices_to_size(inputs_i, output_i, size_i, ssa, target_size,
                                        allow_output_slicing=allow_output_slicing)
            if found is None:
                raise ValueError(f"target_size (log2={math.log2(target_size):.6g}) is unreachable: no slicing "
                                 "meets it")
            sliced_legs = found
    plan_wall = time.perf_counter() - t0
    t1 = time.perf_counter()
    result = contract_sliced(inputs_i, output_i, size_i, arrays, sliced_legs, ssa_path=ssa, precision=precision)
    exec_wall = time.perf_counter() - t1
    if return_info:
        info = {"path": ssa, "sliced_legs": list(sliced_legs), "sliced": bool(sliced_legs),
                "execution_backend": backend, "execution_implementation": "arctn_b200.contract_sliced",
                "planning_wall_s": plan_wall, "execution_wall_s": exec_wall, "target_size": target_size,
                "target_log2_size": math.log2(target_size) if target_size is not None else None,
                "allow_output_slicing": allow_output_slicing, "preset": preset, "seed": seed,
                "slicing_mode": slicing_mode, "max_time": max_time, "flops_weight": flops_weight,
                "read_write_weight": read_write_weight, "planner": "greedy + find_slices_to_size"}
        info.update(simulate_path(inputs_i, output_i, size_i, ssa))
        return result, info
    return result

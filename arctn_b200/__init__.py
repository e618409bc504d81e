"""arctn_b200: B200-native executor for ArcTN's numerical contraction path.

The compute path is the in-tree CUDA library ``libarctn_b200.so`` (sm_100a),
reached through the C ABI of ``include/arctn_b200.h``.  There is no CPU
fallback: executing without a CUDA device raises ``ValueError``.
"""

__version__ = "0.2.0"

from ._capi import ArcTNB200Error
from .execution_plan import (ArcTNExecutionPlan, ExecutionPlan, PlanValidationError, arctn_plan, load_tensors_bin,
                             save_tensors_bin)
from .api import (
    ArcTNCompiledContraction,
    CompiledContraction,
    Finalize,
    InputPrep,
    PairStep,
    ProgramBatch,
    SlicedProgram,
    arctn_contract,
    build_info,
    contract_sliced,
    find_slices_to_size,
    greedy,
    linear_to_ssa,
    simulate_path,
    slice_parallel_chunks,
    slice_range,
    ssa_to_linear,
    tensor_pipe_peak,
)
from .sharding import lpt_shard, run_sharded
from .tuning import TuneTable, autotune

__all__ = [
    "__version__",
    "ArcTNB200Error",
    "ArcTNCompiledContraction",
    "ArcTNExecutionPlan",
    "ExecutionPlan",
    "PlanValidationError",
    "CompiledContraction",
    "Finalize",
    "InputPrep",
    "PairStep",
    "ProgramBatch",
    "SlicedProgram",
    "TuneTable",
    "autotune",
    "arctn_contract",
    "arctn_plan",
    "build_info",
    "contract_sliced",
    "find_slices_to_size",
    "load_tensors_bin",
    "save_tensors_bin",
    "greedy",
    "linear_to_ssa",
    "lpt_shard",
    "simulate_path",
    "slice_parallel_chunks",
    "run_sharded",
    "slice_range",
    "ssa_to_linear",
    "tensor_pipe_peak",
]

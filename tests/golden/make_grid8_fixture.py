"""Generates tests/golden/grid8_bond6.json: oracle values for the 8x8 grid, bond 6 adjoint check.

The network is the benchmark's grid8 workload (8x8 open grid, bond 6, complex64 entries N(0,1)/sqrt(6^rank),
seed 0), every entry multiplied by 4 (exact in binary floating point; it lifts the ~1e-35 scalar off the
bottom of FP32's range).  The path is the oracle's greedy path.  Recorded, all from oracle/ only:

- ``c128``: the plan replayed stage by stage in complex128 (oracle/torch_replay.py);
- ``oracle_c128``: the oracle executor in complex128 on the same (promoted) inputs;
- ``oracle_c64``: the oracle executor in complex64, i.e. the reference's own CPU result in that dtype;
- ``directional``: for 8 random complex directions V (numpy PCG64 seed 2024, independent of the inputs'
  seed, V_i ~ (N + iN)/sqrt(6^rank)),
  the Richardson-extrapolated central difference (4 d(eps/2) - d(eps)) / 3 of f(T + h V) in complex128,
  eps = 1e-3, where d(h) = (f(T + h V) - f(T - h V)) / (2 h).  For the holomorphic f this is
  sum_i <df/dT_i, V_i>.

Run from the repository root:  python tests/golden/make_grid8_fixture.py
"""

import json
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from arctn_b200 import networks as N  # noqa: E402  (NumPy generators only)
from oracle import oracle as O  # noqa: E402
from oracle.torch_replay import replay  # noqa: E402

EPS = 1e-3
N_DIRECTIONS = 8


def grid8_inputs():
    net, arrays = N.workload_grid8(6, np.complex64, seed=0)
    return net, [a * np.float32(4.0) for a in arrays]


DIRECTION_SEED = 2024


def directions(arrays):
    rng = np.random.default_rng(DIRECTION_SEED)
    return [[(rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape)) / np.sqrt(6.0 ** a.ndim)
             for a in arrays] for _ in range(N_DIRECTIONS)]


def main():
    net, arrays = grid8_inputs()
    path = O.greedy(*net.as_tuple())
    base = [a.astype(np.complex128) for a in arrays]

    def f(xs):
        with torch.no_grad():
            return complex(replay(*net.as_tuple(), path, [torch.from_numpy(x) for x in xs]).item())

    out = {"network": "grid8x8_bond6_c64_seed0_x4", "path_len": len(path), "eps": EPS,
           "direction_seed": DIRECTION_SEED,
           "c128": None, "oracle_c128": None, "oracle_c64": None, "directional": []}
    c = f(base)
    out["c128"] = [c.real, c.imag]
    oc = complex(O.contract_sliced(*net.as_tuple(), path, [], base))
    out["oracle_c128"] = [oc.real, oc.imag]
    o64 = complex(O.contract_sliced(*net.as_tuple(), path, [], arrays))
    out["oracle_c64"] = [o64.real, o64.imag]
    for v in directions(arrays):
        def d(h):
            return (f([x + h * dv for x, dv in zip(base, v)]) - f([x - h * dv for x, dv in zip(base, v)])) / (2 * h)
        rich = (4 * d(EPS / 2) - d(EPS)) / 3
        out["directional"].append([rich.real, rich.imag])
        print(rich, flush=True)
    with open(os.path.join(ROOT, "tests", "golden", "grid8_bond6.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main()

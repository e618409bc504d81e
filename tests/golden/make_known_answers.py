"""Writes tests/golden/known_answers.json: the reference's own known-answer cases.

The reference (Rust) cannot be built in this image, so its golden values are
transcribed from its test sources into JSON: each case records the network,
path, sliced legs, inputs and the expected result, with the file:line of the
reference test it comes from.  Run: python tests/golden/make_known_answers.py
"""

import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def cx(pairs):
    return [[float(a), float(b)] for a, b in pairs]


CASES = []

# tests/slice_validation.rs:23-31 -- dot product, sliced and unsliced, is exactly 13.0.
for sliced in ([], [0]):
    CASES.append(dict(name=f"dot_sliced{sliced}", source="tests/slice_validation.rs:23-31", dtype="float64",
                      inputs=[[0], [0]], output=[], size_dict={"0": 2}, ssa_path=[[0, 1]], sliced=sliced,
                      arrays=[[1.0, 2.0], [3.0, 5.0]], shapes=[[2], [2]], expected=[13.0], exact=True))

# tests/slice_output.rs:52-70 -- unary output blocks keep output order; exact values.
unary = [float(100 * a + 10 * b + c) for a in range(2) for b in range(3) for c in range(4)]
for sliced in ([0], [2], [2, 0], [1, 2], [2, 1, 0]):
    CASES.append(dict(name=f"unary_blocks{sliced}", source="tests/slice_output.rs:52-70", dtype="float64",
                      inputs=[[0, 1, 2]], output=[2, 0], size_dict={"0": 2, "1": 3, "2": 4}, ssa_path=[],
                      sliced=sliced, arrays=[unary], shapes=[[2, 3, 4]],
                      expected=[30.0, 330.0, 33.0, 333.0, 36.0, 336.0, 39.0, 339.0], exact=True))

# tests/mpi_cli.rs:25-150 -- hand-computed results for all four dtypes, unsliced, internal,
# output and mixed slicing.
vals_m = [(1.0, 1.0), (2.0, -2.0), (3.0, 0.5), (4.0, 1.0), (5.0, -1.0), (6.0, 2.0), (7.0, 3.0), (8.0, -0.5)]
vals_s = [(1.0, 1.0), (2.0, -2.0), (5.0, -1.0), (6.0, 2.0)]
for dtype in ("float32", "float64", "complex64", "complex128"):
    complex_ = dtype.startswith("complex")
    for scalar in (False, True):
        vals = vals_s if scalar else vals_m
        half = len(vals) // 2
        if complex_:
            a, b = cx(vals[:half]), cx(vals[half:])
            exp = cx([(22.0, -4.0)]) if scalar else cx([(26.0, -4.0), (19.0, -9.0), (40.5, 18.5), (49.5, 15.0)])
        else:
            a, b = [v[0] for v in vals[:half]], [v[0] for v in vals[half:]]
            exp = [17.0] if scalar else [19.0, 22.0, 43.0, 50.0]
        if scalar:
            net = dict(inputs=[[0], [0]], output=[], size_dict={"0": 2}, shapes=[[2], [2]])
            slicings = [[], [0]]
        else:
            net = dict(inputs=[[0, 1], [1, 2]], output=[0, 2], size_dict={"0": 2, "1": 2, "2": 2},
                       shapes=[[2, 2], [2, 2]])
            slicings = [[], [1], [2, 0], [0, 1]]
        for sliced in slicings:
            CASES.append(dict(name=f"mpi_fixture_{dtype}_{'scalar' if scalar else 'matrix'}_{sliced}",
                              source="tests/mpi_cli.rs:25-150", dtype=dtype, ssa_path=[[0, 1]], sliced=sliced,
                              arrays=[a, b], expected=exp, exact=True, **net))

# tests/scalar32.rs:99-148 -- hand-valued 2x3 . 3x2 GEMM; f32 < 2e-6, c32 < 1e-5 of naive.
CASES.append(dict(name="scalar32_real", source="tests/scalar32.rs:99-121", dtype="float32",
                  inputs=[[0, 1], [1, 2]], output=[0, 2], size_dict={"0": 2, "1": 3, "2": 2}, ssa_path=[[0, 1]],
                  sliced=[], shapes=[[2, 3], [3, 2]],
                  arrays=[[1.0, -2.0, 0.5, 3.0, 4.0, -1.0], [2.0, 1.0, -1.0, 0.25, 0.5, -3.0]],
                  expected=None, tol=2e-6, exact=False))
CASES.append(dict(name="scalar32_complex", source="tests/scalar32.rs:123-148", dtype="complex64",
                  inputs=[[0, 1], [1, 2]], output=[0, 2], size_dict={"0": 2, "1": 3, "2": 2}, ssa_path=[[0, 1]],
                  sliced=[], shapes=[[2, 3], [3, 2]],
                  arrays=[cx([(1.0, 0.5), (-2.0, 1.0), (0.5, -0.25), (3.0, -1.0), (4.0, 0.75), (-1.0, 2.0)]),
                          cx([(2.0, -0.5), (1.0, 1.0), (-1.0, 0.25), (0.25, -2.0), (0.5, 1.5), (-3.0, 0.5)])],
                  expected=None, tol=1e-5, exact=False))

METRICS = [
    # src/path.rs:559-574: A[2,3] x B[3,5] -> 31 elements contraction size / rw, 10 total / max, peak 31.
    dict(source="src/path.rs:559-574", inputs=[[0, 1], [1, 2]], output=[0, 2], size_dict={"0": 2, "1": 3, "2": 5},
         ssa_path=[[0, 1]], expect={"log2_max_contraction_size": 31, "log2_read_write": 31, "log2_total_size": 10,
                                    "log2_max_size": 10, "log2_peak_size": 31}),
    # src/path.rs:576-587
    dict(source="src/path.rs:576-587", inputs=[[0, 1], [1, 2], [2, 3]], output=[0, 3],
         size_dict={"0": 2, "1": 3, "2": 5, "3": 7}, ssa_path=[[0, 1], [3, 2]],
         expect={"log2_read_write": 90, "log2_total_size": 24}),
    # src/path.rs:589-612
    dict(source="src/path.rs:591-600", inputs=[[0, 1], [1, 2]], output=[2], size_dict={"0": 7, "1": 3, "2": 5},
         ssa_path=[[0, 1]], expect={"log2_max_contraction_size": 23, "log2_read_write": 41}),
    dict(source="src/path.rs:602-611", inputs=[[0, 0, 1], [1, 2]], output=[2], size_dict={"0": 7, "1": 3, "2": 5},
         ssa_path=[[0, 1]], expect={"log2_max_contraction_size": 23, "log2_read_write": 167}),
    # src/path.rs:614-651
    dict(source="src/path.rs:618-625", inputs=[[0, 0, 1], [0, 1, 2]], output=[0, 2],
         size_dict={"0": 7, "1": 3, "2": 5}, ssa_path=[[0, 1]], expect={"log2_max_contraction_size": 161}),
    dict(source="src/path.rs:629-643", inputs=[[0, 1], [1, 2], [1, 3]], output=[0, 2, 3],
         size_dict={"0": 2, "1": 3, "2": 5, "3": 7}, ssa_path=[[0, 1], [3, 2]],
         expect={"log2_max_contraction_size": 121}),
    dict(source="src/path.rs:645-650", inputs=[[0, 1], [1, 2], [1, 3]], output=[0, 2, 3],
         size_dict={"0": 2, "1": 1, "2": 5, "3": 7}, ssa_path=[[0, 1], [3, 2]],
         expect={"log2_max_contraction_size": 87}),
    # src/compiled.rs:615-637: live peak 16 elements, max intermediate 4.
    dict(source="src/compiled.rs:615-637", inputs=[[0, 1], [1, 2], [2, 3]], output=[0, 3],
         size_dict={"0": 2, "1": 2, "2": 2, "3": 2}, ssa_path=[[0, 1], [3, 2]],
         expect={"log2_max_size": 4, "log2_peak_size": 16}),
    # tests/correctness.rs:286-305: chain A(2x4) B(4x8) C(8x3) along A(BC): FLOPs 120, rw 94.
    dict(source="tests/correctness.rs:286-305", inputs=[[0, 1], [1, 2], [2, 3]], output=[0, 3],
         size_dict={"0": 2, "1": 4, "2": 8, "3": 3}, ssa_path=[[1, 2], [0, 3]],
         expect={"log10_flops": 120, "log2_read_write": 94}),
]

# src/slice.rs:1339-1414 and :1290-1306 -- exact integer slicing targets.
SLICE_TARGETS = [
    dict(source="src/slice.rs:1341-1376", inputs=[[0, 2], [2, 1]], output=[0, 1],
         size_dict={"0": 499, "1": 465, "2": 2}, ssa_path=[[0, 1]], target=499 * 465, expect=[]),
    dict(source="src/slice.rs:1341-1376", inputs=[[0, 2], [2, 1]], output=[0, 1],
         size_dict={"0": 499, "1": 465, "2": 2}, ssa_path=[[0, 1]], target=499 * 465 - 1, expect=None),
    dict(source="src/slice.rs:1378-1396", inputs=[[0], []], output=[0], size_dict={"0": (1 << 40) + 1},
         ssa_path=[[0, 1]], target=1 << 40, expect=None),
    dict(source="src/slice.rs:1398-1414", inputs=[[0, 1]], output=[0], size_dict={"0": (1 << 40) + 1, "1": 2},
         ssa_path=[], target=1 << 40, expect=None),
    dict(source="src/slice.rs:1398-1414", inputs=[[0, 1]], output=[0], size_dict={"0": (1 << 40) + 1, "1": 2},
         ssa_path=[], target=(1 << 40) + 1, expect=[]),
    dict(source="src/slice.rs:1291-1306", inputs=[[0, 0, 1], [0, 2], [0, 3]], output=[1, 2, 3],
         size_dict={"0": 8, "1": 2, "2": 2, "3": 2}, ssa_path=[[0, 1], [3, 2]], target=16, expect=None),
]

# tests/slice_parallel.rs:97-140 -- chunk coverage known points.
CHUNKS = [dict(source="tests/slice_parallel.rs:125-139", n_slices=257, out_numel=1, ragged=True),
          dict(source="tests/slice_parallel.rs:127", n_slices=3, out_numel=1 << 21, ragged=None),
          dict(source="tests/slice_parallel.rs:139", n_slices=1000, out_numel=(1 << 64) - 1, expect=1)]

if __name__ == "__main__":
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump({"cases": CASES, "metrics": METRICS, "slice_targets": SLICE_TARGETS, "chunks": CHUNKS}, f,
                  indent=1)
    print(f"wrote {len(CASES)} execution cases, {len(METRICS)} metric cases")

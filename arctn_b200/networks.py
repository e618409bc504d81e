"""Tensor-network generators and the benchmark workloads.

Structure generators restate the reference's ``TensorNetwork`` constructors
(``src/network.rs:430-540``).  The reference draws randomness from ChaCha8
(crate rand_chacha 0.3.1), which is not reproducible here, so every random
choice uses NumPy's PCG64 with the stated seed; the algorithms (stub shuffle
with self-loop rejection, random spanning tree plus extra/open legs) are the
reference's.  Tensor values follow the workload definitions: i.i.d. N(0,1)
real and imaginary parts scaled by 1/sqrt(bond^rank).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Net:
    inputs: list
    output: list
    size_dict: dict
    name: str = "net"
    meta: dict = field(default_factory=dict)

    def shapes(self):
        return [tuple(self.size_dict[l] for l in t) for t in self.inputs]

    def as_tuple(self):
        return self.inputs, self.output, self.size_dict


def grid_2d(rows, cols, dim):
    """Open-boundary 2D grid, nearest-neighbour legs, scalar output (src/network.rs:460-488)."""
    inputs = [[] for _ in range(rows * cols)]
    size = {}
    nxt = 0
    for r in range(rows):
        for c in range(cols):
            if c + 1 < cols:
                inputs[r * cols + c].append(nxt)
                inputs[r * cols + c + 1].append(nxt)
                size[nxt] = dim
                nxt += 1
            if r + 1 < rows:
                inputs[r * cols + c].append(nxt)
                inputs[(r + 1) * cols + c].append(nxt)
                size[nxt] = dim
                nxt += 1
    return Net(inputs, [], size, name=f"grid_{rows}x{cols}")


def rand_regular(n, degree, dim, seed):
    """Random d-regular multigraph by stub shuffling, self-loops resampled (src/network.rs:430-458)."""
    assert n * degree % 2 == 0, "n*degree must be even"
    rng = np.random.Generator(np.random.PCG64(seed))
    stubs = np.repeat(np.arange(n), degree)
    while True:
        rng.shuffle(stubs)
        pairs = stubs.reshape(-1, 2)
        if np.all(pairs[:, 0] != pairs[:, 1]):
            break
    inputs = [[] for _ in range(n)]
    size = {}
    for leg, (a, b) in enumerate(pairs.tolist()):
        inputs[a].append(leg)
        inputs[b].append(leg)
        size[leg] = dim
    return Net(inputs, [], size, name=f"rand{degree}reg_n{n}")


def random_connected(n, extra, dims, n_open, seed):
    """Small connected random network: spanning tree + extra legs + open legs (src/network.rs:490-540)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    inputs = [[] for _ in range(n)]
    size = {}
    nxt = 0

    def add(a, b):
        nonlocal nxt
        inputs[a].append(nxt)
        inputs[b].append(nxt)
        size[nxt] = int(dims[rng.integers(len(dims))])
        nxt += 1

    for i in range(1, n):
        add(i, int(rng.integers(i)))
    for _ in range(extra):
        a = int(rng.integers(n))
        b = int(rng.integers(n))
        while b == a:
            b = int(rng.integers(n))
        add(a, b)
    output = []
    for _ in range(n_open):
        t = int(rng.integers(n))
        inputs[t].append(nxt)
        output.append(nxt)
        size[nxt] = int(dims[rng.integers(len(dims))])
        nxt += 1
    return Net(inputs, output, size, name=f"rand_conn_n{n}")


def brickwork_circuit(n_wires, depth, seed):
    """Closed brickwork circuit amplitude <bits| U |0...0>.

    Gates are 4x4 unitaries Q from the QR decomposition of a complex Gaussian
    matrix with phases fixed by the sign of diag(R); layer t acts on wire
    pairs (0,1),(2,3),... for even t and (1,2),(3,4),... for odd t.  Inputs
    are |0> caps (rank 1, dim 2), the gates (rank 4: out_a, out_b, in_a,
    in_b) and one closing cap per wire holding a random computational-basis
    bit.  Returns the network and its complex128 tensors.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    inputs, tensors, size = [], [], {}
    nxt = 0

    def new_leg():
        nonlocal nxt
        size[nxt] = 2
        nxt += 1
        return nxt - 1

    cur = []
    for _ in range(n_wires):
        leg = new_leg()
        inputs.append([leg])
        tensors.append(np.array([1.0, 0.0], dtype=np.complex128))
        cur.append(leg)
    for t in range(depth):
        for a in range(t % 2, n_wires - 1, 2):
            z = (rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))) / np.sqrt(2)
            q, r = np.linalg.qr(z)
            d = np.diag(r)
            q = q * (d / np.abs(d))
            oa, ob = new_leg(), new_leg()
            inputs.append([oa, ob, cur[a], cur[a + 1]])
            tensors.append(q.reshape(2, 2, 2, 2).astype(np.complex128))
            cur[a], cur[a + 1] = oa, ob
    bits = rng.integers(0, 2, size=n_wires)
    for w in range(n_wires):
        inputs.append([cur[w]])
        cap = np.zeros(2, dtype=np.complex128)
        cap[bits[w]] = 1.0
        tensors.append(cap)
    net = Net(inputs, [], size, name=f"brickwork_{n_wires}x{depth}", meta={"bits": bits.tolist()})
    return net, tensors


def gaussian_tensors(net, dtype, seed, scale_base=None):
    """i.i.d. N(0,1) entries (real and imaginary parts for complex dtypes) scaled by 1/sqrt(scale_base^rank).

    ``scale_base=None`` uses each tensor's own mean leg dimension.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    dtype = np.dtype(dtype)
    out = []
    for shape in net.shapes():
        rank = len(shape)
        base = scale_base if scale_base is not None else (np.mean(shape) if shape else 1.0)
        scale = 1.0 / np.sqrt(float(base) ** rank)
        if np.issubdtype(dtype, np.complexfloating):
            v = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * scale
        else:
            v = rng.standard_normal(shape) * scale
        out.append(np.array(np.asarray(v), dtype=dtype, order="C"))
    return out


# ------------------------------------------------------------------------------------------- workloads


def workload_grid6(dtype=np.complex128, seed=0):
    """6x6 open grid, bond 4, complex128 N(0,1)/sqrt(4^rank), scalar output, unsliced."""
    net = grid_2d(6, 6, 4)
    return net, gaussian_tensors(net, dtype, seed, scale_base=4)


def workload_rand3reg(n=64, bond=2, graph_seed=1, dtype=np.complex64, seed=0):
    """Random 3-regular graph, bond 2 per edge, complex64 N(0,1)/sqrt(8) entries, scalar output."""
    net = rand_regular(n, 3, bond, graph_seed)
    return net, gaussian_tensors(net, dtype, seed, scale_base=2)


def workload_grid8(bond=6, dtype=np.complex64, seed=0):
    """8x8 open grid, bond 6, complex64 N(0,1)/sqrt(6^rank), scalar output."""
    net = grid_2d(8, 8, bond)
    return net, gaussian_tensors(net, dtype, seed, scale_base=bond)


def workload_batch(count=256, seed=0):
    """Many uneven networks: random 3-regular graphs with n ~ U{20, 22, ..., 50} nodes and a bond
    dimension ~ U{2, 3, 4} per network, entries N(0,1)/sqrt(bond^3); even-numbered networks are float32,
    odd-numbered complex64.  Returns [(net, arrays)], graph j seeded by (seed, j)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for j in range(count):
        n = int(rng.integers(10, 26)) * 2
        bond = int(rng.integers(2, 5))
        net = rand_regular(n, 3, bond, seed * 100003 + j)
        dtype = np.float32 if j % 2 == 0 else np.complex64
        out.append((net, gaussian_tensors(net, dtype, seed * 100003 + j, scale_base=bond)))
    return out

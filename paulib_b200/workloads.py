"""Seeded synthetic workloads with the shapes of the Pauli-sum benchmarks.

Each generator returns host SoA planes (``x``/``z`` as (AS, n) uint64,
``flags`` uint8, ``val`` float64) and, for circuits, a rotation table plus
an op list.  There is no public dataset behind these workloads; the shapes,
sizes and value distributions follow the benchmark definitions:

* ``product_operands``   -- two PauliSum<64,double> of 4096 terms each over
  20 active qubits, weight U{1..4} on distinct qubits, op U{I,X,Y,Z} per
  chosen site, coefficients N(0,1).
* ``brickwork_circuit``  -- Heisenberg propagation: observable sum_i Z_i,
  layers of CNOTs on alternating neighbour pairs (pair offset = layer & 1),
  then RX(theta) on every qubit, then RZ(theta) on every qubit,
  theta ~ U[0, 2pi).
* ``window_sums``        -- PauliSum<256,double> terms supported on a random
  contiguous window of 2..6 qubits, op U{I,X,Y,Z}, coefficients U[-1,1].
* ``batch_instances``    -- independent propagation instances with qubit
  counts from {16,32,64,128}, depth U{4..24}, a single weight-1..3
  observable.

Rotations follow the evolve()/propagate() convention of the reference
(generator P with angle theta; PauliSumOperations.h:107-183).  A CNOT is
applied with apply_CNOT (PauliSumClifford.h:213-239).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

OP_ROT = 0
OP_CNOT = 1


@dataclass
class SoA:
    x: np.ndarray
    z: np.ndarray
    flags: np.ndarray
    val: np.ndarray
    num_qubits: int = 64

    @property
    def n(self) -> int:
        return int(self.val.shape[0])

    @property
    def array_size(self) -> int:
        return int(self.x.shape[0])


def words_for(num_qubits: int) -> int:
    return max(1, (num_qubits + 63) // 64)


def _set_sites(x, z, term, qubits, ops):
    """ops: 0=I, 1=X, 2=Y, 3=Z (I leaves both bits clear)."""
    for q, op in zip(qubits, ops):
        w, b = divmod(int(q), 64)
        bit = np.uint64(1) << np.uint64(b)
        if op in (1, 2):
            x[w, term] |= bit
        if op in (2, 3):
            z[w, term] |= bit


def product_operands(seed: int = 1, terms: int = 4096, active_qubits: int = 20,
                     max_weight: int = 4):
    """Two sums for the product + collate workload (64-qubit capacity)."""
    out = []
    for which in range(2):
        rng = np.random.default_rng([seed, which])
        x = np.zeros((1, terms), np.uint64)
        z = np.zeros((1, terms), np.uint64)
        weights = rng.integers(1, max_weight + 1, size=terms)
        for t in range(terms):
            qs = rng.choice(active_qubits, size=int(weights[t]), replace=False)
            ops = rng.integers(0, 4, size=int(weights[t]))
            _set_sites(x, z, t, qs, ops)
        val = rng.standard_normal(terms)
        out.append(SoA(x, z, np.zeros(terms, np.uint8), val, 64))
    return out[0], out[1]


def window_sums(seed: int = 3, terms: int = 16384, num_qubits: int = 256,
                min_len: int = 2, max_len: int = 6):
    """Two sums of windowed-support terms (commutator workload)."""
    aw = words_for(num_qubits)
    out = []
    for which in range(2):
        rng = np.random.default_rng([seed, which])
        x = np.zeros((aw, terms), np.uint64)
        z = np.zeros((aw, terms), np.uint64)
        lens = rng.integers(min_len, max_len + 1, size=terms)
        for t in range(terms):
            ln = int(lens[t])
            start = int(rng.integers(0, num_qubits - ln + 1))
            ops = rng.integers(0, 4, size=ln)
            _set_sites(x, z, t, range(start, start + ln), ops)
        val = rng.uniform(-1.0, 1.0, size=terms)
        out.append(SoA(x, z, np.zeros(terms, np.uint8), val, num_qubits))
    return out[0], out[1]


@dataclass
class Circuit:
    """Rotation table (generators + angles) and an op list in application order.

    ``ops`` rows are (kind, a, b): kind OP_ROT = rotation number a of
    ``rotations``; kind OP_CNOT = CNOT(control=a, target=b).
    """

    rotations: SoA
    ops: np.ndarray  # (n_ops, 3) int32
    num_qubits: int
    meta: dict = field(default_factory=dict)

    @property
    def n_rotations(self) -> int:
        return self.rotations.n


def brickwork_circuit(num_qubits: int, layers: int, rng: np.random.Generator) -> Circuit:
    """Layers of CNOT(q, q+1) for q = (layer & 1), (layer & 1) + 2, ...;
    then RX(theta) on every qubit; then RZ(theta) on every qubit."""
    aw = words_for(num_qubits)
    n_rot = 2 * num_qubits * layers
    x = np.zeros((aw, n_rot), np.uint64)
    z = np.zeros((aw, n_rot), np.uint64)
    theta = rng.uniform(0.0, 2.0 * np.pi, size=n_rot)
    ops = []
    r = 0
    for layer in range(layers):
        for q in range(layer & 1, num_qubits - 1, 2):
            ops.append((OP_CNOT, q, q + 1))
        for axis in ("X", "Z"):
            for q in range(num_qubits):
                w, b = divmod(q, 64)
                bit = np.uint64(1) << np.uint64(b)
                if axis == "X":
                    x[w, r] = bit
                else:
                    z[w, r] = bit
                ops.append((OP_ROT, r, 0))
                r += 1
    rot = SoA(x, z, np.zeros(n_rot, np.uint8), theta, num_qubits)
    return Circuit(rot, np.asarray(ops, np.int32).reshape(-1, 3), num_qubits,
                   {"layers": layers})


def sum_of_z(num_qubits: int) -> SoA:
    """Observable sum_i Z_i with unit coefficients."""
    aw = words_for(num_qubits)
    x = np.zeros((aw, num_qubits), np.uint64)
    z = np.zeros((aw, num_qubits), np.uint64)
    for q in range(num_qubits):
        w, b = divmod(q, 64)
        z[w, q] = np.uint64(1) << np.uint64(b)
    return SoA(x, z, np.zeros(num_qubits, np.uint8), np.ones(num_qubits), num_qubits)


def heisenberg_workload(seed: int = 2, num_qubits: int = 64, layers: int = 20):
    """Observable sum_i Z_i propagated through a brickwork CNOT+RX+RZ circuit.

    Truncation for this workload: |c| < 1e-4 dropped, Pauli weight > 8
    dropped."""
    rng = np.random.default_rng(seed)
    circ = brickwork_circuit(num_qubits, layers, rng)
    return sum_of_z(num_qubits), circ, {"max_weight": 8, "cutoff": 1e-4}


def single_pauli(num_qubits: int, rng: np.random.Generator, max_weight: int = 3) -> SoA:
    aw = words_for(num_qubits)
    x = np.zeros((aw, 1), np.uint64)
    z = np.zeros((aw, 1), np.uint64)
    w = int(rng.integers(1, max_weight + 1))
    qs = rng.choice(num_qubits, size=w, replace=False)
    ops = rng.integers(1, 4, size=w)  # X, Y or Z
    _set_sites(x, z, 0, qs, ops)
    return SoA(x, z, np.zeros(1, np.uint8), np.ones(1), num_qubits)


@dataclass
class Instance:
    observable: SoA
    circuit: Circuit
    max_weight: int
    cutoff: float


def batch_instances(seed: int = 4, count: int = 512, qubit_choices=(16, 32, 64, 128),
                    depth_range=(4, 24), max_weight: int = 10, cutoff: float = 1e-5):
    """Independent propagation instances of mixed width and depth."""
    out = []
    for i in range(count):
        rng = np.random.default_rng([seed, i])
        nq = int(rng.choice(qubit_choices))
        depth = int(rng.integers(depth_range[0], depth_range[1] + 1))
        obs = single_pauli(nq, rng)
        circ = brickwork_circuit(nq, depth, rng)
        out.append(Instance(obs, circ, max_weight, cutoff))
    return out


def heavy_instance(seed: int = 5, num_qubits: int = 128, depth: int = 40,
                   max_weight: int = 10, cutoff: float = 1e-5) -> Instance:
    rng = np.random.default_rng([seed, 999])
    return Instance(single_pauli(num_qubits, rng), brickwork_circuit(num_qubits, depth, rng),
                    max_weight, cutoff)

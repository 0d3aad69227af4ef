"""Seeded synthetic workloads of the compressed-state path.

Five circuits, each with the shape, sizes and value distribution of one of
the engine's measured configurations:

* ghz_fanout(n)            -- H(0) then CNOT(0 -> i), i = 1..n-1, from |0...0>
* qft_basis(n, seed)       -- QFT of a seeded random basis state x prepared
                              with X gates (the compressed state has no
                              basis-state setter in the reference, so inputs
                              are prepared by gates); per qubit j (high to
                              low) H(j), then controlled phases
                              R_k = diag(1, e^{2 pi i / 2^k}) from j onto every
                              lower qubit, then bit-reversal SWAPs
* brickwork(n, layers, seed) -- per layer a Haar-random SU(2) on every qubit,
                              then CZ on (0,1),(2,3),... in even layers and
                              (1,2),(3,4),... in odd layers
* hea(n, depth, seed)      -- per layer RY(theta) RZ(phi) on every qubit and a
                              CNOT ladder (i, i+1); angles U[0, 2 pi)
* qaoa_maxcut(n, p, seed)  -- H on all qubits, then per layer RZZ(gamma) on
                              every edge of a seeded random 3-regular graph
                              and RX(beta) on every qubit; gamma, beta U[0, pi)

Gates use Qulacs conventions (RX(t) = exp(+i t X/2), RZ(t) =
diag(e^{i t/2}, e^{-i t/2})).  parametric=True builds the rotations as
parametric gates for gradients.
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

import qulacs
from qulacs import gate as G


def ghz_fanout(n: int) -> qulacs.QuantumCircuit:
    c = qulacs.QuantumCircuit(n)
    c.add_H_gate(0)
    for i in range(1, n):
        c.add_CNOT_gate(0, i)
    return c


def qft_input(n: int, seed: int = 0) -> int:
    return int(np.random.default_rng(seed).integers(0, 2 ** n))


def controlled_phase(control: int, target: int, angle: float):
    g = G.DenseMatrix(target, np.diag([1.0, np.exp(1j * angle)]))
    g.add_control_qubit(control, 1)
    return g


def qft_basis(n: int, seed: int = 0, with_input: bool = True, swaps: bool = True) -> qulacs.QuantumCircuit:
    c = qulacs.QuantumCircuit(n)
    if with_input:
        x = qft_input(n, seed)
        for q in range(n):
            if (x >> q) & 1:
                c.add_X_gate(q)
    for j in reversed(range(n)):
        c.add_H_gate(j)
        for k in reversed(range(j)):
            c.add_gate(controlled_phase(j, k, 2.0 * math.pi / 2 ** (j - k + 1)))
    if swaps:
        for i in range(n // 2):
            c.add_SWAP_gate(i, n - 1 - i)
    return c


def qft_expected(n: int, x: int) -> np.ndarray:
    """Analytic QFT of |x> with this circuit's conventions: amplitude
    2^{-n/2} e^{2 pi i x k / 2^n} at basis k."""
    k = np.arange(1 << n, dtype=np.float64)
    return np.exp(2j * np.pi * ((x * k) % (1 << n)) / (1 << n)) / np.sqrt(1 << n)


def haar_su2(rng: np.random.Generator) -> np.ndarray:
    z = (rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))) / np.sqrt(2.0)
    q, r = np.linalg.qr(z)
    q = q * (np.diag(r) / np.abs(np.diag(r)))
    return q / np.sqrt(np.linalg.det(q))


def brickwork(n: int, layers: int = 20, seed: int = 0) -> qulacs.QuantumCircuit:
    rng = np.random.default_rng(seed)
    c = qulacs.QuantumCircuit(n)
    for layer in range(layers):
        for q in range(n):
            c.add_gate(G.DenseMatrix(q, haar_su2(rng)))
        for a in range(layer % 2, n - 1, 2):
            c.add_CZ_gate(a, a + 1)
    return c


def hea(n: int, depth: int = 8, seed: int = 0, parametric: bool = False):
    rng = np.random.default_rng(seed)
    angles = rng.uniform(0.0, 2.0 * math.pi, size=(depth, n, 2))
    c = qulacs.ParametricQuantumCircuit(n) if parametric else qulacs.QuantumCircuit(n)
    for d in range(depth):
        for q in range(n):
            if parametric:
                c.add_parametric_RY_gate(q, angles[d, q, 0])
                c.add_parametric_RZ_gate(q, angles[d, q, 1])
            else:
                c.add_RY_gate(q, angles[d, q, 0])
                c.add_RZ_gate(q, angles[d, q, 1])
        for q in range(n - 1):
            c.add_CNOT_gate(q, q + 1)
    return c


def hea_observable_terms(n: int) -> List[Tuple[float, str, Tuple[int, ...]]]:
    """H = sum_i Z_i Z_{i+1} + 0.5 sum_i X_i as (coef, pauli, qubits)."""
    terms = [(1.0, "ZZ", (i, i + 1)) for i in range(n - 1)]
    terms += [(0.5, "X", (i,)) for i in range(n)]
    return terms


def regular_graph_edges(n: int, degree: int = 3, seed: int = 0) -> List[Tuple[int, int]]:
    import networkx as nx
    g = nx.random_regular_graph(degree, n, seed=seed)
    return sorted((min(a, b), max(a, b)) for a, b in g.edges())


def rzz(a: int, b: int, angle: float):
    """exp(+i angle/2 Z_a Z_b) in the Qulacs sign convention of RZ."""
    ph = np.exp(0.5j * angle)
    return G.DenseMatrix([a, b], np.diag([ph, np.conj(ph), np.conj(ph), ph]))


def qaoa_params(p: int, seed: int = 0):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, math.pi, size=p), rng.uniform(0.0, math.pi, size=p)


def qaoa_maxcut(n: int, p: int = 4, seed: int = 0) -> qulacs.QuantumCircuit:
    edges = regular_graph_edges(n, 3, seed)
    gammas, betas = qaoa_params(p, seed)
    c = qulacs.QuantumCircuit(n)
    for q in range(n):
        c.add_H_gate(q)
    for layer in range(p):
        for a, b in edges:
            c.add_gate(rzz(a, b, gammas[layer]))
        for q in range(n):
            c.add_RX_gate(q, betas[layer])
    return c


WORKLOADS = {
    "ghz20": dict(builder=lambda: ghz_fanout(20), n=20, block_size=12, inner_size=4, dtype="complex128",
                  eps_rel=1e-3, eps_abs=1e-7),
    "qft30": dict(builder=lambda: qft_basis(30, seed=0), qft_input=qft_input(30, 0), n=30, block_size=20, inner_size=4, dtype="complex128",
                  eps_rel=1e-3, eps_abs=1e-7),
    "qft26": dict(builder=lambda: qft_basis(26, seed=0), qft_input=qft_input(26, 0), n=26, block_size=20, inner_size=4, dtype="complex128",
                  eps_rel=1e-3, eps_abs=1e-7),
    # the QFT workload in the complex64 pipeline (FP32 gate arithmetic, FP64 reductions)
    "qft30c64": dict(builder=lambda: qft_basis(30, seed=0), qft_input=qft_input(30, 0), n=30, block_size=20, inner_size=4, dtype="complex64",
                     eps_rel=1e-3, eps_abs=1e-7),
    "brickwork32": dict(builder=lambda: brickwork(32, 20, seed=0), n=32, block_size=22, inner_size=4,
                        dtype="complex64", eps_rel=1e-3, eps_abs=1e-7),
    "hea24": dict(builder=lambda: hea(24, 8, seed=0), n=24, block_size=18, inner_size=4, dtype="complex64",
                  eps_rel=1e-3, eps_abs=1e-7),
    "qaoa34": dict(builder=lambda: qaoa_maxcut(34, 4, seed=0), n=34, block_size=24, inner_size=4,
                   dtype="complex64", eps_rel=1e-3, eps_abs=1e-7),
}

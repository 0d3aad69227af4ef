"""Shared test helpers: golden fixtures and gate-list conversions."""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

_circuits = None
_states = None


def golden_circuits():
    global _circuits
    if _circuits is None:
        with open(os.path.join(GOLDEN, "reference_circuits.json")) as f:
            _circuits = json.load(f)
    return _circuits


def golden_states():
    global _states
    if _states is None:
        _states = dict(np.load(os.path.join(GOLDEN, "reference_states.npz")))
    return _states


def build_circuit(key: str):
    """Rebuild a golden circuit with the product's gate classes."""
    import qulacs
    from qulacs._gates import ControlQubitInfo, QuantumGateBase, TargetQubitInfo

    rec = golden_circuits()[key]
    c = qulacs.QuantumCircuit(rec["n"])
    for g in rec["gates"]:
        m = np.array(g["matrix_re"]) + 1j * np.array(g["matrix_im"])
        gate = QuantumGateBase(g["name"], [TargetQubitInfo(t, p) for t, p in zip(g["targets"], g["target_props"])],
                               [ControlQubitInfo(c_, v) for c_, v in zip(g["controls"], g["control_values"])],
                               m, g["gate_property"])
        c._gates.append(gate)
    return c


def optimized(circuit, block_size: int = 0):
    from qulacs.circuit import QuantumCircuitOptimizer
    c = circuit.copy()
    QuantumCircuitOptimizer(sv_block_size=block_size).optimize(c, block_size=2)
    return c


def fidelity(a: np.ndarray, b: np.ndarray) -> float:
    """|<a|b>| as script/run_sim.py:201-206 defines it (not squared)."""
    return float(abs(np.vdot(a, b)))


def random_circuit(n: int, ngates: int, seed: int, controlled: bool = True):
    """Seeded random circuit over every gate form the engine accepts."""
    import qulacs
    from qulacs import gate as G
    rng = np.random.default_rng(seed)
    c = qulacs.QuantumCircuit(n)

    def ru(k):
        z = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
        q, r = np.linalg.qr(z)
        return q * (np.diag(r) / np.abs(np.diag(r)))

    for _ in range(ngates):
        kind = rng.integers(0, 9 if controlled else 7)
        a, b = (int(x) for x in rng.choice(n, size=2, replace=False))
        if kind == 0:
            c.add_H_gate(a)
        elif kind == 1:
            c.add_RX_gate(a, rng.uniform(-3, 3))
        elif kind == 2:
            c.add_RZ_gate(a, rng.uniform(-3, 3))
        elif kind == 3:
            c.add_CNOT_gate(a, b)
        elif kind == 4:
            c.add_gate(G.DenseMatrix([a, b], ru(2)))
        elif kind == 5:
            c.add_gate(G.DenseMatrix(a, ru(1)))
        elif kind == 6:
            c.add_SWAP_gate(a, b)
        elif kind == 7:
            c.add_CZ_gate(a, b)
        else:
            g = G.DenseMatrix(a, ru(1))
            g.add_control_qubit(b, int(rng.integers(0, 2)))
            c.add_gate(g)
    return c


def perm_heavy_circuit(n, C, ngates, seed):
    """Random gates with many SWAP / X / CNOT gates on qubits >= C."""
    import qulacs
    from qulacs import gate as G
    rng = np.random.default_rng(seed)
    base = random_circuit(n, ngates, seed)
    c = qulacs.QuantumCircuit(n)
    hi = list(range(C, n))
    for g in base._gates:
        c.add_gate(g)
        r = rng.integers(0, 4)
        a, b = (int(x) for x in rng.choice(hi, size=2, replace=False))
        if r == 0:
            c.add_SWAP_gate(a, b)
        elif r == 1:
            c.add_X_gate(a)
        elif r == 2:
            c.add_CNOT_gate(a, b)      # a permutation, but not a bit move: stays a gate
        else:
            m = np.zeros((4, 4))
            f = [int(x) for x in rng.permutation(4)]
            for col, row in enumerate(f):
                m[row, col] = 1.0
            c.add_gate(G.DenseMatrix([a, b], m))
    return c

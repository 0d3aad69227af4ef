"""qulacs.gate: the gate factory (src/cppsim/gate_factory.cpp) restricted to
what the compressed-state path and its circuits use."""
from __future__ import annotations

import numpy as np

from .._gates import (ParametricPauliRotationGate, ParametricRotationGate, QuantumGateBase, QuantumGateMatrix, cnot,
                      cz, ibmq_matrix, merge, one_qubit_named, rotation, swap, to_matrix_gate)


def Identity(index: int) -> QuantumGateBase:
    return one_qubit_named("I", index)


def X(index: int) -> QuantumGateBase:
    return one_qubit_named("X", index)


def Y(index: int) -> QuantumGateBase:
    return one_qubit_named("Y", index)


def Z(index: int) -> QuantumGateBase:
    return one_qubit_named("Z", index)


def H(index: int) -> QuantumGateBase:
    return one_qubit_named("H", index)


def S(index: int) -> QuantumGateBase:
    return one_qubit_named("S", index)


def Sdag(index: int) -> QuantumGateBase:
    return one_qubit_named("Sdag", index)


def T(index: int) -> QuantumGateBase:
    return one_qubit_named("T", index)


def Tdag(index: int) -> QuantumGateBase:
    return one_qubit_named("Tdag", index)


def sqrtX(index: int) -> QuantumGateBase:
    return one_qubit_named("sqrtX", index)


def sqrtXdag(index: int) -> QuantumGateBase:
    return one_qubit_named("sqrtXdag", index)


def sqrtY(index: int) -> QuantumGateBase:
    return one_qubit_named("sqrtY", index)


def sqrtYdag(index: int) -> QuantumGateBase:
    return one_qubit_named("sqrtYdag", index)


def P0(index: int) -> QuantumGateBase:
    return one_qubit_named("Projection-0", index)


def P1(index: int) -> QuantumGateBase:
    return one_qubit_named("Projection-1", index)


def RX(index: int, angle: float) -> QuantumGateBase:
    return rotation("X", index, angle)


def RY(index: int, angle: float) -> QuantumGateBase:
    return rotation("Y", index, angle)


def RZ(index: int, angle: float) -> QuantumGateBase:
    return rotation("Z", index, angle)


# gate_factory.cpp:137-165: RotInv* = R*(angle), Rot* = R*(-angle)
def RotInvX(index: int, angle: float) -> QuantumGateBase:
    return rotation("X", index, angle)


def RotInvY(index: int, angle: float) -> QuantumGateBase:
    return rotation("Y", index, angle)


def RotInvZ(index: int, angle: float) -> QuantumGateBase:
    return rotation("Z", index, angle)


def RotX(index: int, angle: float) -> QuantumGateBase:
    return rotation("X", index, -angle)


def RotY(index: int, angle: float) -> QuantumGateBase:
    return rotation("Y", index, -angle)


def RotZ(index: int, angle: float) -> QuantumGateBase:
    return rotation("Z", index, -angle)


def U1(index: int, lam: float) -> QuantumGateMatrix:
    return QuantumGateMatrix([index], ibmq_matrix(0.0, 0.0, lam))


def U2(index: int, phi: float, lam: float) -> QuantumGateMatrix:
    return QuantumGateMatrix([index], ibmq_matrix(np.pi / 2, phi, lam))


def U3(index: int, theta: float, phi: float, lam: float) -> QuantumGateMatrix:
    return QuantumGateMatrix([index], ibmq_matrix(theta, phi, lam))


def CNOT(control: int, target: int) -> QuantumGateBase:
    return cnot(control, target)


def CZ(control: int, target: int) -> QuantumGateBase:
    return cz(control, target)


def SWAP(a: int, b: int) -> QuantumGateBase:
    return swap(a, b)


def DenseMatrix(targets, matrix) -> QuantumGateMatrix:
    if isinstance(targets, (int, np.integer)):
        targets = [int(targets)]
    targets = [int(t) for t in targets]
    if len(set(targets)) != len(targets):
        raise ValueError("target list contains duplicated values")
    return QuantumGateMatrix(targets, np.asarray(matrix, dtype=np.complex128))


def ParametricRX(index: int, angle: float = 0.0) -> ParametricRotationGate:
    return ParametricRotationGate("X", index, angle)


def ParametricRY(index: int, angle: float = 0.0) -> ParametricRotationGate:
    return ParametricRotationGate("Y", index, angle)


def ParametricRZ(index: int, angle: float = 0.0) -> ParametricRotationGate:
    return ParametricRotationGate("Z", index, angle)


def ParametricPauliRotation(targets, pauli_ids, angle: float = 0.0) -> ParametricPauliRotationGate:
    return ParametricPauliRotationGate(targets, pauli_ids, angle)


__all__ = [n for n in dir() if not n.startswith("_") and n not in ("np",)]

"""Gate model of the qulacs API on the compressed-state path.

Restates the parts of Qulacs' gate classes that decide what the compressed
engine sees: names, target/control lists, commutation flags and matrices.

* Commutation flags per target qubit (src/cppsim/qubit_info.hpp:7-11) and the
  commutation test (src/cppsim/gate.cpp:12-31, src/cppsim/qubit_info.cpp).
* Named one-qubit gates and their matrices
  (src/cppsim/gate_named_one.hpp:95-463), rotations with the Qulacs sign
  convention RX(t) = [[cos t/2, i sin t/2], [i sin t/2, cos t/2]]
  (gate_named_one.hpp:426-427), RZ(t) = diag(e^{i t/2}, e^{-i t/2}) (:462-463),
  and "RotX" = RX(-t) (src/cppsim/gate_factory.cpp:152-165).
* CNOT / CZ as one target + one control with a 2x2 matrix
  (src/cppsim/gate_named_two.hpp:188-224), SWAP as a 4x4 on two targets (:74-91).
* Dense matrix gates named "DenseMatrix" with commutation flags 0
  (src/cppsim/gate_matrix.cpp:16-30).
* Parametric rotations (src/vqcsim/parametric_gate.hpp:102-190).
Matrix index bit i corresponds to target_index_list[i] (little endian), as in
Qulacs' csim kernels.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence

import numpy as np

FLAG_X_COMMUTE = 0x01
FLAG_Y_COMMUTE = 0x02
FLAG_Z_COMMUTE = 0x04

FLAG_PAULI = 0x01
FLAG_CLIFFORD = 0x02
FLAG_GAUSSIAN = 0x04
FLAG_PARAMETRIC = 0x08


class TargetQubitInfo:
    __slots__ = ("index", "prop")

    def __init__(self, index: int, prop: int = 0):
        self.index = int(index)
        self.prop = int(prop)

    def commutes_with_target(self, other: "TargetQubitInfo") -> bool:
        # qubit_info.cpp: different qubits commute; same qubit commutes when
        # the two share a Pauli they both commute with.
        return self.index != other.index or (self.prop & other.prop) != 0

    def commutes_with_control(self, other: "ControlQubitInfo") -> bool:
        return self.index != other.index or (self.prop & FLAG_Z_COMMUTE) != 0

    def __repr__(self):
        return f"T({self.index},{self.prop})"


class ControlQubitInfo:
    __slots__ = ("index", "value")

    def __init__(self, index: int, value: int = 1):
        self.index = int(index)
        self.value = int(value)

    def __repr__(self):
        return f"C({self.index},{self.value})"


class QuantumGateBase:
    """Base of every gate: name, qubit infos, matrix and property bits."""

    def __init__(self, name: str, targets: Sequence[TargetQubitInfo],
                 controls: Sequence[ControlQubitInfo], matrix: np.ndarray,
                 gate_property: int = 0):
        self._name = name
        self.target_qubit_list: List[TargetQubitInfo] = list(targets)
        self.control_qubit_list: List[ControlQubitInfo] = list(controls)
        self._matrix = np.array(matrix, dtype=np.complex128)
        self._gate_property = int(gate_property)

    # --- qulacs accessors -------------------------------------------------
    def get_name(self) -> str:
        return self._name

    def set_name(self, name: str) -> None:
        self._name = name

    def get_target_index_list(self) -> List[int]:
        return [t.index for t in self.target_qubit_list]

    def get_control_index_list(self) -> List[int]:
        return [c.index for c in self.control_qubit_list]

    def get_control_value_list(self) -> List[int]:
        return [c.value for c in self.control_qubit_list]

    def get_matrix(self) -> np.ndarray:
        return self._matrix.copy()

    def get_property_value(self) -> int:
        return self._gate_property

    def is_parametric(self) -> bool:
        return (self._gate_property & FLAG_PARAMETRIC) != 0

    def is_diagonal(self) -> bool:
        return all(t.prop & FLAG_Z_COMMUTE for t in self.target_qubit_list)

    def is_commute(self, other: "QuantumGateBase") -> bool:
        """gate.cpp:12-31 -- target/target, target/control, control/target."""
        for a in self.target_qubit_list:
            for b in other.target_qubit_list:
                if not a.commutes_with_target(b):
                    return False
            for b in other.control_qubit_list:
                if not a.commutes_with_control(b):
                    return False
        for a in self.control_qubit_list:
            for b in other.target_qubit_list:
                if not b.commutes_with_control(a):
                    return False
        return True

    def copy(self) -> "QuantumGateBase":
        g = QuantumGateBase.__new__(type(self))
        g.__dict__.update(self.__dict__)
        g.target_qubit_list = [TargetQubitInfo(t.index, t.prop) for t in self.target_qubit_list]
        g.control_qubit_list = [ControlQubitInfo(c.index, c.value) for c in self.control_qubit_list]
        g._matrix = self._matrix.copy()
        return g

    def get_inverse(self) -> "QuantumGateBase":
        g = self.copy()
        if hasattr(g, "_angle") and hasattr(g, "set_parameter_value"):
            g.set_parameter_value(-self._angle)
        else:
            g._matrix = self.get_matrix().conj().T.copy()
        return g

    def update_quantum_state(self, state) -> None:
        state._apply_gates([self])

    def full_qubits(self) -> List[int]:
        return self.get_target_index_list() + self.get_control_index_list()

    def __repr__(self):
        return (f"{self._name}(targets={self.get_target_index_list()}, "
                f"controls={self.get_control_index_list()})")

    __str__ = __repr__


class QuantumGateMatrix(QuantumGateBase):
    """Dense matrix gate; name "DenseMatrix" (gate_matrix.cpp:16-30)."""

    def __init__(self, targets, matrix, controls=None, gate_property: int = 0):
        tl = [t if isinstance(t, TargetQubitInfo) else TargetQubitInfo(t, 0) for t in targets]
        cl = [c if isinstance(c, ControlQubitInfo) else ControlQubitInfo(c, 1) for c in (controls or [])]
        m = np.asarray(matrix, dtype=np.complex128)
        if m.shape != (1 << len(tl), 1 << len(tl)):
            raise ValueError("matrix size does not match the number of targets")
        super().__init__("DenseMatrix", tl, cl, m, gate_property)

    def add_control_qubit(self, index: int, control_value: int) -> None:
        self.control_qubit_list.append(ControlQubitInfo(index, control_value))


class ParametricRotationGate(QuantumGateBase):
    """ParametricRX/RY/RZ (src/vqcsim/parametric_gate.hpp:102-190)."""

    _AXIS_PROP = {"X": FLAG_X_COMMUTE, "Y": FLAG_Y_COMMUTE, "Z": FLAG_Z_COMMUTE}

    def __init__(self, axis: str, target: int, angle: float):
        self._axis = axis
        self._angle = float(angle)
        super().__init__("Parametric R" + axis, [TargetQubitInfo(target, self._AXIS_PROP[axis])],
                         [], _rotation_matrix(axis, angle), FLAG_PARAMETRIC)
        self._name = "ParametricR" + axis

    def get_parameter_value(self) -> float:
        return self._angle

    def set_parameter_value(self, value: float) -> None:
        self._angle = float(value)
        self._matrix = _rotation_matrix(self._axis, self._angle)

    def get_matrix(self) -> np.ndarray:
        return _rotation_matrix(self._axis, self._angle)

    @property
    def axis(self) -> str:
        return self._axis

    def generator_masks(self):
        """(flip mask, sign mask, #Y) of the generator P of exp(i theta/2 P)."""
        q = 1 << self.get_target_index_list()[0]
        return {"X": (q, 0, 0), "Y": (q, q, 1), "Z": (0, q, 0)}[self._axis]


_PAULI_1Q = {
    1: np.array([[0, 1], [1, 0]], dtype=np.complex128),
    2: np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
    3: np.array([[1, 0], [0, -1]], dtype=np.complex128),
}
_PAULI_PROP = {1: FLAG_X_COMMUTE, 2: FLAG_Y_COMMUTE, 3: FLAG_Z_COMMUTE}


def pauli_matrix(pauli_ids) -> np.ndarray:
    """Matrix of a Pauli string; matrix bit i <-> the i-th listed qubit."""
    m = np.eye(1, dtype=np.complex128)
    for pid in pauli_ids:
        m = np.kron(_PAULI_1Q[int(pid)], m)
    return m


class ParametricPauliRotationGate(QuantumGateBase):
    """exp(i theta/2 P) for a Pauli string P (src/vqcsim/parametric_gate.hpp:213+,
    matrix cos(theta/2) I + i sin(theta/2) P as src/cppsim/gate_named_pauli.hpp:221-226)."""

    def __init__(self, targets, pauli_ids, angle: float):
        self._pids = [int(p) for p in pauli_ids]
        if len(self._pids) != len(targets) or any(p not in (1, 2, 3) for p in self._pids):
            raise ValueError("pauli_ids must list 1 (X), 2 (Y) or 3 (Z) per target")
        self._angle = float(angle)
        tl = [TargetQubitInfo(t, _PAULI_PROP[p]) for t, p in zip(targets, self._pids)]
        super().__init__("ParametricPauliRotation", tl, [], self._mat(), FLAG_PARAMETRIC)

    def _mat(self):
        P = pauli_matrix(self._pids)
        c, s_ = math.cos(self._angle / 2), math.sin(self._angle / 2)
        return c * np.eye(P.shape[0], dtype=np.complex128) + 1j * s_ * P

    def get_parameter_value(self) -> float:
        return self._angle

    def set_parameter_value(self, value: float) -> None:
        self._angle = float(value)
        self._matrix = self._mat()

    def get_matrix(self) -> np.ndarray:
        return self._mat()

    def generator_masks(self):
        xm = zm = ny = 0
        for t, p in zip(self.get_target_index_list(), self._pids):
            if p in (1, 2):
                xm |= 1 << t
            if p in (2, 3):
                zm |= 1 << t
            ny += p == 2
        return xm, zm, ny


def _rotation_matrix(axis: str, angle: float) -> np.ndarray:
    c, s = math.cos(angle / 2), math.sin(angle / 2)
    if axis == "X":
        return np.array([[c, 1j * s], [1j * s, c]], dtype=np.complex128)
    if axis == "Y":
        return np.array([[c, s], [-s, c]], dtype=np.complex128)
    if axis == "Z":
        return np.array([[c + 1j * s, 0], [0, c - 1j * s]], dtype=np.complex128)
    raise ValueError(axis)


_SQ2 = 1.0 / math.sqrt(2.0)
_ONE_QUBIT = {
    # name: (matrix, commutation flag, gate property)
    "I": ([[1, 0], [0, 1]], FLAG_X_COMMUTE | FLAG_Y_COMMUTE | FLAG_Z_COMMUTE,
          FLAG_PAULI | FLAG_CLIFFORD | FLAG_GAUSSIAN),
    "X": ([[0, 1], [1, 0]], FLAG_X_COMMUTE, FLAG_PAULI | FLAG_CLIFFORD),
    "Y": ([[0, -1j], [1j, 0]], FLAG_Y_COMMUTE, FLAG_PAULI | FLAG_CLIFFORD),
    "Z": ([[1, 0], [0, -1]], FLAG_Z_COMMUTE, FLAG_PAULI | FLAG_CLIFFORD | FLAG_GAUSSIAN),
    "H": ([[_SQ2, _SQ2], [_SQ2, -_SQ2]], 0, FLAG_CLIFFORD),
    "S": ([[1, 0], [0, 1j]], FLAG_Z_COMMUTE, FLAG_CLIFFORD | FLAG_GAUSSIAN),
    "Sdag": ([[1, 0], [0, -1j]], FLAG_Z_COMMUTE, FLAG_CLIFFORD | FLAG_GAUSSIAN),
    "T": ([[1, 0], [0, (1 + 1j) * _SQ2]], FLAG_Z_COMMUTE, FLAG_GAUSSIAN),
    "Tdag": ([[1, 0], [0, (1 - 1j) * _SQ2]], FLAG_Z_COMMUTE, FLAG_GAUSSIAN),
    "sqrtX": ([[0.5 + 0.5j, 0.5 - 0.5j], [0.5 - 0.5j, 0.5 + 0.5j]], FLAG_X_COMMUTE, FLAG_CLIFFORD),
    "sqrtXdag": ([[0.5 - 0.5j, 0.5 + 0.5j], [0.5 + 0.5j, 0.5 - 0.5j]], FLAG_X_COMMUTE, FLAG_CLIFFORD),
    "sqrtY": ([[0.5 + 0.5j, -0.5 - 0.5j], [0.5 + 0.5j, 0.5 + 0.5j]], FLAG_Y_COMMUTE, FLAG_CLIFFORD),
    "sqrtYdag": ([[0.5 - 0.5j, 0.5 - 0.5j], [-0.5 + 0.5j, 0.5 - 0.5j]], FLAG_Y_COMMUTE, FLAG_CLIFFORD),
    "Projection-0": ([[1, 0], [0, 0]], 0, FLAG_CLIFFORD | FLAG_GAUSSIAN),
    "Projection-1": ([[0, 0], [0, 1]], 0, FLAG_CLIFFORD | FLAG_GAUSSIAN),
}


def one_qubit_named(name: str, target: int) -> QuantumGateBase:
    mat, prop, gprop = _ONE_QUBIT[name]
    return QuantumGateBase(name, [TargetQubitInfo(target, prop)], [], np.array(mat, dtype=np.complex128), gprop)


_ROT_NAME = {"X": "X-rotation", "Y": "Y-rotation", "Z": "Z-rotation"}


def rotation(axis: str, target: int, angle: float) -> QuantumGateBase:
    prop = ParametricRotationGate._AXIS_PROP[axis]
    return QuantumGateBase(_ROT_NAME[axis], [TargetQubitInfo(target, prop)], [],
                           _rotation_matrix(axis, angle), 0)


def cnot(control: int, target: int) -> QuantumGateBase:
    if control == target:
        raise ValueError("CNOT: control and target must differ")
    return QuantumGateBase("CNOT", [TargetQubitInfo(target, FLAG_X_COMMUTE)], [ControlQubitInfo(control, 1)],
                           np.array([[0, 1], [1, 0]], dtype=np.complex128), FLAG_CLIFFORD)


def cz(control: int, target: int) -> QuantumGateBase:
    if control == target:
        raise ValueError("CZ: control and target must differ")
    return QuantumGateBase("CZ", [TargetQubitInfo(target, FLAG_Z_COMMUTE)], [ControlQubitInfo(control, 1)],
                           np.array([[1, 0], [0, -1]], dtype=np.complex128), FLAG_CLIFFORD)


def swap(a: int, b: int) -> QuantumGateBase:
    if a == b:
        raise ValueError("SWAP: qubits must differ")
    m = np.zeros((4, 4), dtype=np.complex128)
    m[0, 0] = m[1, 2] = m[2, 1] = m[3, 3] = 1
    return QuantumGateBase("SWAP", [TargetQubitInfo(a, 0), TargetQubitInfo(b, 0)], [], m, FLAG_CLIFFORD)


def ibmq_matrix(theta: float, phi: float, lam: float) -> np.ndarray:
    """U3 matrix as gate_factory.cpp:168-181 builds it."""
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    e1, e2 = np.exp(1j * phi), np.exp(1j * lam)
    return np.array([[c, -e2 * s], [e1 * s, e1 * e2 * c]], dtype=np.complex128)


# ---------------------------------------------------------------------------
# gate::merge (src/cppsim/gate_merge.cpp:19-356)
# ---------------------------------------------------------------------------

def _find(lst, index):
    for x in lst:
        if x.index == index:
            return x
    return None


def _new_qubit_list(g1: QuantumGateBase, g2: QuantumGateBase):
    """The nine-case classification of gate_merge.cpp:19-149."""
    new_t: List[TargetQubitInfo] = []
    new_c: List[ControlQubitInfo] = []
    for t1 in g1.target_qubit_list:
        t2 = _find(g2.target_qubit_list, t1.index)
        if t2 is not None:                                   # case 0
            new_t.append(TargetQubitInfo(t1.index, t1.prop & t2.prop))
            continue
        if _find(g2.control_qubit_list, t1.index) is not None:  # case 1
            new_t.append(TargetQubitInfo(t1.index, t1.prop & FLAG_Z_COMMUTE))
            continue
        new_t.append(TargetQubitInfo(t1.index, t1.prop))       # case 2
    for c1 in g1.control_qubit_list:
        t2 = _find(g2.target_qubit_list, c1.index)
        if t2 is not None:                                   # case 3
            new_t.append(TargetQubitInfo(c1.index, t2.prop & FLAG_Z_COMMUTE))
            continue
        c2 = _find(g2.control_qubit_list, c1.index)
        if c2 is not None:                                   # case 4
            if c1.value == c2.value:
                new_c.append(ControlQubitInfo(c1.index, c1.value))
            else:
                new_t.append(TargetQubitInfo(c1.index, FLAG_Z_COMMUTE))
            continue
        new_t.append(TargetQubitInfo(c1.index, FLAG_Z_COMMUTE))  # case 5
    for t2 in g2.target_qubit_list:
        if _find(g1.target_qubit_list, t2.index) is not None or _find(g1.control_qubit_list, t2.index) is not None:
            continue
        new_t.append(TargetQubitInfo(t2.index, t2.prop))       # case 6
    for c2 in g2.control_qubit_list:
        if _find(g1.target_qubit_list, c2.index) is not None or _find(g1.control_qubit_list, c2.index) is not None:
            continue
        new_t.append(TargetQubitInfo(c2.index, FLAG_Z_COMMUTE))  # case 7
    return new_t, new_c


def permute_matrix_qubits(mat: np.ndarray, order: Sequence[int], new_order: Sequence[int]) -> np.ndarray:
    """Re-express a matrix whose index bit i belongs to qubit order[i] in the
    basis where index bit j belongs to qubit new_order[j]."""
    k = len(order)
    if list(order) == list(new_order):
        return mat
    # reshape: numpy's axis 0 is the most significant bit -> bit k-1
    t = mat.reshape([2] * (2 * k))
    pos = {q: i for i, q in enumerate(order)}
    # new axis for bit j (most significant first) comes from old bit pos[new_order[j]]
    row_axes = [k - 1 - pos[new_order[j]] for j in reversed(range(k))]
    col_axes = [k + a for a in row_axes]
    return t.transpose(row_axes + col_axes).reshape(1 << k, 1 << k)


def _extended_matrix(g: QuantumGateBase, new_t: List[TargetQubitInfo]) -> np.ndarray:
    """gate_merge.cpp:153-308: embed g into the merged target list."""
    a_list = g.get_target_index_list()
    b_list, control_mask = [], 0
    for t in new_t:
        c = _find(g.control_qubit_list, t.index)
        if c is not None:
            b_list.append(t.index)
            if c.value == 1:
                control_mask ^= 1 << (len(b_list) - 1)
    c_list = [t.index for t in new_t
              if _find(g.target_qubit_list, t.index) is None and _find(g.control_qubit_list, t.index) is None]
    unsorted = a_list + c_list + b_list
    dim = 1 << len(new_t)
    mat = np.eye(dim, dtype=np.complex128)
    start = (1 << (len(a_list) + len(c_list))) * control_mask
    org = g.get_matrix()
    od = 1 << len(a_list)
    for r in range(1 << len(c_list)):
        p = start + r * od
        mat[p:p + od, p:p + od] = org
    return permute_matrix_qubits(mat, unsorted, sorted(unsorted))


def merge(g1: QuantumGateBase, g2: QuantumGateBase) -> QuantumGateMatrix:
    """gate::merge(first, second): the product second*first on the union."""
    if isinstance(g1, (list, tuple)):
        gates = list(g1)
        out = to_matrix_gate(gates[0])
        for g in gates[1:]:
            out = merge(out, g)
        return out
    new_t, new_c = _new_qubit_list(g1, g2)
    new_t.sort(key=lambda t: t.index)
    new_c.sort(key=lambda c: c.index)
    m1 = _extended_matrix(g1, new_t)
    m2 = _extended_matrix(g2, new_t)
    g = QuantumGateMatrix(new_t, m2 @ m1, new_c)
    g._gate_property = g1.get_property_value() & g2.get_property_value()
    return g


def to_matrix_gate(g: QuantumGateBase) -> QuantumGateMatrix:
    """gate_merge.cpp:428-433: same qubit infos, name "DenseMatrix"."""
    return QuantumGateMatrix([TargetQubitInfo(t.index, t.prop) for t in g.target_qubit_list], g.get_matrix(),
                             [ControlQubitInfo(c.index, c.value) for c in g.control_qubit_list])


def full_matrix(g: QuantumGateBase, qubits: Optional[Sequence[int]] = None):
    """Matrix of g over `qubits` (default: sorted targets+controls), with the
    controls folded in.  Index bit i <-> qubits[i]."""
    tq = g.get_target_index_list()
    cq = g.get_control_index_list()
    allq = tq + cq
    nt, nc = len(tq), len(cq)
    dim = 1 << (nt + nc)
    m = np.eye(dim, dtype=np.complex128)
    cmask = 0
    for i, c in enumerate(g.control_qubit_list):
        if c.value:
            cmask |= 1 << i
    base = cmask << nt
    od = 1 << nt
    m[base:base + od, base:base + od] = g.get_matrix()
    order = sorted(allq) if qubits is None else list(qubits)
    return permute_matrix_qubits(m, allq, order), order

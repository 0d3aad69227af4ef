"""qulacs -- the Python surface of the B200 compressed state-vector engine.

Mirrors the parts of the qulacs / QompSim API that the compressed-state path
uses (python/cppsim_wrapper.cpp:347-516, 624-628, 1287-1420, 1706-1715 of the
reference) so that scripts written for the reference (script/run_sim.py,
benchmark/circuit_factory.py) run unchanged on one GPU:

* QuantumState(n)            -- uncompressed state vector on the device
* QuantumCircuit(n)          -- gate list, update_quantum_state(state)
* CompressedQuantumState(n, block_size) -- the block-wise compressed state
* circuit.QuantumCircuitOptimizer        -- gate fusion (optimize)
* gate.*                     -- gate factory
* check_build_for_mpi()      -- False: one GPU, no MPI ranks

Device work goes through the C ABI of libqompsim.so (qulacs/_native.py).
There is no CPU execution path: without the library or a CUDA device every
state constructor raises.
"""
from __future__ import annotations

import os
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _native as _n
from ._gates import (ControlQubitInfo, ParametricRotationGate, QuantumGateBase, QuantumGateMatrix,
                     TargetQubitInfo, merge, to_matrix_gate)
from . import gate as gate  # noqa: F401  (qulacs.gate)
from . import circuit as circuit  # noqa: F401  (qulacs.circuit)

__version__ = "0.1.0-b200"

QompsimError = _n.QompsimError


def check_build_for_mpi() -> bool:
    """python/cppsim_wrapper.cpp:624-628: this build has no MPI ranks."""
    return False


# =====================================================================
# circuits
# =====================================================================
class QuantumCircuit:
    """Gate list of a circuit (src/cppsim/circuit.hpp).  add_gate copies the
    gate, get_gate returns a copy, as the reference binding does."""

    def __init__(self, qubit_count: int):
        self._n = int(qubit_count)
        self._gates: List[QuantumGateBase] = []

    # ---- structure
    def get_qubit_count(self) -> int:
        return self._n

    def get_gate_count(self) -> int:
        return len(self._gates)

    def get_gate(self, index: int) -> QuantumGateBase:
        return self._gates[index].copy()

    def get_gate_list(self) -> List[QuantumGateBase]:
        return [g.copy() for g in self._gates]

    def _check(self, g: QuantumGateBase) -> None:
        for q in g.full_qubits():
            if q < 0 or q >= self._n:
                raise ValueError(f"gate {g.get_name()} acts on qubit {q} outside a {self._n}-qubit circuit")

    def add_gate(self, gate: QuantumGateBase, position: Optional[int] = None) -> None:
        self._check(gate)
        g = gate.copy()
        if position is None:
            self._gates.append(g)
        else:
            self._gates.insert(position, g)

    def remove_gate(self, index: int) -> None:
        del self._gates[index]

    def copy(self) -> "QuantumCircuit":
        c = type(self).__new__(type(self))
        c.__dict__.update(self.__dict__)
        c._gates = [g.copy() for g in self._gates]
        return c

    def update_quantum_state(self, state, start: int = 0, end: Optional[int] = None) -> None:
        """QuantumCircuit::update_quantum_state (src/cppsim/circuit.cpp:23-34)."""
        gates = self._gates[start:end]
        state._apply_gates(gates)

    # ---- add_*_gate (cppsim_wrapper.cpp:1287-1420)
    def add_X_gate(self, i): self.add_gate(gate.X(i))
    def add_Y_gate(self, i): self.add_gate(gate.Y(i))
    def add_Z_gate(self, i): self.add_gate(gate.Z(i))
    def add_H_gate(self, i): self.add_gate(gate.H(i))
    def add_S_gate(self, i): self.add_gate(gate.S(i))
    def add_Sdag_gate(self, i): self.add_gate(gate.Sdag(i))
    def add_T_gate(self, i): self.add_gate(gate.T(i))
    def add_Tdag_gate(self, i): self.add_gate(gate.Tdag(i))
    def add_sqrtX_gate(self, i): self.add_gate(gate.sqrtX(i))
    def add_sqrtXdag_gate(self, i): self.add_gate(gate.sqrtXdag(i))
    def add_sqrtY_gate(self, i): self.add_gate(gate.sqrtY(i))
    def add_sqrtYdag_gate(self, i): self.add_gate(gate.sqrtYdag(i))
    def add_P0_gate(self, i): self.add_gate(gate.P0(i))
    def add_P1_gate(self, i): self.add_gate(gate.P1(i))
    def add_RX_gate(self, i, angle): self.add_gate(gate.RX(i, angle))
    def add_RY_gate(self, i, angle): self.add_gate(gate.RY(i, angle))
    def add_RZ_gate(self, i, angle): self.add_gate(gate.RZ(i, angle))
    def add_RotInvX_gate(self, i, angle): self.add_gate(gate.RotInvX(i, angle))
    def add_RotInvY_gate(self, i, angle): self.add_gate(gate.RotInvY(i, angle))
    def add_RotInvZ_gate(self, i, angle): self.add_gate(gate.RotInvZ(i, angle))
    def add_RotX_gate(self, i, angle): self.add_gate(gate.RotX(i, angle))
    def add_RotY_gate(self, i, angle): self.add_gate(gate.RotY(i, angle))
    def add_RotZ_gate(self, i, angle): self.add_gate(gate.RotZ(i, angle))
    def add_U1_gate(self, i, lam): self.add_gate(gate.U1(i, lam))
    def add_U2_gate(self, i, phi, lam): self.add_gate(gate.U2(i, phi, lam))
    def add_U3_gate(self, i, theta, phi, lam): self.add_gate(gate.U3(i, theta, phi, lam))
    def add_CNOT_gate(self, c, t): self.add_gate(gate.CNOT(c, t))
    def add_CZ_gate(self, c, t): self.add_gate(gate.CZ(c, t))
    def add_SWAP_gate(self, a, b): self.add_gate(gate.SWAP(a, b))

    def add_dense_matrix_gate(self, targets, matrix):
        self.add_gate(gate.DenseMatrix(targets, matrix))

    def __repr__(self):
        return f"QuantumCircuit(qubits={self._n}, gates={len(self._gates)})"


class ParametricQuantumCircuit(QuantumCircuit):
    """Circuit with parametric rotations (src/vqcsim/parametric_circuit.hpp)."""

    def __init__(self, qubit_count: int):
        super().__init__(qubit_count)
        self._param_pos: List[int] = []

    def copy(self):
        c = super().copy()
        c._param_pos = list(self._param_pos)
        return c

    def _add_param(self, g):
        self._param_pos.append(len(self._gates))
        self._check(g)
        self._gates.append(g.copy())

    def add_parametric_multi_Pauli_rotation_gate(self, targets, pauli_ids, angle):
        self._add_param(gate.ParametricPauliRotation(targets, pauli_ids, angle))

    def add_parametric_RX_gate(self, i, angle): self._add_param(gate.ParametricRX(i, angle))
    def add_parametric_RY_gate(self, i, angle): self._add_param(gate.ParametricRY(i, angle))
    def add_parametric_RZ_gate(self, i, angle): self._add_param(gate.ParametricRZ(i, angle))

    def add_gate(self, g, position=None):
        if position is not None and position < len(self._gates):
            self._param_pos = [p + 1 if p >= position else p for p in self._param_pos]
        super().add_gate(g, position)
        if g.is_parametric():
            self._param_pos.append(len(self._gates) - 1 if position is None else position)
            self._param_pos.sort()

    def remove_gate(self, index: int):
        self._param_pos = [p - (1 if p > index else 0) for p in self._param_pos if p != index]
        super().remove_gate(index)

    def get_parameter_count(self) -> int:
        return len(self._param_pos)

    def get_parameter(self, i: int) -> float:
        return self._gates[self._param_pos[i]].get_parameter_value()

    def set_parameter(self, i: int, value: float) -> None:
        self._gates[self._param_pos[i]].set_parameter_value(value)

    def get_parametric_gate_position(self, i: int) -> int:
        return self._param_pos[i]


# =====================================================================
# observables
# =====================================================================
_PAULI_IDS = {"I": 0, "X": 1, "Y": 2, "Z": 3}


def _parse_pauli(pauli: str):
    """'X 0 Z 3 Y 5' -> (x_mask, z_mask, number of Y factors)."""
    tok = pauli.split()
    if len(tok) % 2:
        raise ValueError(f"malformed Pauli string {pauli!r}")
    xm = zm = ny = 0
    for a, b in zip(tok[0::2], tok[1::2]):
        p, q = a.upper(), int(b)
        if p not in _PAULI_IDS:
            raise ValueError(f"unknown Pauli {a!r}")
        bit = 1 << q
        if (xm | zm) & bit:
            raise ValueError(f"qubit {q} appears twice in {pauli!r}")
        if p in ("X", "Y"):
            xm |= bit
        if p in ("Z", "Y"):
            zm |= bit
        ny += p == "Y"
    return xm, zm, ny


class Observable:
    """A sum of Pauli strings with real coefficients (src/cppsim/observable.hpp).

    get_expectation_value(state) evaluates every term on the device with FP64
    accumulation (qs_expectation_pauli / qs_dense_expectation_pauli).  On a
    CompressedQuantumState the value is divided by the state's squared norm,
    as the reference renormalises the compressed state on readout."""

    def __init__(self, qubit_count: int):
        self._n = int(qubit_count)
        self._terms: List[tuple] = []   # (coef, x_mask, z_mask, ny, text)

    def add_operator(self, coef, pauli: str) -> None:
        xm, zm, ny = _parse_pauli(pauli)
        if (xm | zm) >> self._n:
            raise ValueError("Pauli string acts outside the observable's qubits")
        self._terms.append((complex(coef), xm, zm, ny, pauli))

    def get_term_count(self) -> int:
        return len(self._terms)

    def get_qubit_count(self) -> int:
        return self._n

    def term_masks(self):
        return ([t[1] for t in self._terms], [t[2] for t in self._terms], [t[3] for t in self._terms],
                [t[0] for t in self._terms])

    def get_term_values(self, state) -> np.ndarray:
        """<P_t> for every term (complex, without coefficients)."""
        xs, zs, nys, _ = self.term_masks()
        sums = state._pauli_sums(xs + [0], zs + [0])
        norm = sums[-1].real if isinstance(state, CompressedQuantumState) else 1.0
        return np.array([(1j ** ny) * v / norm for ny, v in zip(nys, sums[:-1])])

    def get_expectation_value(self, state) -> float:
        vals = self.get_term_values(state)
        coefs = np.array([t[0] for t in self._terms])
        return float(np.real(np.sum(coefs * vals)))


def _pauli_sums(fn, handle, checker, xs, zs):
    n = len(xs)
    xa = np.ascontiguousarray(np.asarray(xs, dtype=np.uint64))
    za = np.ascontiguousarray(np.asarray(zs, dtype=np.uint64))
    out = np.zeros(2 * max(1, n), dtype=np.float64)
    checker(fn(handle, xa.ctypes.data_as(_n.ct.POINTER(_n.ct.c_uint64)), za.ctypes.data_as(_n.ct.POINTER(_n.ct.c_uint64)),
               n, out.ctypes.data_as(_n.ct.POINTER(_n.ct.c_double))))
    return out[0:2 * n:2] + 1j * out[1:2 * n:2]


# =====================================================================
# uncompressed state
# =====================================================================
class QuantumState:
    """QuantumState(n) -- an uncompressed complex128 (or, with
    QOMPSIM_DTYPE=complex64, complex64) state vector in device memory,
    initialised to |0...0>.  update_quantum_state runs fused tile passes."""

    def __init__(self, qubit_count: int, use_multi_cpu: bool = False, dtype=None):
        L = _n.lib()
        self._n = int(qubit_count)
        self._dtype = _n.env_dtype() if dtype is None else _n.dtype_code(dtype)
        h = _n.ct.c_void_p()
        _n.check(L.qs_dense_create(_n.ct.byref(h), self._n, self._dtype), None, dense=True)
        self._h = h
        self._pergate = os.environ.get("QOMPSIM_PERGATE", "0") == "1"

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _n.lib().qs_dense_destroy(h)
            except Exception:
                pass
            self._h = None

    def _check(self, st):
        _n.check(st, self._h, dense=True)

    def get_qubit_count(self) -> int:
        return self._n

    def get_fused_swap_time(self) -> float:
        return 0.0

    def set_zero_state(self) -> None:
        self._check(_n.lib().qs_dense_set_basis_state(self._h, 0))

    def set_computational_basis(self, basis: int) -> None:
        self._check(_n.lib().qs_dense_set_basis_state(self._h, int(basis)))

    def load(self, vec) -> None:
        v = np.ascontiguousarray(np.asarray(vec, dtype=np.complex128).reshape(-1))
        if v.size != 1 << self._n:
            raise ValueError("vector length must be 2^n")
        self._check(_n.lib().qs_dense_set_vector(self._h, v.view(np.float64).ctypes.data_as(_n.ct.POINTER(_n.ct.c_double))))

    def get_vector(self) -> np.ndarray:
        out = np.empty(1 << self._n, dtype=np.complex128)
        self._check(_n.lib().qs_dense_get_vector(self._h, out.view(np.float64).ctypes.data_as(_n.ct.POINTER(_n.ct.c_double))))
        return out

    def get_amplitudes(self, first: int, count: int) -> np.ndarray:
        """Amplitudes [first, first + count) as complex128."""
        out = np.empty(int(count), dtype=np.complex128)
        self._check(_n.lib().qs_dense_get_amplitudes(self._h, int(first), int(count),
                                                     out.view(np.float64).ctypes.data_as(_n.ct.POINTER(_n.ct.c_double))))
        return out

    def get_amplitudes_to(self, address: int, first: int, count: int) -> None:
        """get_amplitudes written as 2*count interleaved doubles at `address`
        (host memory or device memory of the state's GPU)."""
        self._check(_n.lib().qs_dense_get_amplitudes(self._h, int(first), int(count),
                                                     _n.ct.cast(_n.ct.c_void_p(int(address)),
                                                                _n.ct.POINTER(_n.ct.c_double))))

    def get_squared_norm(self) -> float:
        v = _n.ct.c_double()
        self._check(_n.lib().qs_dense_norm_squared(self._h, _n.ct.byref(v)))
        return v.value

    def _apply_gates(self, gates: Sequence[QuantumGateBase], pergate: Optional[bool] = None) -> None:
        if not gates:
            return
        arr = _n.make_gate_array(list(gates))
        fn = _n.lib().qs_dense_apply_gates_pergate if (self._pergate if pergate is None else pergate) \
            else _n.lib().qs_dense_apply_gates
        self._check(fn(self._h, arr, len(gates)))

    def _pauli_sums(self, xs, zs):
        return _pauli_sums(_n.lib().qs_dense_expectation_pauli, self._h, self._check, xs, zs)

    def device_pointer(self) -> int:
        p = _n.ct.c_void_p()
        self._check(_n.lib().qs_dense_device_ptr(self._h, _n.ct.byref(p)))
        return p.value

    def __repr__(self):
        return f"QuantumState(qubits={self._n})"


# =====================================================================
# compressed state
# =====================================================================
_TIMER_KEYS = ["decomp", "gate", "comp", "fused_swap", "allgather", "hmalloc", "dmalloc", "h2d", "d2h", "dfree"]


def _env_float(name: str, default: float) -> float:
    v = os.environ.get(name)
    return float(v) if v is not None else default


class CompressedQuantumState:
    """CompressedQuantumState(qubit_count, block_size) (compressed_state.hpp:87-239).

    Error bounds come from BITCOMP_REL_EB (default 1e-3) and BITCOMP_ABS_EB
    (default 1e-7) at construction, as in the reference.  QOMPSIM_DTYPE picks
    complex128 (default) or complex64.  QOMPSIM_ZERO_TEST=exact selects the
    reference GPU build's exact zero-block test (default: all codes zero);
    QOMPSIM_REFERENCE_CONTROLS=1 reproduces the reference's control handling.
    host_store=True (or QOMPSIM_HOST_STORE=1) keeps the compressed payload in
    pinned host memory that the device passes stream over the bus: the
    spill tier for stores larger than HBM."""

    def __init__(self, qubit_count: int, block_size: int, dtype=None, eps_rel: Optional[float] = None,
                 eps_abs: Optional[float] = None, flags: Optional[int] = None, host_store: bool = False):
        L = _n.lib()
        self._n = int(qubit_count)
        self._B = int(block_size)
        self._dtype = _n.env_dtype() if dtype is None else _n.dtype_code(dtype)
        self._eps_rel = _env_float("BITCOMP_REL_EB", 1e-3) if eps_rel is None else float(eps_rel)
        self._eps_abs = _env_float("BITCOMP_ABS_EB", 1e-7) if eps_abs is None else float(eps_abs)
        if flags is None:
            flags = 0
            if os.environ.get("QOMPSIM_ZERO_TEST", "code") == "exact":
                flags |= _n.QS_FLAG_EXACT_ZERO_TEST
            if os.environ.get("QOMPSIM_REFERENCE_CONTROLS", "0") == "1":
                flags |= _n.QS_FLAG_REFERENCE_CONTROLS
            if os.environ.get("QOMPSIM_QUIET", "0") == "1":
                flags |= _n.QS_FLAG_QUIET
        if host_store:
            flags |= _n.QS_FLAG_HOST_STORE
        self._flags = int(flags)
        h = _n.ct.c_void_p()
        _n.check(L.qs_create(_n.ct.byref(h), self._n, self._B, self._dtype, self._eps_rel, self._eps_abs,
                             self._flags), None)
        self._h = h
        self._gates: List[QuantumGateBase] = []

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _n.lib().qs_destroy(h)
            except Exception:
                pass
            self._h = None

    def _check(self, st):
        _n.check(st, self._h)

    # ---- geometry
    def get_qubit_count(self) -> int:
        return self._n

    @property
    def block_size(self) -> int:
        return self._B

    @property
    def nblocks(self) -> int:
        return 1 << (self._n - self._B)

    def print_info(self) -> None:
        print(f" block_size: {self._B}")
        print(f" namps_per_block: {1 << self._B}")
        print(f" nblocks: {self.nblocks}")

    # ---- registration (cppsim_wrapper.cpp:450-482)
    def _register(self, circuit_: QuantumCircuit) -> None:
        gl = circuit_._gates
        arr = _n.make_gate_array(gl)
        self._check(_n.lib().qs_register_gates(self._h, arr, len(gl)))
        self._gates = [g.copy() for g in gl]

    def partition_and_register_circuit(self, circuit_: QuantumCircuit, inner_size: int, verbose: int = 0) -> None:
        self._register(circuit_)
        self._check(_n.lib().qs_partition(self._h, int(inner_size), int(verbose)))

    def register_circuit_stages(self, circuit_: QuantumCircuit, stages, block_groups_list) -> None:
        """Backward-compatible form (compressed_state.hpp:477-507): per stage
        a list of groups, each a list of block ids."""
        self._register(circuit_)
        ns = len(stages)
        sizes = (_n.ct.c_uint32 * max(1, ns))(*[len(s) for s in stages])
        flat = [int(g) for s in stages for g in s]
        ids = (_n.ct.c_uint32 * max(1, len(flat)))(*flat)
        nb = self.nblocks
        b2g = np.zeros((max(1, ns), nb), dtype=np.uint32)
        ng = []
        for si, groups in enumerate(block_groups_list):
            ng.append(len(groups))
            for gi, blocks in enumerate(groups):
                for b in blocks:
                    b2g[si, int(b)] = gi
        ngroups = (_n.ct.c_uint32 * max(1, ns))(*ng)
        self._check(_n.lib().qs_register_stages(
            self._h, sizes, ns, ids, b2g.ctypes.data_as(_n.ct.POINTER(_n.ct.c_uint32)), ngroups))

    def get_stage_list(self) -> List[List[int]]:
        ns, nb = _n.ct.c_uint32(), _n.ct.c_uint32()
        self._check(_n.lib().qs_get_plan_info(self._h, _n.ct.byref(ns), _n.ct.byref(nb)))
        out = []
        for s in range(ns.value):
            cnt = _n.ct.c_uint32()
            self._check(_n.lib().qs_get_stage(self._h, s, None, 0, _n.ct.byref(cnt), None, None))
            ids = (_n.ct.c_uint32 * max(1, cnt.value))()
            self._check(_n.lib().qs_get_stage(self._h, s, ids, cnt.value, _n.ct.byref(cnt), None, None))
            out.append(list(ids)[:cnt.value])
        return out

    def get_block_to_group(self, stage: int):
        nb = self.nblocks
        arr = np.zeros(nb, dtype=np.uint32)
        ng = _n.ct.c_uint32()
        cnt = _n.ct.c_uint32()
        self._check(_n.lib().qs_get_stage(self._h, int(stage), None, 0, _n.ct.byref(cnt),
                                          arr.ctypes.data_as(_n.ct.POINTER(_n.ct.c_uint32)), _n.ct.byref(ng)))
        return arr, ng.value

    # ---- execution
    def apply_circuit(self) -> None:
        self._check(_n.lib().qs_apply_circuit(self._h))

    def get_vector(self, renormalize: bool = True) -> np.ndarray:
        """get_decompressed_state_vector: dense complex128, renormalised (Q6)."""
        out = np.empty(1 << self._n, dtype=np.complex128)
        self._check(_n.lib().qs_get_vector(self._h, out.view(np.float64).ctypes.data_as(_n.ct.POINTER(_n.ct.c_double)),
                                           1 if renormalize else 0))
        return out

    def get_amplitudes(self, first: int, count: int, renormalize: bool = True) -> np.ndarray:
        """Amplitudes [first, first + count) of get_vector (first and count
        multiples of the chunk size, get_stats()['chunk_log2'])."""
        out = np.empty(int(count), dtype=np.complex128)
        self._check(_n.lib().qs_get_amplitudes(self._h, int(first), int(count),
                                               out.view(np.float64).ctypes.data_as(_n.ct.POINTER(_n.ct.c_double)),
                                               1 if renormalize else 0))
        return out

    def get_amplitudes_to(self, address: int, first: int, count: int, renormalize: bool = True) -> None:
        """The amplitudes of get_amplitudes written as 2*count interleaved
        doubles at `address`: host memory or device memory of the state's
        GPU (e.g. a torch CUDA tensor's data_ptr())."""
        self._check(_n.lib().qs_get_amplitudes(self._h, int(first), int(count),
                                               _n.ct.cast(_n.ct.c_void_p(int(address)), _n.ct.POINTER(_n.ct.c_double)),
                                               1 if renormalize else 0))

    def get_squared_norm(self) -> float:
        v = _n.ct.c_double()
        self._check(_n.lib().qs_norm_squared(self._h, _n.ct.byref(v)))
        return v.value

    def set_computational_basis(self, basis: int) -> None:
        self._check(_n.lib().qs_set_basis_state(self._h, int(basis)))

    def _pauli_sums(self, xs, zs):
        return _pauli_sums(_n.lib().qs_expectation_pauli, self._h, self._check, xs, zs)

    def set_zero_state(self) -> None:
        self.set_computational_basis(0)

    def load(self, vec) -> None:
        v = np.ascontiguousarray(np.asarray(vec, dtype=np.complex128).reshape(-1))
        if v.size != 1 << self._n:
            raise ValueError("vector length must be 2^n")
        self._check(_n.lib().qs_load_vector(self._h, v.view(np.float64).ctypes.data_as(_n.ct.POINTER(_n.ct.c_double))))

    # ---- accounting
    def get_max_SV_bytes(self) -> int:
        v = _n.ct.c_uint64()
        self._check(_n.lib().qs_get_max_sv_bytes(self._h, _n.ct.byref(v)))
        return v.value

    def get_SV_bytes_history(self) -> List[int]:
        cnt = _n.ct.c_size_t()
        self._check(_n.lib().qs_get_sv_bytes_history(self._h, None, 0, _n.ct.byref(cnt)))
        arr = (_n.ct.c_uint64 * max(1, cnt.value))()
        self._check(_n.lib().qs_get_sv_bytes_history(self._h, arr, cnt.value, _n.ct.byref(cnt)))
        return list(arr)[:cnt.value]

    def get_zero_mask(self) -> np.ndarray:
        out = np.zeros(self.nblocks, dtype=np.uint8)
        self._check(_n.lib().qs_get_zero_mask(self._h, out.ctypes.data_as(_n.ct.POINTER(_n.ct.c_uint8))))
        return out

    def get_block_bytes(self) -> np.ndarray:
        out = np.zeros(self.nblocks, dtype=np.uint64)
        self._check(_n.lib().qs_get_block_bytes(self._h, out.ctypes.data_as(_n.ct.POINTER(_n.ct.c_uint64))))
        return out

    def get_total_times(self) -> Dict[str, float]:
        arr = (_n.ct.c_double * 10)()
        self._check(_n.lib().qs_get_total_times(self._h, arr))
        return {k: float(v) for k, v in zip(_TIMER_KEYS, arr)}

    def get_stats(self) -> Dict[str, float]:
        st = _n.qs_stats()
        self._check(_n.lib().qs_get_stats(self._h, _n.ct.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def transition_pauli_sums(self, bra: "CompressedQuantumState", xs, zs) -> np.ndarray:
        """sum_x conj(bra[x ^ x_t]) (-1)^{|x & z_t|} self[x] for every term
        (qs_transition_pauli; no normalisation)."""
        n = len(xs)
        xa = np.ascontiguousarray(np.asarray(xs, dtype=np.uint64))
        za = np.ascontiguousarray(np.asarray(zs, dtype=np.uint64))
        out = np.zeros(2 * max(1, n), dtype=np.float64)
        self._check(_n.lib().qs_transition_pauli(bra._h, self._h, xa.ctypes.data_as(_n.ct.POINTER(_n.ct.c_uint64)),
                                                 za.ctypes.data_as(_n.ct.POINTER(_n.ct.c_uint64)), n,
                                                 out.ctypes.data_as(_n.ct.POINTER(_n.ct.c_double))))
        return out[0:2 * n:2] + 1j * out[1:2 * n:2]

    def load_diagonal_pauli_sum(self, source: "CompressedQuantumState", zs, coefs) -> None:
        """self := (sum_t coefs[t] Z^{zs[t]}) source (qs_apply_diagonal_pauli_sum)."""
        za = np.ascontiguousarray(np.asarray(zs, dtype=np.uint64))
        ca = np.ascontiguousarray(np.asarray(coefs, dtype=np.complex128))
        self._check(_n.lib().qs_apply_diagonal_pauli_sum(self._h, source._h,
                                                         za.ctypes.data_as(_n.ct.POINTER(_n.ct.c_uint64)),
                                                         ca.view(np.float64).ctypes.data_as(_n.ct.POINTER(_n.ct.c_double)),
                                                         len(za)))

    def apply_dense_gate(self, targets, matrix) -> None:
        """Apply one dense gate on 4 or 5 qubits (matrix bit i <-> targets[i])
        at once as a stage of its own (qs_apply_dense_gate): complex64 on the
        tensor cores, complex128 on the CUDA cores."""
        t = [int(q) for q in targets]
        m = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128).reshape(1 << len(t), 1 << len(t)))
        ta = (_n.ct.c_uint32 * len(t))(*t)
        self._check(_n.lib().qs_apply_dense_gate(self._h, ta, len(t),
                                                 m.reshape(-1).view(np.float64).ctypes.data_as(
                                                     _n.ct.POINTER(_n.ct.c_double))))

    def apply_gates(self, gates: Sequence[QuantumGateBase], inner_size: int = 4) -> None:
        """Apply a gate list that may hold fused gates on 3 to 5 qubits
        (QuantumCircuitOptimizer.optimize(c, block_size=k)): every run of
        gates on at most two qubits is registered and applied as a circuit
        (the reference's stages), every larger gate as one dense pass; a
        3-qubit gate is widened to 4 qubits with an idle qubit.  The
        reference's compressed engine rejects gates on more than two qubits."""
        from ._gates import full_matrix
        run: List[QuantumGateBase] = []

        def flush():
            if run:
                c = QuantumCircuit(self._n)
                c._gates = list(run)
                self.partition_and_register_circuit(c, inner_size, 0)
                self.apply_circuit()
                run.clear()

        for g in gates:
            qs = g.full_qubits()
            if len(qs) <= 2:
                run.append(g)
                continue
            flush()
            m, order = full_matrix(g)
            if len(order) == 3:
                extra = next(q for q in range(self._n) if q not in order)
                order = list(order) + [extra]
                m = np.kron(np.eye(2), m)
            self.apply_dense_gate(order, m)
        flush()

    def load_pauli_sum(self, source: "CompressedQuantumState", xs, zs, coefs) -> None:
        """self := (sum_t coefs[t] X^{xs[t]} Z^{zs[t]}) source for general
        Pauli strings, with any i^{ny} of Y factors folded into coefs
        (qs_apply_pauli_sum): the adjoint's lambda = H psi."""
        xa = np.ascontiguousarray(np.asarray(xs, dtype=np.uint64))
        za = np.ascontiguousarray(np.asarray(zs, dtype=np.uint64))
        ca = np.ascontiguousarray(np.asarray(coefs, dtype=np.complex128))
        self._check(_n.lib().qs_apply_pauli_sum(self._h, source._h, xa.ctypes.data_as(_n.ct.POINTER(_n.ct.c_uint64)),
                                                za.ctypes.data_as(_n.ct.POINTER(_n.ct.c_uint64)),
                                                ca.view(np.float64).ctypes.data_as(_n.ct.POINTER(_n.ct.c_double)),
                                                len(xa)))

    def checkpoint(self, slot: int = 0) -> None:
        """Copy the compressed store into device checkpoint `slot`."""
        self._check(_n.lib().qs_checkpoint(self._h, int(slot)))

    def restore(self, slot: int = 0) -> None:
        self._check(_n.lib().qs_restore(self._h, int(slot)))

    def free_checkpoint(self, slot: int = 0) -> None:
        self._check(_n.lib().qs_free_checkpoint(self._h, int(slot)))

    def export_store(self) -> bytes:
        size = _n.ct.c_uint64()
        self._check(_n.lib().qs_export_store(self._h, None, 0, _n.ct.byref(size)))
        buf = np.empty(size.value, dtype=np.uint8)
        self._check(_n.lib().qs_export_store(self._h, buf.ctypes.data, size.value, _n.ct.byref(size)))
        return buf.tobytes()

    def import_store(self, data: bytes) -> None:
        buf = np.frombuffer(data, dtype=np.uint8)
        self._check(_n.lib().qs_import_store(self._h, buf.ctypes.data, buf.size))

    def sampling_blockwise(self, sampling_count: int, random_seed: int) -> List[int]:
        """Draw `sampling_count` basis-state indices block by block
        (compressed_state.hpp:1600-1681): block masses and the searches inside
        blocks on the device, the reference's seeded generators on the host,
        so that equal amplitudes give the reference's samples.  Raises
        ValueError when the state has no finite positive probability mass."""
        n = int(sampling_count)
        if n < 0 or n >= 1 << 32:
            raise ValueError("sampling_count must fit an unsigned 32-bit integer")
        out = np.empty(max(n, 1), dtype=np.uint64)
        self._check(_n.lib().qs_sample_blockwise(self._h, n, int(random_seed) & 0xFFFFFFFF,
                                                 out.ctypes.data_as(_n.ct.POINTER(_n.ct.c_uint64))))
        return [int(x) for x in out[:n]]

    def __repr__(self):
        return f"CompressedQuantumState(qubits={self._n}, block_size={self._B})"


__all__ = [
    "QuantumState", "QuantumCircuit", "ParametricQuantumCircuit", "CompressedQuantumState", "Observable",
    "QuantumGateBase", "QuantumGateMatrix", "check_build_for_mpi", "gate", "circuit", "QompsimError",
]

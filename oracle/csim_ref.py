"""ORACLE (test infrastructure only): the reference's FP64 csim kernels.

Loads oracle/_ref/libcsim_ref.so (built from the reference's src/csim by
oracle/Makefile) and applies a qulacs gate list to a dense complex128 vector
with the kernel the reference would call for that gate:

* "CNOT" / "CZ" / "SWAP"  -> CNOT_gate / CZ_gate / SWAP_gate
  (src/csim/update_ops_named_{CNOT,CZ,SWAP}.cpp)
* a matrix gate without controls -> single_qubit_dense_matrix_gate or
  double_qubit_dense_matrix_gate_c (gate_matrix.cpp:128-160 dispatch)
* with controls -> multi_qubit_control_multi_qubit_dense_matrix_gate
"""
from __future__ import annotations

import ctypes as ct
import os
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcsim_ref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} missing: run `make -C oracle` where the reference is mounted")
        L = ct.CDLL(LIB_PATH)
        P = ct.c_void_p
        U = ct.c_uint
        U64 = ct.c_uint64
        L.csimref_dense1.argtypes = [U, P, P, U64]
        L.csimref_dense2.argtypes = [U, U, P, P, U64]
        L.csimref_dense_multi.argtypes = [P, U, P, P, U64]
        L.csimref_controlled.argtypes = [P, P, U, P, U, P, P, U64]
        L.csimref_cnot.argtypes = [U, U, P, U64]
        L.csimref_cz.argtypes = [U, U, P, U64]
        L.csimref_swap.argtypes = [U, U, P, U64]
        L.csimref_norm_squared.argtypes = [P, U64]
        L.csimref_norm_squared.restype = ct.c_double
        L.csimref_inner_product.argtypes = [P, P, U64, P]
        L.csimref_init_zero.argtypes = [P, U64]
        L.csimref_max_threads.restype = ct.c_int
        _lib = L
    return _lib


def zero_state(n: int) -> np.ndarray:
    s = np.empty(1 << n, dtype=np.complex128)
    lib().csimref_init_zero(s.ctypes.data, s.size)
    return s


def _ptr(a):
    return a.ctypes.data


def apply_gate(state: np.ndarray, g) -> None:
    assert state.dtype == np.complex128 and state.flags.c_contiguous
    L = lib()
    dim = state.size
    name = g.get_name()
    t = g.get_target_index_list()
    c = g.get_control_index_list()
    cv = g.get_control_value_list()
    if name == "CNOT":
        L.csimref_cnot(c[0], t[0], _ptr(state), dim)
        return
    if name == "CZ":
        L.csimref_cz(c[0], t[0], _ptr(state), dim)
        return
    if name == "SWAP":
        L.csimref_swap(t[0], t[1], _ptr(state), dim)
        return
    m = np.ascontiguousarray(g.get_matrix(), dtype=np.complex128)
    if not c:
        if len(t) == 1:
            L.csimref_dense1(t[0], _ptr(m), _ptr(state), dim)
        elif len(t) == 2:
            L.csimref_dense2(t[0], t[1], _ptr(m), _ptr(state), dim)
        else:
            ta = np.asarray(t, dtype=np.uint32)
            L.csimref_dense_multi(_ptr(ta), len(t), _ptr(m), _ptr(state), dim)
        return
    ca = np.asarray(c, dtype=np.uint32)
    va = np.asarray(cv, dtype=np.uint32)
    ta = np.asarray(t, dtype=np.uint32)
    L.csimref_controlled(_ptr(ca), _ptr(va), len(c), _ptr(ta), len(t), _ptr(m), _ptr(state), dim)


def apply_gates(state: np.ndarray, gates: Sequence) -> np.ndarray:
    for g in gates:
        apply_gate(state, g)
    return state


def run_circuit(n: int, gates: Sequence, init: np.ndarray | None = None) -> np.ndarray:
    s = zero_state(n) if init is None else np.array(init, dtype=np.complex128, copy=True)
    return apply_gates(s, gates)


def norm_squared(state: np.ndarray) -> float:
    return float(lib().csimref_norm_squared(_ptr(state), state.size))


def inner_product(bra: np.ndarray, ket: np.ndarray) -> complex:
    out = np.zeros(2)
    lib().csimref_inner_product(_ptr(bra), _ptr(ket), bra.size, _ptr(out))
    return complex(out[0], out[1])


def max_threads() -> int:
    return int(lib().csimref_max_threads())

"""ORACLE / BASELINE INFRASTRUCTURE ONLY: the reference's plain complex128 GPU
simulator (Qulacs gpusim, src/gpusim), built from the reference sources by
oracle/Makefile into oracle/_ref/libgpusim_ref.so with the gate-by-gate C
ABI of oracle/gpusim_shim.cu.

Used by tests/ to cross-check this package's uncompressed per-gate and fused
paths against the reference's own GPU kernels, and by bench.py to time the
reference's per-gate GPU path on the benchmark's gate list.  One gate = one
call into the reference (its kernels run on its own stream).
"""
from __future__ import annotations

import ctypes as ct
import os
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libgpusim_ref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} missing: run `make -C oracle gpusim REF=<reference checkout>`")
        L = ct.CDLL(LIB_PATH)
        P = ct.c_void_p
        U32 = ct.c_uint32
        U64 = ct.c_uint64
        L.gsref_init.argtypes = [ct.c_uint]
        L.gsref_init.restype = ct.c_int
        L.gsref_alloc.argtypes = [U64]
        L.gsref_alloc.restype = P
        L.gsref_free.argtypes = [P]
        L.gsref_init_zero.argtypes = [P, U64]
        L.gsref_apply.argtypes = [P, U64, ct.c_char_p, U32, ct.POINTER(U32), U32, ct.POINTER(U32), ct.POINTER(U32),
                                  ct.POINTER(ct.c_double)]
        L.gsref_apply.restype = ct.c_int
        L.gsref_get.argtypes = [P, U64, U64, ct.POINTER(ct.c_double)]
        L.gsref_get.restype = ct.c_int
        L.gsref_sync.restype = ct.c_int
        if L.gsref_init(0) != 0:
            raise RuntimeError("gpusim: no CUDA stream")
        _lib = L
    return _lib


class GpuState:
    """A reference QuantumStateGpu-style state vector: 2^n complex128 in
    device memory, initialised to |0...0>."""

    def __init__(self, n: int):
        self.n = int(n)
        self.dim = 1 << self.n
        self._p = lib().gsref_alloc(self.dim)
        if not self._p:
            raise MemoryError("gpusim: device allocation failed")
        lib().gsref_init_zero(self._p, self.dim)

    def __del__(self):
        p = getattr(self, "_p", None)
        if p:
            try:
                lib().gsref_free(p)
            except Exception:
                pass
            self._p = None

    def set_zero_state(self) -> None:
        lib().gsref_init_zero(self._p, self.dim)

    def prepare(self, gates: Sequence):
        """Per-gate call records of `gates` (built once, so that timing loops
        measure the reference's kernels, not this wrapper's conversions)."""
        recs = []
        for g in gates:
            t = list(g.get_target_index_list())
            c = list(g.get_control_index_list())
            v = list(g.get_control_value_list())
            m = np.ascontiguousarray(np.asarray(g.get_matrix(), dtype=np.complex128).reshape(-1))
            recs.append((g.get_name().encode(), len(t), (ct.c_uint32 * max(1, len(t)))(*t), len(c),
                         (ct.c_uint32 * max(1, len(c)))(*c), (ct.c_uint32 * max(1, len(v)))(*v), m,
                         m.view(np.float64).ctypes.data_as(ct.POINTER(ct.c_double))))
        return recs

    def apply_prepared(self, recs) -> None:
        L = lib()
        for name, nt, t, nc, c, v, _m, mp in recs:
            if L.gsref_apply(self._p, self.dim, name, nt, t, nc, c, v, mp) != 0:
                raise RuntimeError("gpusim: unsupported gate")

    def apply(self, gates: Sequence) -> None:
        self.apply_prepared(self.prepare(gates))

    def sync(self) -> None:
        lib().gsref_sync()

    def get_amplitudes(self, first: int, count: int) -> np.ndarray:
        out = np.empty(int(count), dtype=np.complex128)
        if lib().gsref_get(self._p, int(first), int(count),
                           out.view(np.float64).ctypes.data_as(ct.POINTER(ct.c_double))) != 0:
            raise RuntimeError("gpusim: copy failed")
        return out

    def get_vector(self) -> np.ndarray:
        return self.get_amplitudes(0, self.dim)

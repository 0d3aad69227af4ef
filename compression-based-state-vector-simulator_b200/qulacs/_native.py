"""ctypes binding of the engine's C ABI (include/qompsim.h).

This is the whole native boundary of the Python package: every struct and
entry point below mirrors the header one to one.  The shared library is
built in-tree (build_ext.py); loading fails loudly when it is missing or when
no CUDA device can be used -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as ct
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PKG = os.path.dirname(_HERE)
LIB_PATH = os.path.join(_PKG, "lib", "libqompsim.so")

QS_OK = 0
QS_ERR_ARG = 1
QS_ERR_CUDA = 2
QS_ERR_CAPACITY = 3
QS_ERR_UNSUPPORTED_GATE = 4
QS_ERR_TIMEOUT = 5
QS_ERR_CORRUPT = 6
QS_ERR_STATE = 7
QS_ERR_NOMEM = 8
QS_ERR_DOMAIN = 9

QS_COMPLEX128 = 0
QS_COMPLEX64 = 1

QS_FLAG_EXACT_ZERO_TEST = 0x1
QS_FLAG_REFERENCE_CONTROLS = 0x2
QS_FLAG_QUIET = 0x4
QS_FLAG_PROFILE = 0x8
QS_FLAG_HOST_STORE = 0x10

STATUS_NAMES = {
    0: "QS_OK", 1: "QS_ERR_ARG", 2: "QS_ERR_CUDA", 3: "QS_ERR_CAPACITY",
    4: "QS_ERR_UNSUPPORTED_GATE", 5: "QS_ERR_TIMEOUT", 6: "QS_ERR_CORRUPT",
    7: "QS_ERR_STATE", 8: "QS_ERR_NOMEM", 9: "QS_ERR_DOMAIN",
}


class qs_gate(ct.Structure):
    _fields_ = [
        ("name", ct.c_char * 24),
        ("ntargets", ct.c_uint32),
        ("ncontrols", ct.c_uint32),
        ("targets", ct.c_uint32 * 2),
        ("controls", ct.c_uint32 * 2),
        ("control_values", ct.c_uint32 * 2),
        ("matrix", ct.c_double * 32),
    ]


class qs_stats(ct.Structure):
    _fields_ = [
        ("stages", ct.c_uint64),
        ("passes", ct.c_uint64),
        ("tiles", ct.c_uint64),
        ("bytes_read", ct.c_uint64),
        ("bytes_written", ct.c_uint64),
        ("amp_gate_updates", ct.c_uint64),
        ("kernel_ms", ct.c_double),
        ("apply_ms", ct.c_double),
        ("mantissa_bits", ct.c_int32),
        ("linear_exp", ct.c_int32),
        ("chunk_log2", ct.c_int32),
        ("tile_log2", ct.c_int32),
        ("sweeps", ct.c_uint64),
        ("ops", ct.c_uint64),
        ("perm_passes", ct.c_uint64),
        ("perm_bytes", ct.c_uint64),
        ("perm_ms", ct.c_double),
        ("code_move_passes", ct.c_uint64),
        ("arena_capacity", ct.c_uint64),
        ("host_store", ct.c_uint64),
        ("merged_from", ct.c_int64),
        ("tail_passes", ct.c_uint64),
        ("pair_ms", ct.c_double),
    ]


# (name, restype, argtypes) of every exported symbol of qompsim.h
_P = ct.c_void_p
_U32 = ct.c_uint32
_U64 = ct.c_uint64
_I32 = ct.c_int32
_D = ct.c_double
SIGNATURES = [
    ("qs_last_error", ct.c_char_p, [_P]),
    ("qs_dense_last_error", ct.c_char_p, [_P]),
    ("qs_create", ct.c_int, [ct.POINTER(_P), _U32, _U32, ct.c_int, _D, _D, _U32]),
    ("qs_destroy", ct.c_int, [_P]),
    ("qs_set_stream", ct.c_int, [_P, _P]),
    ("qs_register_gates", ct.c_int, [_P, ct.POINTER(qs_gate), ct.c_size_t]),
    ("qs_partition", ct.c_int, [_P, _U32, ct.c_int]),
    ("qs_register_stages", ct.c_int, [_P, ct.POINTER(_U32), ct.c_size_t, ct.POINTER(_U32),
                                      ct.POINTER(_U32), ct.POINTER(_U32)]),
    ("qs_plan_stages", ct.c_int, [ct.POINTER(qs_gate), ct.c_size_t, _U32, _U32, _U32, ct.POINTER(ct.c_size_t),
                                  ct.POINTER(_U32), ct.POINTER(_U32), ct.POINTER(_U32), ct.POINTER(_U32)]),
    ("qs_stage_chunk_permutation", ct.c_int, [ct.POINTER(qs_gate), ct.c_size_t, _U32, _U32, ct.c_int,
                                              ct.POINTER(qs_gate), ct.POINTER(ct.c_size_t),
                                              ct.POINTER(ct.c_int32), ct.POINTER(_U64)]),
    ("qs_get_plan_info", ct.c_int, [_P, ct.POINTER(_U32), ct.POINTER(_U32)]),
    ("qs_get_stage", ct.c_int, [_P, _U32, ct.POINTER(_U32), _U32, ct.POINTER(_U32),
                                ct.POINTER(_U32), ct.POINTER(_U32)]),
    ("qs_apply_circuit", ct.c_int, [_P]),
    ("qs_get_vector", ct.c_int, [_P, ct.POINTER(_D), ct.c_int]),
    ("qs_get_amplitudes", ct.c_int, [_P, _U64, _U64, ct.POINTER(_D), ct.c_int]),
    ("qs_sample_blockwise", ct.c_int, [_P, ct.c_uint32, ct.c_uint32, ct.POINTER(_U64)]),
    ("qs_norm_squared", ct.c_int, [_P, ct.POINTER(_D)]),
    ("qs_expectation_pauli", ct.c_int, [_P, ct.POINTER(_U64), ct.POINTER(_U64), ct.c_size_t, ct.POINTER(_D)]),
    ("qs_transition_pauli", ct.c_int, [_P, _P, ct.POINTER(_U64), ct.POINTER(_U64), ct.c_size_t, ct.POINTER(_D)]),
    ("qs_apply_diagonal_pauli_sum", ct.c_int, [_P, _P, ct.POINTER(_U64), ct.POINTER(_D), ct.c_size_t]),
    ("qs_apply_pauli_sum", ct.c_int, [_P, _P, ct.POINTER(_U64), ct.POINTER(_U64), ct.POINTER(_D), ct.c_size_t]),
    ("qs_apply_dense_gate", ct.c_int, [_P, ct.POINTER(_U32), _U32, ct.POINTER(_D)]),
    ("qs_adjoint", ct.c_int, [_P, _P, _P, ct.POINTER(_I32), ct.POINTER(_U64), ct.POINTER(_U64), ct.c_size_t,
                              ct.POINTER(_D), _U32]),
    ("qs_dense_expectation_pauli", ct.c_int, [_P, ct.POINTER(_U64), ct.POINTER(_U64), ct.c_size_t, ct.POINTER(_D)]),
    ("qs_dense_copy", ct.c_int, [_P, _P]),
    ("qs_dense_apply_pauli_sum", ct.c_int, [_P, _P, ct.POINTER(_U64), ct.POINTER(_U64), ct.POINTER(_D), ct.c_size_t]),
    ("qs_dense_transition_pauli", ct.c_int, [_P, _P, ct.POINTER(_U64), ct.POINTER(_U64), ct.c_size_t,
                                             ct.POINTER(_D)]),
    ("qs_dense_adjoint", ct.c_int, [_P, _P, ct.POINTER(qs_gate), ct.POINTER(ct.c_int32), ct.POINTER(_U64),
                                    ct.POINTER(_U64), ct.c_size_t, ct.POINTER(_D), _U32]),
    ("qs_get_zero_mask", ct.c_int, [_P, ct.POINTER(ct.c_uint8)]),
    ("qs_get_block_bytes", ct.c_int, [_P, ct.POINTER(_U64)]),
    ("qs_get_max_sv_bytes", ct.c_int, [_P, ct.POINTER(_U64)]),
    ("qs_get_sv_bytes_history", ct.c_int, [_P, ct.POINTER(_U64), ct.c_size_t, ct.POINTER(ct.c_size_t)]),
    ("qs_get_total_times", ct.c_int, [_P, ct.POINTER(_D)]),
    ("qs_get_stats", ct.c_int, [_P, ct.POINTER(qs_stats)]),
    ("qs_export_store", ct.c_int, [_P, _P, _U64, ct.POINTER(_U64)]),
    ("qs_import_store", ct.c_int, [_P, _P, _U64]),
    ("qs_export_half", ct.c_int, [_P, _U32, _U32, _P, _U64, ct.POINTER(_U64)]),
    ("qs_import_half", ct.c_int, [_P, _U32, _U32, _P, _U64]),
    ("qs_set_zero_vector", ct.c_int, [_P]),
    ("qs_selftest_bounded_wait", ct.c_int, [_U32, ct.POINTER(ct.c_int32)]),
    ("qs_checkpoint", ct.c_int, [_P, _U32]),
    ("qs_restore", ct.c_int, [_P, _U32]),
    ("qs_free_checkpoint", ct.c_int, [_P, _U32]),
    ("qs_set_basis_state", ct.c_int, [_P, _U64]),
    ("qs_load_vector", ct.c_int, [_P, ct.POINTER(_D)]),
    ("qs_dense_create", ct.c_int, [ct.POINTER(_P), _U32, ct.c_int]),
    ("qs_dense_destroy", ct.c_int, [_P]),
    ("qs_dense_set_stream", ct.c_int, [_P, _P]),
    ("qs_dense_apply_gates", ct.c_int, [_P, ct.POINTER(qs_gate), ct.c_size_t]),
    ("qs_dense_apply_gates_pergate", ct.c_int, [_P, ct.POINTER(qs_gate), ct.c_size_t]),
    ("qs_dense_get_vector", ct.c_int, [_P, ct.POINTER(_D)]),
    ("qs_dense_get_amplitudes", ct.c_int, [_P, _U64, _U64, ct.POINTER(_D)]),
    ("qs_dense_set_vector", ct.c_int, [_P, ct.POINTER(_D)]),
    ("qs_dense_set_basis_state", ct.c_int, [_P, _U64]),
    ("qs_dense_norm_squared", ct.c_int, [_P, ct.POINTER(_D)]),
    ("qs_dense_device_ptr", ct.c_int, [_P, ct.POINTER(_P)]),
    ("qs_codec_params", ct.c_int, [ct.c_int, _D, _D, ct.POINTER(_I32), ct.POINTER(_I32)]),
    ("qs_codec_test", ct.c_int, [ct.c_int, _D, _D, _U32, _P, _U64, ct.POINTER(_U32),
                                 ct.POINTER(_I32), ct.POINTER(_U32), _P]),
    ("qs_codec_roundtrip_noalloc", ct.c_int, [ct.c_int, _D, _D, _U32, _P, _U64, _P, _P, _P, _P]),
]

_lib = None
_lock = threading.Lock()


class QompsimError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class QompsimDomainError(QompsimError, ValueError):
    """QS_ERR_DOMAIN: the reference raises std::domain_error, which its
    bindings turn into ValueError."""


def load_library(path: str = LIB_PATH):
    """Load libqompsim.so and declare its C signatures (no device work)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise ImportError(
                f"{path} is missing: build it with `python build_ext.py` (nvcc, sm_100a). "
                "The engine has no CPU fallback.")
        lib = ct.CDLL(path)
        for name, res, args in SIGNATURES:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
        return lib


def lib():
    return load_library()


def check(status: int, handle=None, dense: bool = False) -> None:
    if status == QS_OK:
        return
    L = lib()
    msg = (L.qs_dense_last_error(handle) if dense else L.qs_last_error(handle)) or b""
    cls = QompsimDomainError if status == QS_ERR_DOMAIN else QompsimError
    raise cls(status, msg.decode(errors="replace"))


def make_gate_array(gates):
    """Pack qulacs gate objects into a qs_gate array (to_matrix_gate with the
    original name kept, as python/cppsim_wrapper.cpp:465-482 does)."""
    arr = (qs_gate * max(1, len(gates)))()
    for i, g in enumerate(gates):
        tg = g.get_target_index_list()
        cl = g.get_control_index_list()
        cv = g.get_control_value_list()
        if len(tg) > 2 or len(cl) > 2:
            raise QompsimError(QS_ERR_UNSUPPORTED_GATE,
                               f"gate {i} ({g.get_name()}): only single- or two-qubit gates are implemented")
        rec = arr[i]
        rec.name = g.get_name().encode()[:23]
        rec.ntargets = len(tg)
        rec.ncontrols = len(cl)
        for k, t in enumerate(tg):
            rec.targets[k] = t
        for k, (c, v) in enumerate(zip(cl, cv)):
            rec.controls[k] = c
            rec.control_values[k] = v
        m = np.ascontiguousarray(g.get_matrix(), dtype=np.complex128).reshape(-1)
        if m.size > 16:
            raise QompsimError(QS_ERR_UNSUPPORTED_GATE, f"gate {i} ({g.get_name()}): matrix larger than 4x4")
        ct.memmove(ct.addressof(rec) + qs_gate.matrix.offset, m.ctypes.data, m.nbytes)
    return arr


def dtype_code(dtype) -> int:
    if dtype in (QS_COMPLEX128, "complex128", np.complex128):
        return QS_COMPLEX128
    if dtype in (QS_COMPLEX64, "complex64", np.complex64):
        return QS_COMPLEX64
    raise ValueError(f"unsupported dtype {dtype!r}")


def env_dtype() -> int:
    """QOMPSIM_DTYPE={complex128,complex64} (default complex128)."""
    return dtype_code(os.environ.get("QOMPSIM_DTYPE", "complex128"))

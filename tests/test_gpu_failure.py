"""Failure detection on the GPU without a GPU fault (run with -m gpu).

The staged and tensor-core passes wait on mbarriers with an iteration limit;
a wait that gives up sets the pass's error flag and the call returns
QS_ERR_TIMEOUT.  qs_selftest_bounded_wait runs that wait on an mbarrier that
nothing completes (no copy is ever issued), so it must give up; the context
must stay usable: a compressed circuit runs afterwards and matches csim.
"""
import ctypes as ct

import numpy as np
import pytest

import helpers  # noqa: F401  (sys.path)
from oracle import csim_ref

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_survives():
    import qulacs
    from qulacs import _native
    L = _native.load_library()
    gave_up = ct.c_int32(-1)
    _native.check(L.qs_selftest_bounded_wait(256, ct.byref(gave_up)))
    assert gave_up.value == 1
    n = 10
    c = qulacs.QuantumCircuit(n)
    for q in range(n):
        c.add_H_gate(q)
    c.add_CNOT_gate(0, 9)
    c.add_RZ_gate(3, 0.4)
    cq = qulacs.CompressedQuantumState(n, 6, dtype="complex128", eps_rel=2.0 ** -24, eps_abs=1e-14,
                                       flags=_native.QS_FLAG_QUIET)
    cq.partition_and_register_circuit(c, 3, 0)
    cq.apply_circuit()
    ref = csim_ref.run_circuit(n, c._gates)
    assert np.abs(cq.get_vector() - ref).max() < 1e-6


def test_bounded_wait_rejects_bad_arguments():
    from qulacs import _native
    L = _native.load_library()
    gave_up = ct.c_int32(-1)
    assert L.qs_selftest_bounded_wait(0, ct.byref(gave_up)) == _native.QS_ERR_ARG

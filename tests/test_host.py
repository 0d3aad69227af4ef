"""Host logic of the product, checked on the CPU against the oracle.

* the C ABI library loads and exports every entry point of include/qompsim.h
  (no device call is made);
* the restated fusion optimizer keeps every golden circuit's state (applied
  with the reference's csim kernels) and reproduces the known fused lists;
* the engine's stage planner (qs_plan_stages, host only) equals the oracle
  planner stage for stage and block for block;
* argument errors come back as status codes, not crashes.
"""
import ctypes as ct
import os
import re

import numpy as np
import pytest

import helpers
from oracle import csim_ref, planner

ROOT = helpers.HERE and os.path.dirname(helpers.HERE)
HEADER = os.path.join(ROOT, "include", "qompsim.h")


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(qs_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_symbol():
    from qulacs import _native
    L = _native.load_library()
    names = header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    declared = {n for n, _, _ in _native.SIGNATURES}
    assert set(names) == declared, set(names) ^ declared


def test_codec_params_from_library_match_oracle():
    from qulacs import _native
    from oracle import codec as oc
    L = _native.load_library()
    for f64 in (True, False):
        for er, ea in [(1e-3, 1e-7), (1e-2, 0.0), (2 ** -24, 1e-12), (0.5, 1.0)]:
            m, Lp = ct.c_int32(), ct.c_int32()
            assert L.qs_codec_params(0 if f64 else 1, er, ea, ct.byref(m), ct.byref(Lp)) == 0
            assert (m.value, Lp.value) == oc.params(f64, er, ea)
    assert L.qs_codec_params(0, 0.0, 1e-7, None, None) == _native.QS_ERR_ARG
    assert L.qs_codec_params(0, 1.5, 1e-7, None, None) == _native.QS_ERR_ARG


@pytest.mark.skipif(not csim_ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("key", sorted(helpers.golden_circuits()))
def test_optimizer_preserves_state(key):
    c = helpers.build_circuit(key)
    o = helpers.optimized(c, 4)
    assert o.get_gate_count() <= c.get_gate_count()
    for g in o._gates:
        assert len(g.get_target_index_list()) + len(g.get_control_index_list()) <= 2
    v = csim_ref.run_circuit(o.get_qubit_count(), o._gates)
    assert np.abs(v - helpers.golden_states()[key]).max() < 1e-12


def test_optimizer_ghz_fanout_fused_list():
    from qompsim import circuits as C
    o = helpers.optimized(C.ghz_fanout(20), 12)
    names = [(g.get_name(), g.get_target_index_list(), g.get_control_index_list()) for g in o._gates]
    assert names[0] == ("DenseMatrix", [0, 1], [])
    assert names[1:] == [("CNOT", [i], [0]) for i in range(2, 20)]
    m = o._gates[0].get_matrix()
    s = 1 / np.sqrt(2)
    expect = np.array([[s, s, 0, 0], [0, 0, s, -s], [0, 0, s, s], [s, -s, 0, 0]])
    assert np.abs(m - expect).max() < 1e-15


def test_optimizer_merge_shared_control_keeps_control():
    # gate_merge.cpp case 4: equal control values stay a control
    import qulacs
    c = qulacs.QuantumCircuit(3)
    c.add_CNOT_gate(0, 1)
    c.add_CZ_gate(0, 1)
    o = helpers.optimized(c)
    assert o.get_gate_count() == 1
    g = o._gates[0]
    assert g.get_control_index_list() == [0] and g.get_target_index_list() == [1]
    assert np.abs(g.get_matrix() - np.array([[0, 1], [-1, 0]])).max() == 0


def _plan(gates, n, B, I):
    from qulacs import _native
    L = _native.load_library()
    arr = _native.make_gate_array(gates)
    ns = ct.c_size_t()
    st = L.qs_plan_stages(arr, len(gates), n, B, I, ct.byref(ns), None, None, None, None)
    assert st == 0, L.qs_last_error(None)
    k = ns.value
    sizes = (ct.c_uint32 * max(1, k))()
    ids = (ct.c_uint32 * max(1, len(gates)))()
    nb = 1 << (n - B)
    b2g = np.zeros(max(1, k) * nb, dtype=np.uint32)
    ng = (ct.c_uint32 * max(1, k))()
    assert L.qs_plan_stages(arr, len(gates), n, B, I, ct.byref(ns), sizes, ids,
                            b2g.ctypes.data_as(ct.POINTER(ct.c_uint32)), ng) == 0
    stages, off = [], 0
    for s in range(k):
        stages.append(list(ids[off:off + sizes[s]]))
        off += sizes[s]
    return stages, [list(b2g[s * nb:(s + 1) * nb]) for s in range(k)], list(ng)[:k]


@pytest.mark.parametrize("key", sorted(helpers.golden_circuits()))
def test_engine_planner_matches_oracle(key):
    c = helpers.optimized(helpers.build_circuit(key), 4)
    n = c.get_qubit_count()
    g = planner.describe(c._gates)
    for B in range(4, n):
        for I in (0, 1, 2, 3, 4):
            st, maps, counts = _plan(c._gates, n, B, I)
            ost = planner.partition_circuit(g, B, I)
            omaps, ocounts = planner.make_block_groups(g, ost, n, B)
            assert st == ost, (B, I)
            assert maps == omaps and counts == ocounts, (B, I)


def test_engine_planner_unoptimized_and_config_circuits():
    from qompsim import circuits as C
    cases = [(C.ghz_fanout(20), 20, 12, 4), (C.qft_basis(14, 1), 14, 8, 4), (C.hea(12, 3, 0), 12, 6, 2),
             (C.qaoa_maxcut(12, 2, 0), 12, 7, 4), (C.brickwork(10, 4, 0), 10, 5, 3)]
    for c, n, B, I in cases:
        for circ in (c, helpers.optimized(c, B)):
            g = planner.describe(circ._gates)
            st, maps, counts = _plan(circ._gates, n, B, I)
            ost = planner.partition_circuit(g, B, I)
            omaps, ocounts = planner.make_block_groups(g, ost, n, B)
            assert (st, maps, counts) == (ost, omaps, ocounts)
    st, _, _ = _plan(helpers.optimized(C.ghz_fanout(20), 12)._gates, 20, 12, 4)
    assert [len(s) for s in st] == [15, 4]


def test_plan_rejects_bad_arguments():
    import qulacs
    from qulacs import _native
    L = _native.load_library()
    c = qulacs.QuantumCircuit(6)
    c.add_CNOT_gate(0, 5)
    arr = _native.make_gate_array(c._gates)
    ns = ct.c_size_t()
    assert L.qs_plan_stages(arr, 1, 4, 2, 2, ct.byref(ns), None, None, None, None) == _native.QS_ERR_ARG
    assert b"range" in L.qs_last_error(None)
    assert L.qs_plan_stages(arr, 1, 6, 7, 2, ct.byref(ns), None, None, None, None) == _native.QS_ERR_ARG
    assert L.qs_plan_stages(arr, 1, 6, 2, 2, None, None, None, None, None) == _native.QS_ERR_ARG


def test_three_qubit_gate_rejected_before_device():
    import qulacs
    from qulacs import gate as G, _native
    c = qulacs.QuantumCircuit(4)
    c.add_gate(G.DenseMatrix([0, 1, 2], np.eye(8)))
    with pytest.raises(_native.QompsimError) as e:
        _native.make_gate_array(c._gates)
    assert e.value.status == _native.QS_ERR_UNSUPPORTED_GATE


def test_check_build_for_mpi_false():
    import qulacs
    assert qulacs.check_build_for_mpi() is False


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_stage_chunk_permutation_keeps_the_state(seed):
    """Folding SWAP / X on qubits >= C into a chunk permutation and relabelling
    the later gates gives the same state (csim kernels, FP64) once the
    permutation is applied to the stored amplitudes."""
    from qulacs import _native
    from qulacs import gate as G
    L = _native.load_library()
    n, C = 9, 3
    c = helpers.perm_heavy_circuit(n, C, 40, seed)
    gates = c._gates
    arr = _native.make_gate_array(gates)
    out = (_native.qs_gate * len(gates))()
    cnt = ct.c_size_t()
    dst = (ct.c_int32 * (n - C))()
    flip = ct.c_uint64()
    assert L.qs_stage_chunk_permutation(arr, len(gates), n, C, 0, out, ct.byref(cnt), dst, ct.byref(flip)) == 0
    assert cnt.value < len(gates)            # something was folded
    rel = []
    for k in range(cnt.value):
        g = out[k]
        d = 1 << g.ntargets
        m = np.array(g.matrix[:2 * d * d]).view(np.complex128).reshape(d, d)
        rel.append(G.DenseMatrix([g.targets[i] for i in range(g.ntargets)], m))
    stored = csim_ref.run_circuit(n, rel)
    idx = np.arange(1 << n, dtype=np.int64)
    ch = idx >> C
    sig = np.full_like(ch, flip.value)
    for b in range(n - C):
        sig ^= ((ch >> b) & 1) << dst[b]
    true = np.empty_like(stored)
    true[(sig << C) | (idx & ((1 << C) - 1))] = stored
    ref = csim_ref.run_circuit(n, gates)
    assert np.max(np.abs(true - ref)) < 1e-12
    assert sorted(dst[b] for b in range(n - C)) == list(range(n - C))


def test_stage_chunk_permutation_leaves_low_qubits_alone():
    import qulacs
    from qulacs import _native
    L = _native.load_library()
    c = qulacs.QuantumCircuit(6)
    c.add_SWAP_gate(0, 5)     # touches a chunk bit: a real gate
    c.add_X_gate(1)
    c.add_SWAP_gate(3, 5)     # folded
    c.add_X_gate(4)           # folded
    c.add_H_gate(3)           # relabelled to qubit 5
    arr = _native.make_gate_array(c._gates)
    out = (_native.qs_gate * 5)()
    cnt = ct.c_size_t()
    dst = (ct.c_int32 * 4)()
    flip = ct.c_uint64()
    assert L.qs_stage_chunk_permutation(arr, 5, 6, 2, 0, out, ct.byref(cnt), dst, ct.byref(flip)) == 0
    assert cnt.value == 3
    assert [out[k].targets[0] for k in range(3)] == [0, 1, 5]
    assert list(dst) == [0, 3, 2, 1] and flip.value == 1 << 2


def test_bench_workload_update_count_qft30():
    """The QFT n=30 bench workload's amplitude-gate updates per apply, as
    bench.py's reference arm computes them on the host, equal the engine's
    device count for that workload (341525397504, read from its stats on a
    B200)."""
    import bench
    spec = bench.workload_spec("qft30")
    gates, updates = bench.reference_setup(spec)
    assert len(gates) == 456
    assert updates == 341525397504

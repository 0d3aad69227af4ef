"""The measured configurations at reduced size, against the FP64 oracle and
the reference model (run with -m gpu).

Each test builds a configuration's circuit with its construction (seeded
brickwork, hardware-efficient ansatz, QAOA MaxCut), fuses it as
script/run_sim.py does (optimize(block_size=2)) and runs it through the
compressed pipeline at the reference's default bounds (BITCOMP_REL_EB 1e-3,
BITCOMP_ABS_EB 1e-7), in complex128 and complex64.  Bars, per result:

* fidelity |<psi_FP64|psi>| >= 0.999 against the reference's csim FP64
  kernels on the same gates, and the largest amplitude error below 1e-3;
* fidelity at least the reference model's: the oracle's restatement of the
  reference's stage loop with its compander + Bitcomp quantiser emulated
  (oracle.codec.ref_compander_roundtrip) at the same bounds, minus 1e-4;
* zero-block masks and stage lists equal to the oracle's restatement of the
  reference planner and pipeline under the same zero test;
* energies (hardware-efficient ansatz, QAOA) within 5e-3 of the FP64 energy.

The update count that bench.py's reference arm divides by is checked here
against the engine's own count on the QFT workload family.
"""
import numpy as np
import pytest

import helpers
from oracle import codec as oc
from oracle import csim_ref, pipeline, planner

pytestmark = pytest.mark.gpu

FID = 0.999
AMP_TOL = 1e-3
ENERGY_TOL = 5e-3


@pytest.fixture(scope="module")
def qulacs_mod():
    import qulacs
    from qulacs import _native
    _native.load_library()
    return qulacs


def _run(qulacs, c, B, I, dtype):
    from qulacs import _native
    cq = qulacs.CompressedQuantumState(c.get_qubit_count(), B, dtype=dtype, eps_rel=1e-3, eps_abs=1e-7,
                                       flags=_native.QS_FLAG_QUIET)
    cq.partition_and_register_circuit(c, I, 0)
    cq.apply_circuit()
    return cq


def _oracle(c, n, B, I, codec=None, zero_test="exact"):
    g = planner.describe(c._gates)
    st = planner.partition_circuit(g, B, I)
    maps, counts = planner.make_block_groups(g, st, n, B)
    o = pipeline.CompressedOracle(n, B, codec=codec, zero_test=zero_test)
    o.apply(c._gates, st, maps, counts)
    return o, st


def _check_config(qulacs, c, B, I, dtype):
    n = c.get_qubit_count()
    ref = csim_ref.run_circuit(n, c._gates)
    cq = _run(qulacs, c, B, I, dtype)
    v = cq.get_vector()
    f = helpers.fidelity(ref, v)
    assert f >= FID, f
    assert np.abs(v - ref).max() < AMP_TOL
    # the engine's default zero test: every component quantises to code 0
    L = oc.params(dtype == "complex128", 1e-3, 1e-7)[1]
    o, st = _oracle(c, n, B, I, zero_test=("code", L))
    assert cq.get_stage_list() == st
    assert np.array_equal(cq.get_zero_mask(), o.mask())
    # the reference model at the same bounds
    o_ref, _ = _oracle(c, n, B, I, codec=lambda x: oc.ref_compander_roundtrip_complex(x, 1e-3, 1e-7))
    f_ref = helpers.fidelity(ref, o_ref.vector())
    assert f >= f_ref - 1e-4, (f, f_ref)
    return cq, ref


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
def test_brickwork20(qulacs_mod, dtype):
    """Brickwork n=20, 20 layers (the n=32 configuration's construction),
    B=12, I=4: a dense state with no zero blocks after the first layers."""
    from qompsim import circuits as C
    c = helpers.optimized(C.brickwork(20, 20, seed=0), 12)
    cq, _ = _check_config(qulacs_mod, c, 12, 4, dtype)
    assert cq.get_zero_mask().all()


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
def test_hea16_forward(qulacs_mod, dtype):
    """Hardware-efficient ansatz n=16, depth 8 (RY RZ per qubit + CNOT
    ladder), B=10, I=4, compressed forward pass and its energy
    H = sum Z_i Z_i+1 + 0.5 sum X_i."""
    from qompsim import circuits as C
    n = 16
    c = helpers.optimized(C.hea(n, 8, seed=0), 10)
    cq, ref = _check_config(qulacs_mod, c, 10, 4, dtype)
    obs = qulacs_mod.Observable(n)
    for coef, pauli, qubits in C.hea_observable_terms(n):
        obs.add_operator(coef, " ".join(f"{p} {q}" for p, q in zip(pauli, qubits)))
    s = qulacs_mod.QuantumState(n)
    s.load(ref)
    assert abs(obs.get_expectation_value(cq) - obs.get_expectation_value(s)) < ENERGY_TOL


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
def test_qaoa20(qulacs_mod, dtype):
    """QAOA MaxCut n=20, p=4 on a seeded 3-regular graph (the n=34
    configuration's construction), B=10, I=4, and its cut energy
    sum over edges of Z_a Z_b."""
    from qompsim import circuits as C
    n = 20
    c = helpers.optimized(C.qaoa_maxcut(n, 4, seed=0), 10)
    cq, ref = _check_config(qulacs_mod, c, 10, 4, dtype)
    obs = qulacs_mod.Observable(n)
    for a, b in C.regular_graph_edges(n, 3, 0):
        obs.add_operator(1.0, f"Z {a} Z {b}")
    s = qulacs_mod.QuantumState(n)
    s.load(ref)
    assert abs(obs.get_expectation_value(cq) - obs.get_expectation_value(s)) < ENERGY_TOL


@pytest.mark.parametrize("n,B", [(20, 14), (22, 16), (24, 18)])
def test_workload_update_count(qulacs_mod, n, B):
    """bench.py's reference arm divides the QFT workload's update count,
    computed on the host from the stage plan and block support, by its time:
    it equals the engine's own device count."""
    import bench
    from qompsim import circuits as C
    c = helpers.optimized(C.qft_basis(n, seed=0), B)
    cq = _run(qulacs_mod, c, B, 4, "complex128")
    assert bench.workload_updates(list(c._gates), n, B, 4) == int(cq.get_stats()["amp_gate_updates"])

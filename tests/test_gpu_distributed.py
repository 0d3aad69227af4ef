"""The engine's half-store exchange and the sharded compressed state on one
GPU (run with -m gpu).

qs_export_half / qs_import_half move compressed chunks between two stores
of one geometry without decoding them: the receiving store's decoded
amplitudes at the received positions equal the sender's bit for bit.  The
sharded state runs P ranks as threads of this process, each with its own
compressed store and stream, exchanging packed halves through host-side
hand-over (no kernel waits on another rank's), against the reference's csim
FP64 kernels on the whole state.
"""
import threading

import numpy as np
import pytest

import helpers  # noqa: F401  (sys.path)
from oracle import csim_ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def qulacs_mod():
    import qulacs
    from qulacs import _native
    _native.load_library()
    return qulacs


def _rand_state(n, seed, zero_blocks_of=None):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    if zero_blocks_of is not None:
        B, keep = zero_blocks_of
        blk = np.arange(1 << n) >> B
        v[~np.isin(blk, keep)] = 0
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
@pytest.mark.parametrize("qubit", [8, 9, 10])   # chunk-level (8 < B=9) and block-level (9, 10)
@pytest.mark.parametrize("value", [0, 1])
def test_half_exchange_moves_codes(qulacs_mod, dtype, qubit, value):
    from qulacs.distributed import CompressedShard
    n, B = 11, 9
    a = CompressedShard(n, B, dtype=dtype)
    b = CompressedShard(n, B, dtype=dtype)
    if a.chunk_bits > qubit:
        pytest.skip("qubit inside the chunk bits")
    a.state.load(_rand_state(n, 1))
    # b: only blocks 0 and 3 stored, so the import meets unstored blocks
    b.state.load(_rand_state(n, 2, zero_blocks_of=(B, [0, 3])))
    va, vb = a.vector(), b.vector()
    buf = a.export_half(qubit, value)
    b.import_half(qubit, value, buf)
    got = b.vector()
    sel = ((np.arange(1 << n) >> qubit) & 1) == value
    assert np.array_equal(got[sel], va[sel])
    assert np.array_equal(got[~sel], vb[~sel])
    # stored-block bookkeeping: a block is stored when any of its amplitudes is
    mask = b.state.get_zero_mask().astype(bool)
    nz = np.abs(got.reshape(-1, 1 << B)).max(axis=1) > 0
    assert np.all(mask >= nz)
    assert np.all(b.state.get_block_bytes()[~mask] == 0)
    # the store keeps working: one more circuit on it
    from qulacs import QuantumCircuit
    c = QuantumCircuit(n)
    c.add_H_gate(qubit)
    c.add_CNOT_gate(qubit, 0)
    b.apply([([qubit], np.array([[1, 1], [1, -1]]) / np.sqrt(2)), ([qubit, 0], np.eye(4)[[0, 3, 2, 1]])])
    ref = csim_ref.run_circuit(n, c._gates, init=got)
    # re-quantised at the default bound (relative 1e-3)
    assert np.abs(b.vector() - ref).max() < 2e-3 * np.abs(ref).max()


def test_import_rejects_foreign_buffer(qulacs_mod):
    import torch
    from qulacs import _native
    from qulacs.distributed import CompressedShard
    a = CompressedShard(10, 8)
    b = CompressedShard(11, 8)
    buf = a.export_half(8, 0)
    with pytest.raises(_native.QompsimError):
        b.import_half(8, 0, buf)
    bad = buf.clone()
    bad[:8] = 0
    with pytest.raises(_native.QompsimError):
        a.import_half(8, 0, bad)
    del torch


def _sharded_run(n, B, P, circuit, dtype, **kw):
    from qulacs import distributed as D
    hub = D.ThreadExchange(P, timeout=120)
    out, errs, ex = {}, [], {}

    def rank(r):
        try:
            import torch
            torch.cuda.set_device(0)
            st = D.ShardedCompressedQuantumState(n, B, dtype=dtype, exchange=hub.endpoint(r), **kw)
            st.partition_and_register_circuit(circuit, 3)
            st.apply_circuit()
            out[r] = st.get_vector()
            ex[r] = (st.exchanges, st.exchanged_bytes)
        except Exception as e:  # noqa: BLE001
            errs.append(repr(e))

    th = [threading.Thread(target=rank, args=(r,)) for r in range(P)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    assert not errs, errs
    return out, ex


@pytest.mark.parametrize("P", [2, 4])
def test_sharded_compressed_matches_csim(qulacs_mod, P):
    """Random circuits (H, rotations, CNOT, CZ, SWAP, random 2-qubit unitaries)
    on n=13 over P ranks, complex128 at a tight bound, against csim."""
    import test_distributed as T
    n, B = 13, 9
    c = T._circuit(n, 80, seed=20 + P)
    ref = csim_ref.run_circuit(n, c._gates)
    out, ex = _sharded_run(n, B, P, c, "complex128", eps_rel=2.0 ** -24, eps_abs=1e-14)
    for r in range(P):
        assert np.abs(out[r] - ref).max() < 1e-6
    assert ex[0][0] > 0 and ex[0][1] > 0


def test_sharded_qft_default_bounds(qulacs_mod):
    """QFT n=16 over 2 ranks at the default bounds: fidelity >= 0.999 against
    the analytic state, like the single-store engine."""
    from qompsim import circuits as C
    from qulacs.circuit import QuantumCircuitOptimizer
    n, B = 16, 10
    c = C.qft_basis(n, seed=3)
    QuantumCircuitOptimizer(sv_block_size=B).optimize(c, block_size=2)
    out, _ = _sharded_run(n, B, 2, c, "complex128")
    ref = csim_ref.run_circuit(n, c._gates)
    f = abs(np.vdot(ref, out[0])) / (np.linalg.norm(ref) * np.linalg.norm(out[0]))
    assert f >= 0.999

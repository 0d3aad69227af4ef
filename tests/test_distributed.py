"""The sharded compressed state's orchestration on the CPU (no GPU).

Ranks hold dense numpy local stores (NumpyShard) and exchange halves either
as threads of this process (ThreadExchange) or as gloo processes
(TorchExchange): the layout logic -- local application of gates whose global
qubits do not mix, exchanges before gates that mix a global qubit, SWAP as
relabelling, the final reordering -- is checked against a single dense
state.  The engine's own export/import is checked on the GPU
(tests/test_gpu_engine.py).
"""
import os
import socket
import sys
import threading

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "compression-based-state-vector-simulator_b200"))


def _circuit(n, ngates, seed):
    import qulacs
    from qulacs import gate
    rng = np.random.default_rng(seed)
    c = qulacs.QuantumCircuit(n)
    for q in range(n):
        c.add_H_gate(q)
    for _ in range(ngates):
        k = int(rng.integers(0, 9))
        a, b = (int(x) for x in rng.choice(n, 2, replace=False))
        if k == 0:
            c.add_RZ_gate(a, float(rng.uniform(0, 6.3)))
        elif k == 1:
            c.add_RX_gate(a, float(rng.uniform(0, 6.3)))
        elif k == 2:
            c.add_CNOT_gate(a, b)
        elif k == 3:
            c.add_CZ_gate(a, b)
        elif k == 4:
            c.add_SWAP_gate(a, b)
        elif k == 5:
            m = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))[0]
            c.add_dense_matrix_gate([a, b], m)
        elif k == 6:
            c.add_U3_gate(a, *(float(x) for x in rng.uniform(0, 6.3, 3)))
        elif k == 7:
            c.add_T_gate(a)
        else:
            c.add_gate(gate.DenseMatrix([a], np.diag(np.exp(1j * rng.uniform(0, 6.3, 2)))))
    return c


def _dense(n, c):
    from qulacs import distributed as D
    s = D.NumpyShard(n)
    s.set_basis(0)
    s.apply([D.gate_as_dense(g) for g in c._gates])
    return s.vector()


def _run_threads(n, P, c, chunk_bits=2):
    from qulacs import distributed as D
    hub = D.ThreadExchange(P, timeout=60)
    g = P.bit_length() - 1
    out, errs, stats = {}, [], {}

    def rank(r):
        try:
            st = D.ShardedCompressedQuantumState(n, 0, exchange=hub.endpoint(r),
                                                 shard=D.NumpyShard(n - g, chunk_bits=chunk_bits))
            st.partition_and_register_circuit(c, 4)
            st.apply_circuit()
            out[r] = st.get_vector()
            stats[r] = (st.exchanges, st.l2p)
        except Exception as e:  # noqa: BLE001
            errs.append(e)

    th = [threading.Thread(target=rank, args=(r,)) for r in range(P)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=120)
    assert not errs, errs
    return out, stats


@pytest.mark.parametrize("P", [2, 4])
def test_thread_ranks_match_dense(P):
    n = 7
    c = _circuit(n, 60, seed=P)
    ref = _dense(n, c)
    out, stats = _run_threads(n, P, c)
    for r in range(P):
        assert np.abs(out[r] - ref).max() < 1e-12
        assert stats[r][1] == list(range(n))          # layout restored
    assert stats[0][0] > 0                            # the circuit needed exchanges
    assert len({s[0] for s in stats.values()}) == 1   # every rank made the same exchanges


def test_non_mixing_global_gates_need_no_exchange():
    """Phases, CZ and controls on global qubits restrict to local gates."""
    import qulacs
    n, P = 6, 4
    c = qulacs.QuantumCircuit(n)
    for q in range(n - 2):
        c.add_H_gate(q)
    c.add_RZ_gate(5, 0.3)
    c.add_CZ_gate(4, 5)
    c.add_CNOT_gate(5, 1)      # control on a global qubit, target local
    c.add_CZ_gate(0, 4)
    c.add_T_gate(4)
    ref = _dense(n, c)
    out, stats = _run_threads(n, P, c)
    assert stats[0][0] == 0
    for r in range(P):
        assert np.abs(out[r] - ref).max() < 1e-12


def test_swap_gates_relabel_without_exchange():
    import qulacs
    n, P = 6, 2
    c = qulacs.QuantumCircuit(n)
    c.add_H_gate(0)
    c.add_RX_gate(2, 0.7)
    c.add_SWAP_gate(0, 5)      # qubit 0's amplitudes now sit under global qubit 5
    c.add_CNOT_gate(1, 2)
    ref = _dense(n, c)
    out, stats = _run_threads(n, P, c)
    for r in range(P):
        assert np.abs(out[r] - ref).max() < 1e-12
    # the final reordering puts logical 5 back at the global position: one exchange
    assert stats[0][0] == 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _gloo_rank(rank, world, port, n, seed, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "compression-based-state-vector-simulator_b200"))
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from qulacs import distributed as D
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        g = world.bit_length() - 1
        c = _circuit(n, 50, seed)
        st = D.ShardedCompressedQuantumState(n, 0, exchange=D.TorchExchange(),
                                             shard=D.NumpyShard(n - g, chunk_bits=2))
        st.partition_and_register_circuit(c, 4)
        st.apply_circuit()
        q.put((rank, st.get_vector(), st.exchanges))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_gloo_ranks_match_dense(world):
    import torch.multiprocessing as mp
    n, seed = 7, 11
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, n, seed, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = _dense(n, _circuit(n, 50, seed))
    for _, vec, ex in got:
        assert np.abs(vec - ref).max() < 1e-12
        assert ex > 0

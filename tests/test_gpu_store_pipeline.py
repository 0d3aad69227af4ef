"""Store round trips on two handles that overlap (run with -m gpu).

A caller running circuits back to back keeps two handles of one geometry on
two CUDA streams and host threads: each imports its input store from pinned
host memory, takes its turn at apply_circuit and exports its result store
while the other handle's passes run.  apply_circuit reads its per-stage
"every block stored" flag and its end-of-apply counters through mapped host
memory written by its own kernels, so these overlapping exports must change
nothing: every step's decoded result equals the serial run's bit for bit,
and so do the per-apply counters (stages, passes, bytes, updates, the stage
the merged tail ran from).
"""
import ctypes as ct
import threading

import numpy as np
import pytest

import helpers  # noqa: F401  (sys.path)

pytestmark = pytest.mark.gpu

_COUNTERS = ("stages", "passes", "tiles", "bytes_read", "bytes_written", "amp_gate_updates", "merged_from",
             "tail_passes", "code_move_passes", "perm_passes")


def _setup(n, B, I, dtype):
    import qulacs
    from qulacs import _native
    from qulacs.circuit import QuantumCircuitOptimizer
    from qompsim import circuits as C
    _native.load_library()
    c = C.qft_basis(n, seed=3)
    QuantumCircuitOptimizer(sv_block_size=B).optimize(c, block_size=2)

    def make():
        s = qulacs.CompressedQuantumState(n, B, dtype=dtype, eps_rel=1e-3, eps_abs=1e-7,
                                          flags=_native.QS_FLAG_QUIET)
        s.partition_and_register_circuit(c, I, 0)
        return s
    return make, _native


# (20, 8): 4096 blocks, so the "every block stored" test runs over several CTAs
@pytest.mark.parametrize("n,B,dtype", [(22, 16, "complex128"), (22, 16, "complex64"), (20, 8, "complex64")])
def test_overlapping_handles_match_serial(n, B, dtype):
    import torch
    I, steps = 4, 3
    make, _native = _setup(n, B, I, dtype)
    L = _native.lib()

    ref = make()
    ref.set_computational_basis(0)
    blob_in = ref.export_store()
    ref.apply_circuit()
    want_vec = ref.get_vector(renormalize=False)
    want_stats = {k: ref.get_stats()[k] for k in _COUNTERS}
    out_size = len(ref.export_store())
    del ref

    h_in = torch.frombuffer(bytearray(blob_in), dtype=torch.uint8).pin_memory()
    handles = [make(), make()]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    outs = [torch.empty(out_size + (1 << 20), dtype=torch.uint8).pin_memory() for _ in handles]
    for h, s in zip(handles, streams):
        _native.check(L.qs_set_stream(h._h, ct.c_void_p(s.cuda_stream)), h._h)
    turn = threading.Lock()
    results = [[] for _ in handles]
    errs = []

    def run(k):
        h, hout = handles[k], outs[k]
        try:
            for _ in range(steps):
                _native.check(L.qs_import_store(h._h, ct.c_void_p(h_in.data_ptr()), len(blob_in)), h._h)
                with turn:
                    h.apply_circuit()
                stats = {key: h.get_stats()[key] for key in _COUNTERS}
                sz = ct.c_uint64()
                _native.check(L.qs_export_store(h._h, ct.c_void_p(hout.data_ptr()), hout.numel(), ct.byref(sz)),
                              h._h)
                results[k].append((stats, bytes(hout[:sz.value].numpy())))
        except Exception as e:  # noqa: BLE001
            errs.append(repr(e))

    th = [threading.Thread(target=run, args=(k,)) for k in range(len(handles))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs[0]

    check = make()
    for k in range(len(handles)):
        assert len(results[k]) == steps
        for stats, blob in results[k]:
            assert stats == want_stats
            check.import_store(blob)
            np.testing.assert_array_equal(check.get_vector(renormalize=False), want_vec)
    for h in handles:
        _native.check(L.qs_set_stream(h._h, None), h._h)

"""GPU parity tests of the engine through its C ABI (run with -m gpu).

Bars:
* codec: device codes, packed words, frames and decoded values equal the
  CPU statement (oracle/codec_oracle.c) bit for bit;
* uncompressed path (QuantumState, fused tile passes and the plain per-gate
  kernels): complex128 within 1e-12 per amplitude of the reference's csim
  kernels; complex64 within 2e-6;
* compressed path: zero-block masks and stage lists equal the oracle's
  restatement of the reference planner/pipeline; amplitudes within the codec's
  error budget of the FP64 csim result; fidelity |<psi_ref|psi>| >= 0.999 at
  the reference's default bounds (BITCOMP_REL_EB 1e-3, BITCOMP_ABS_EB 1e-7).
"""
import math

import numpy as np
import pytest

import helpers
from oracle import codec as oc
from oracle import csim_ref, pipeline, planner

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12
F32_TOL = 2e-6


@pytest.fixture(scope="module")
def qulacs_mod():
    import qulacs
    from qulacs import _native
    _native.load_library()
    return qulacs


# ------------------------------------------------------------------ codec
@pytest.mark.parametrize("f64", [True, False])
@pytest.mark.parametrize("C", [4, 5, 7, 8])
def test_device_codec_bit_identical(qulacs_mod, f64, C):
    import ctypes as ct
    from qulacs import _native
    L = _native.lib()
    rng = np.random.default_rng(100 + C)
    nch = 64
    n = 2 << C
    vals = np.concatenate([
        np.zeros(n), np.eye(1, n, 3).ravel(),
        *[rng.normal(scale=10.0 ** -rng.uniform(0, 7), size=n) for _ in range(nch - 3)],
        np.where(rng.random(n) < 0.1, rng.normal(size=n), 0.0),
    ])
    dt = np.float64 if f64 else np.float32
    vals = np.ascontiguousarray(vals.astype(dt))
    words = np.zeros(nch * n, dtype=np.uint32)
    bases = np.zeros(nch, dtype=np.int32)
    widths = np.zeros(nch, dtype=np.uint32)
    dec = np.zeros_like(vals)
    st = L.qs_codec_test(0 if f64 else 1, 1e-3, 1e-7, C, vals.ctypes.data, nch,
                         words.ctypes.data_as(ct.POINTER(ct.c_uint32)), bases.ctypes.data_as(ct.POINTER(ct.c_int32)),
                         widths.ctypes.data_as(ct.POINTER(ct.c_uint32)), dec.ctypes.data)
    assert st == 0, L.qs_dense_last_error(None)
    m, Lp = oc.params(f64, 1e-3, 1e-7)
    for k in range(nch):
        v = vals[k * n:(k + 1) * n]
        w, b, wd = oc.encode_chunk(v, C, m, Lp)
        assert (bases[k], widths[k]) == (b, wd)
        assert np.array_equal(words[k * n:k * n + w.size], w)
        assert np.array_equal(dec[k * n:(k + 1) * n], oc.decode_chunk(w, C, b, wd, m, Lp, f64))


# ------------------------------------------------------------------ uncompressed
def _dense_run(qulacs, c, dtype="complex128", pergate=False):
    s = qulacs.QuantumState(c.get_qubit_count(), dtype=dtype)
    s._apply_gates(c._gates, pergate=pergate)
    return s.get_vector()


@pytest.mark.parametrize("key", sorted(helpers.golden_circuits()))
@pytest.mark.parametrize("pergate", [False, True])
def test_dense_golden_complex128(qulacs_mod, key, pergate):
    c = helpers.build_circuit(key)
    v = _dense_run(qulacs_mod, c, pergate=pergate)
    assert np.abs(v - helpers.golden_states()[key]).max() < F64_TOL


@pytest.mark.parametrize("n,seed", [(6, 1), (9, 2), (12, 3), (14, 4), (16, 5)])
def test_dense_random_complex128(qulacs_mod, n, seed):
    c = helpers.random_circuit(n, 120, seed)
    ref = csim_ref.run_circuit(n, c._gates)
    for pergate in (False, True):
        v = _dense_run(qulacs_mod, c, pergate=pergate)
        assert np.abs(v - ref).max() < F64_TOL, pergate


@pytest.mark.parametrize("n,seed", [(10, 7), (15, 8)])
def test_dense_random_complex64(qulacs_mod, n, seed):
    c = helpers.random_circuit(n, 80, seed)
    ref = csim_ref.run_circuit(n, c._gates)
    v = _dense_run(qulacs_mod, c, dtype="complex64")
    assert np.abs(v - ref).max() < F32_TOL * 10


def test_dense_norm_load_and_basis(qulacs_mod):
    s = qulacs_mod.QuantumState(8)
    rng = np.random.default_rng(0)
    v = rng.normal(size=256) + 1j * rng.normal(size=256)
    s.load(v)
    assert abs(s.get_squared_norm() - np.vdot(v, v).real) < 1e-9
    assert np.array_equal(s.get_vector(), v)
    s.set_computational_basis(77)
    w = s.get_vector()
    assert w[77] == 1 and np.count_nonzero(w) == 1


# ------------------------------------------------------------------ compressed
def _compressed(qulacs, c, B, I, dtype="complex128", eps_rel=1e-3, eps_abs=1e-7, flags=None, basis=None,
                host_store=False):
    from qulacs import _native
    f = _native.QS_FLAG_QUIET if flags is None else flags
    cq = qulacs.CompressedQuantumState(c.get_qubit_count(), B, dtype=dtype, eps_rel=eps_rel, eps_abs=eps_abs,
                                       flags=f, host_store=host_store)
    if basis is not None:
        cq.set_computational_basis(basis)
    cq.partition_and_register_circuit(c, I, 0)
    cq.apply_circuit()
    return cq


def _oracle_masks(c, n, B, I, codec=None, zero_test="exact"):
    """Oracle run of the reference's stage loop; zero_test as in
    oracle.pipeline (the engine's default is ("code", L))."""
    g = planner.describe(c._gates)
    st = planner.partition_circuit(g, B, I)
    maps, counts = planner.make_block_groups(g, st, n, B)
    o = pipeline.CompressedOracle(n, B, codec=codec, zero_test=zero_test)
    o.apply(c._gates, st, maps, counts)
    return o, st


def test_ghz20_config(qulacs_mod):
    from qompsim import circuits as C
    c = helpers.optimized(C.ghz_fanout(20), 12)
    cq = _compressed(qulacs_mod, c, 12, 4)
    assert [len(s) for s in cq.get_stage_list()] == [15, 4]
    assert list(np.nonzero(cq.get_zero_mask())[0]) == [0, 15, 255]
    v = cq.get_vector()
    ref = np.zeros(1 << 20, dtype=np.complex128)
    ref[0] = ref[-1] = 1 / math.sqrt(2)
    assert np.abs(v - ref).max() < 1e-3
    assert helpers.fidelity(ref, v) > 0.999999
    hist = cq.get_SV_bytes_history()
    assert len(hist) == 3 and cq.get_max_SV_bytes() == max(hist)
    bb = cq.get_block_bytes()
    assert np.all(bb[cq.get_zero_mask() == 0] == 0) and np.all(bb[[0, 15, 255]] > 0)
    times = cq.get_total_times()
    assert list(times) == ["decomp", "gate", "comp", "fused_swap", "allgather", "hmalloc", "dmalloc", "h2d", "d2h",
                           "dfree"]
    assert times["gate"] > 0


def test_ghz20_stage0_mask(qulacs_mod):
    """Register only the first stage (register_circuit_stages) and read the
    mask between the stages: {0, 15}."""
    from qompsim import circuits as C
    c = helpers.optimized(C.ghz_fanout(20), 12)
    g = planner.describe(c._gates)
    st = planner.partition_circuit(g, 12, 4)
    maps, counts = planner.make_block_groups(g, st, 20, 12)
    from qulacs import _native
    cq = qulacs_mod.CompressedQuantumState(20, 12, flags=_native.QS_FLAG_QUIET)
    groups = [[[b for b in range(256) if maps[0][b] == gid] for gid in range(counts[0])]]
    cq.register_circuit_stages(c, [st[0]], groups)
    cq.apply_circuit()
    assert list(np.nonzero(cq.get_zero_mask())[0]) == [0, 15]


@pytest.mark.parametrize("key", ["ghz_10", "qft_8", "hea_9", "qaoa_9", "wstate_8", "bv_9", "grover_11",
                                 "ising_8", "qsvm_8", "cc_9", "hadamard_8", "seq_hadamard_9"])
@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
def test_compressed_golden_masks_and_values(qulacs_mod, key, dtype):
    c = helpers.optimized(helpers.build_circuit(key), 4)
    n = c.get_qubit_count()
    ref = helpers.golden_states()[key]
    # tight relative bound, absolute bound (zero-test threshold 2^-(L+1)) well
    # above the relative quantisation noise of intermediate states, so that
    # exact cancellations (H ... H) read as zero on both sides
    L = oc.params(dtype == "complex128", 2.0 ** -20, 1e-4)[1]
    for B, I in [(4, 1), (5, 2), (4, 4), (n - 2, 1)]:
        cq = _compressed(qulacs_mod, c, B, I, dtype=dtype, eps_rel=2.0 ** -20, eps_abs=1e-4)
        o, st = _oracle_masks(c, n, B, I, zero_test=("code", L))
        assert cq.get_stage_list() == st
        assert np.array_equal(cq.get_zero_mask(), o.mask()), (B, I)
        v = cq.get_vector()
        tol = 1e-3
        assert np.abs(v - ref).max() < tol, (B, I)
        # reference default bounds
        cq = _compressed(qulacs_mod, c, B, I, dtype=dtype)
        assert helpers.fidelity(ref, cq.get_vector()) > 0.999, (B, I)


@pytest.mark.parametrize("n,B,seed", [(14, 8, 1), (16, 10, 2), (16, 6, 3)])
def test_compressed_qft_analytic(qulacs_mod, n, B, seed):
    from qompsim import circuits as C
    c = helpers.optimized(C.qft_basis(n, seed), B)
    cq = _compressed(qulacs_mod, c, B, 4)
    v = cq.get_vector()
    ref = C.qft_expected(n, C.qft_input(n, seed))
    f = helpers.fidelity(ref, v)
    assert f > 0.999, f
    # the reference model: same stages, compander + Bitcomp quantiser emulated
    o, _ = _oracle_masks(c, n, B, 4, codec=lambda x: oc.ref_compander_roundtrip_complex(x, 1e-3, 1e-7))
    f_ref = helpers.fidelity(ref, o.vector())
    assert f >= f_ref - 1e-4, (f, f_ref)


@pytest.mark.parametrize("n,seed", [(12, 11), (15, 12)])
def test_compressed_random_circuits_vs_csim(qulacs_mod, n, seed):
    c = helpers.random_circuit(n, 100, seed)
    ref = csim_ref.run_circuit(n, c._gates)
    L = oc.params(True, 2.0 ** -22, 1e-13)[1]
    for B in (4, 7, n - 3):
        cq = _compressed(qulacs_mod, c, B, 3, eps_rel=2.0 ** -22, eps_abs=1e-13)
        v = cq.get_vector()
        assert np.abs(v - ref).max() < 1e-5, B
        o, _ = _oracle_masks(c, n, B, 3, zero_test=("code", L))
        assert np.array_equal(cq.get_zero_mask(), o.mask())


def _permute_chunks_run(qulacs, c, B, I, on, monkeypatch, **kw):
    monkeypatch.setenv("QOMPSIM_PERMUTE_CHUNKS", "1" if on else "0")
    # per-stage plans: a merged tail would plan the two variants' passes differently
    monkeypatch.setenv("QOMPSIM_MERGE_TAIL", "0")
    cq = _compressed(qulacs, c, B, I, **kw)
    return cq, cq.get_vector(renormalize=False), cq.get_zero_mask(), cq.get_SV_bytes_history(), cq.get_stats()


def test_chunk_permutation_stage_bit_identical(qulacs_mod, monkeypatch):
    """Stages made only of SWAP / X gates on qubits >= C run as header-only
    passes: the stored state, masks and byte history equal those of decoding,
    permuting and re-encoding every chunk."""
    import qulacs
    n, B = 14, 8
    c = qulacs.QuantumCircuit(n)
    for q in range(n):
        c.add_H_gate(q)
    for q in range(n - 1):
        c.add_RZ_gate(q, 0.3 + q)
        c.add_CNOT_gate(q, q + 1)
    c.add_SWAP_gate(9, 13)
    c.add_X_gate(12)
    c.add_SWAP_gate(8, 10)
    c.add_SWAP_gate(11, 12)
    c.add_X_gate(11)
    c.add_RY_gate(2, 0.7)
    a = _permute_chunks_run(qulacs_mod, c, B, 2, True, monkeypatch)
    b = _permute_chunks_run(qulacs_mod, c, B, 2, False, monkeypatch)
    assert a[4]["perm_passes"] >= 1 and b[4]["perm_passes"] == 0
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[2], b[2])
    assert list(a[3]) == list(b[3])
    ref = csim_ref.run_circuit(n, c._gates)
    assert helpers.fidelity(ref, a[0].get_vector()) > 0.999


@pytest.mark.parametrize("n,B,seed", [(12, 8, 21), (12, 6, 22), (15, 9, 23)])
def test_chunk_permutation_random_circuits(qulacs_mod, monkeypatch, n, B, seed):
    """Random circuits dense in SWAP / X / permutation gates on high qubits:
    folded into chunk permutations, against csim and against the unfolded
    plan (tight codec bounds: both agree to the codec's error)."""
    C = min(8, B)
    c = helpers.perm_heavy_circuit(n, C, 60, seed)
    ref = csim_ref.run_circuit(n, c._gates)
    kw = dict(eps_rel=2.0 ** -22, eps_abs=1e-13)
    a = _permute_chunks_run(qulacs_mod, c, B, 3, True, monkeypatch, **kw)
    b = _permute_chunks_run(qulacs_mod, c, B, 3, False, monkeypatch, **kw)
    assert np.abs(a[1] - ref).max() < 1e-5
    assert np.abs(a[1] - b[1]).max() < 1e-5
    assert np.array_equal(a[2], b[2])
    L = oc.params(True, 2.0 ** -22, 1e-13)[1]
    o, _ = _oracle_masks(c, n, B, 3, zero_test=("code", L))
    assert np.array_equal(a[2], o.mask())


@pytest.mark.parametrize("key", ["ghz_10", "qft_8", "hea_9", "qaoa_9", "ising_8", "qsvm_8", "hadamard_8"])
def test_exact_zero_test_flag(qulacs_mod, key):
    """QS_FLAG_EXACT_ZERO_TEST: the reference GPU build's exact test gives the
    oracle's masks on circuits without exact cancellations."""
    from qulacs import _native
    c = helpers.optimized(helpers.build_circuit(key), 4)
    n = c.get_qubit_count()
    for B, I in [(4, 1), (5, 2)]:
        cq = _compressed(qulacs_mod, c, B, I, flags=_native.QS_FLAG_QUIET | _native.QS_FLAG_EXACT_ZERO_TEST)
        o, _ = _oracle_masks(c, n, B, I, zero_test="exact")
        assert np.array_equal(cq.get_zero_mask(), o.mask()), (B, I)


def test_compressed_load_vector_bit_exact(qulacs_mod):
    from qulacs import _native
    n, B = 12, 6
    rng = np.random.default_rng(9)
    v = (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)) * 1e-2
    v[: 1 << B] = 0  # block 0 all zero -> not stored
    m, L = oc.params(True, 1e-3, 1e-7)
    cq = qulacs_mod.CompressedQuantumState(n, B, eps_rel=1e-3, eps_abs=1e-7, flags=_native.QS_FLAG_QUIET)
    cq.load(v)
    got = cq.get_vector(renormalize=False)
    assert np.array_equal(got, oc.roundtrip_complex(v, m, L))
    mask = cq.get_zero_mask()
    assert mask[0] == 0 and mask[1:].all()


def test_compressed_export_import_roundtrip(qulacs_mod):
    from qompsim import circuits as C
    from qulacs import _native
    c = helpers.optimized(C.qft_basis(14, 2), 8)
    cq = _compressed(qulacs_mod, c, 8, 4)
    blob = cq.export_store()
    v = cq.get_vector(renormalize=False)
    other = qulacs_mod.CompressedQuantumState(14, 8, flags=_native.QS_FLAG_QUIET)
    other.import_store(blob)
    assert np.array_equal(other.get_vector(renormalize=False), v)
    assert np.array_equal(other.get_zero_mask(), cq.get_zero_mask())
    bad = bytearray(blob)
    bad[0] ^= 0xFF
    with pytest.raises(_native.QompsimError) as e:
        other.import_store(bytes(bad))
    assert e.value.status == _native.QS_ERR_CORRUPT
    with pytest.raises(_native.QompsimError) as e:
        other.import_store(blob[:-16])
    assert e.value.status == _native.QS_ERR_CORRUPT
    # chunk headers of stored blocks: misaligned offset, offset past the
    # arena, width above 32 -- each rejected before anything is launched
    nb, nchunks = 1 << (14 - 8), 1 << (14 - 8)
    meta0 = 56 + (nb + 7) // 8 * 8 + nb * 8
    mask = np.frombuffer(blob, dtype=np.uint8, count=nb, offset=56)
    k = int(np.flatnonzero(mask)[0]) * (nchunks // nb)
    arena_bytes = int(np.frombuffer(blob, dtype=np.uint64, count=1, offset=48)[0])
    for field, value in [("offset", 8), ("offset", arena_bytes + 128), ("width", 40)]:
        bad = bytearray(blob)
        pos = meta0 + 16 * k + (0 if field == "offset" else 12)
        if field == "offset":
            bad[pos:pos + 8] = int(value).to_bytes(8, "little")
        else:
            bad[pos:pos + 4] = int(value).to_bytes(4, "little")
        with pytest.raises(_native.QompsimError) as e:
            other.import_store(bytes(bad))
        assert e.value.status == _native.QS_ERR_CORRUPT, field
    other.import_store(blob)
    assert np.array_equal(other.get_vector(renormalize=False), v)


def test_compressed_error_paths(qulacs_mod, monkeypatch):
    import qulacs
    from qulacs import _native
    cq = qulacs.CompressedQuantumState(10, 5, flags=_native.QS_FLAG_QUIET)
    with pytest.raises(_native.QompsimError) as e:
        cq.apply_circuit()
    assert e.value.status == _native.QS_ERR_STATE
    with pytest.raises(_native.QompsimError) as e:
        qulacs.CompressedQuantumState(10, 3, flags=_native.QS_FLAG_QUIET)
    assert e.value.status == _native.QS_ERR_ARG
    with pytest.raises(_native.QompsimError) as e:
        qulacs.CompressedQuantumState(10, 5, eps_rel=0.0, flags=_native.QS_FLAG_QUIET)
    assert e.value.status == _native.QS_ERR_ARG
    # an arena too small for the state: the kernel refuses to write past it
    monkeypatch.setenv("QOMPSIM_ARENA_BYTES", "4096")
    small = qulacs.CompressedQuantumState(12, 6, flags=_native.QS_FLAG_QUIET)
    c = qulacs.QuantumCircuit(12)
    for q in range(12):
        c.add_H_gate(q)
    small.partition_and_register_circuit(c, 2, 0)
    with pytest.raises(_native.QompsimError) as e:
        small.apply_circuit()
    assert e.value.status == _native.QS_ERR_CAPACITY


def test_reference_controls_flag(qulacs_mod):
    """QS_FLAG_REFERENCE_CONTROLS applies a controlled 2x2 uncontrolled (Q3)."""
    import qulacs
    from qulacs import gate as G, _native
    c = qulacs.QuantumCircuit(8)
    c.add_H_gate(5)
    g = G.DenseMatrix(0, [[0, 1], [1, 0]])
    g.add_control_qubit(5, 1)
    c.add_gate(g)
    ok = _compressed(qulacs, c, 4, 2, eps_rel=2.0 ** -20, eps_abs=1e-12)
    ref = csim_ref.run_circuit(8, c._gates)
    assert np.abs(ok.get_vector() - ref).max() < 1e-5
    quirk = _compressed(qulacs, c, 4, 2, eps_rel=2.0 ** -20, eps_abs=1e-12,
                        flags=_native.QS_FLAG_QUIET | _native.QS_FLAG_REFERENCE_CONTROLS)
    o = pipeline.CompressedOracle(8, 4, reference_controls=True)
    g_ = planner.describe(c._gates)
    st = planner.partition_circuit(g_, 4, 2)
    maps, counts = planner.make_block_groups(g_, st, 8, 4)
    o.apply(c._gates, st, maps, counts)
    assert np.abs(quirk.get_vector() - o.vector()).max() < 1e-5
    assert np.abs(quirk.get_vector() - ref).max() > 0.1


def test_checkpoint_restore(qulacs_mod):
    from qompsim import circuits as C
    from qulacs import _native
    c = helpers.optimized(C.qft_basis(13, 4), 7)
    cq = qulacs_mod.CompressedQuantumState(13, 7, flags=_native.QS_FLAG_QUIET)
    cq.partition_and_register_circuit(c, 3, 0)
    cq.set_computational_basis(5)
    cq.checkpoint(2)
    v0 = cq.get_vector(renormalize=False)
    cq.apply_circuit()
    v1 = cq.get_vector(renormalize=False)
    cq.restore(2)
    assert np.array_equal(cq.get_vector(renormalize=False), v0)
    cq.apply_circuit()
    assert np.array_equal(cq.get_vector(renormalize=False), v1)   # deterministic rerun from the checkpoint
    with pytest.raises(_native.QompsimError) as e:
        cq.restore(9)
    assert e.value.status == _native.QS_ERR_STATE


def test_run_sim_one_rank_fidelity(qulacs_mod, capfd):
    from qompsim import run_sim
    run_sim.run_sim("fidelity", "qft_basis", 12, block_size=6, inner_size=3)
    out = capfd.readouterr().out   # the stage list is printed by the C++ planner
    fid = float(out.split("Fidelity:")[1].split()[0])
    assert fid > 0.999
    assert "Circuit Stages: [" in out


def test_amplitude_slices_match_full_vectors(qulacs_mod):
    from qulacs import _native
    n, B = 12, 7
    c = helpers.optimized(helpers.random_circuit(n, 50, seed=31), B)
    cq = _compressed(qulacs_mod, c, B, 3)
    full = cq.get_vector()
    ch = 1 << cq.get_stats()["chunk_log2"]
    for first, cnt in [(0, ch), (ch * 3, ch * 5), ((1 << n) - ch, ch)]:
        assert np.array_equal(cq.get_amplitudes(first, cnt), full[first:first + cnt])
    with pytest.raises(_native.QompsimError):
        cq.get_amplitudes(1, ch)
    ds = qulacs_mod.QuantumState(n, dtype="complex128")
    c.update_quantum_state(ds)
    dv = ds.get_vector()
    assert np.array_equal(ds.get_amplitudes(100, 57), dv[100:157])
    d64 = qulacs_mod.QuantumState(n, dtype="complex64")
    c.update_quantum_state(d64)
    assert np.array_equal(d64.get_amplitudes(64, 128), d64.get_vector()[64:192])


# ------------------------------------------------------------------ sampling
@pytest.mark.parametrize("dtype,n,B", [("complex128", 12, 6), ("complex128", 14, 10), ("complex128", 10, 4),
                                       ("complex64", 13, 8), ("complex64", 12, 12)])
def test_sampling_blockwise_matches_oracle(qulacs_mod, dtype, n, B):
    """Device block masses and in-block searches with the reference's seeded
    generators on the host: the samples equal the oracle's, drawn from the
    same decoded amplitudes, index for index."""
    from oracle import sampling
    c = helpers.optimized(helpers.random_circuit(n, 60, seed=n + B), B)
    cq = _compressed(qulacs_mod, c, B, 3, dtype=dtype)
    v = cq.get_vector(renormalize=False)
    mask = cq.get_zero_mask()
    for shots, seed in [(0, 1), (1, 2), (1000, 3), (20000, 2 ** 32 - 1)]:
        got = cq.sampling_blockwise(shots, seed)
        want = sampling.sampling_blockwise(v, B, shots, seed, stored=mask)
        assert got == want, (shots, seed)
    # the samples follow |a|^2: chi-square over the 64 heaviest amplitudes
    got = np.asarray(cq.sampling_blockwise(200000, 17))
    p = np.abs(v) ** 2
    p /= p.sum()
    top = np.argsort(p)[-64:]
    cnt = np.bincount(got, minlength=v.size)[top]
    e = p[top] * got.size
    chi = float(((cnt - e) ** 2 / e).sum())
    assert chi < 64 + 6 * math.sqrt(2 * 64), chi


def test_sampling_blockwise_sparse_and_errors(qulacs_mod):
    """GHZ: all mass in the first and last blocks, every sample is 0 or
    2^n - 1.  A zero state has no mass to sample from."""
    from oracle import sampling
    from qompsim import circuits as C
    n, B = 16, 8
    cq = _compressed(qulacs_mod, C.ghz_fanout(n), B, 4)
    mask = cq.get_zero_mask()
    got = cq.sampling_blockwise(5000, 9)
    assert set(got) == {0, (1 << n) - 1}
    assert got == sampling.sampling_blockwise(cq.get_vector(renormalize=False), B, 5000, 9, stored=mask)
    z = qulacs_mod.CompressedQuantumState(10, 5, eps_rel=1e-3, eps_abs=1e-7)
    z.load(np.zeros(1 << 10, dtype=np.complex128))
    with pytest.raises(ValueError):
        z.sampling_blockwise(10, 1)


# ------------------------------------------------------------ spill tier
@pytest.mark.parametrize("dtype,circ", [("complex128", "random"), ("complex64", "random"), ("complex128", "qft")])
def test_host_store_bit_identical(qulacs_mod, dtype, circ):
    """Payload arenas in mapped host memory run the same passes: vectors,
    masks, byte histories and samples equal the HBM store's (the arena
    layout itself depends on the order in which tiles reserve space);
    checkpoints (in HBM) restore into the host arenas and exported stores
    cross between the tiers."""
    from qompsim import circuits as C
    n, B = 16, 9
    c = helpers.random_circuit(n, 120, seed=5) if circ == "random" else C.qft_basis(n, 3)
    c = helpers.optimized(c, B)
    ref = _compressed(qulacs_mod, c, B, 3, dtype=dtype)
    hs = _compressed(qulacs_mod, c, B, 3, dtype=dtype, host_store=True)
    assert hs.get_stats()["host_store"] == 1 and ref.get_stats()["host_store"] == 0
    v = ref.get_vector(renormalize=False)
    assert np.array_equal(v, hs.get_vector(renormalize=False))
    assert np.array_equal(ref.get_zero_mask(), hs.get_zero_mask())
    assert ref.get_SV_bytes_history() == hs.get_SV_bytes_history()
    assert ref.sampling_blockwise(1000, 3) == hs.sampling_blockwise(1000, 3)
    hs.checkpoint(0)
    hs.set_zero_state()
    hs.restore(0)
    assert np.array_equal(v, hs.get_vector(renormalize=False))
    hs.free_checkpoint(0)
    blob = ref.export_store()
    hs.set_zero_state()
    hs.import_store(blob)
    assert np.array_equal(v, hs.get_vector(renormalize=False))
    blob = hs.export_store()
    ref.set_zero_state()
    ref.import_store(blob)
    assert np.array_equal(v, ref.get_vector(renormalize=False))


# ------------------------------------------------------------ code-domain moves
def _moves_circuit(n, seed):
    """Random gates, then blocks of SWAP / X gates alone (bit reversal, which
    pairs chunk bits with high qubits, and X layers), then random gates."""
    import qulacs
    rng = np.random.default_rng(seed)
    c = qulacs.QuantumCircuit(n)
    for g in helpers.random_circuit(n, 40, seed)._gates:
        c.add_gate(g)
    for _ in range(2):
        for q in range(n // 2):
            c.add_SWAP_gate(q, n - 1 - q)
        for q in rng.choice(n, size=3, replace=False):
            c.add_X_gate(int(q))
    for g in helpers.random_circuit(n, 20, seed + 1)._gates:
        c.add_gate(g)
    return c


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
@pytest.mark.parametrize("circ,exact", [("qft", False), ("moves", False), ("moves", True)])
def test_code_move_passes_bit_identical(qulacs_mod, monkeypatch, dtype, circ, exact):
    """Passes made only of X / SWAP moves carry quantised codes through the
    tile; since quantise(dequantise(c)) == c the store decodes to exactly the
    values of the value-domain pass, with the same masks and byte totals."""
    from qulacs import _native
    from qompsim import circuits as C
    n, B = 16, 9
    c = helpers.optimized(C.qft_basis(n, 5), B) if circ == "qft" else _moves_circuit(n, 7)
    flags = _native.QS_FLAG_QUIET | (_native.QS_FLAG_EXACT_ZERO_TEST if exact else 0)
    out = []
    # per-stage plans: in a merged tail the SWAP stages share passes with other gates
    monkeypatch.setenv("QOMPSIM_MERGE_TAIL", "0")
    for on in ("1", "0"):
        monkeypatch.setenv("QOMPSIM_CODE_MOVES", on)
        cq = _compressed(qulacs_mod, c, B, 3, dtype=dtype, flags=flags)
        out.append((cq.get_vector(renormalize=False), cq.get_zero_mask(), cq.get_SV_bytes_history(),
                    cq.get_stats()["code_move_passes"]))
    assert out[0][3] > 0 and out[1][3] == 0
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
def test_arena_slabs_same_store(qulacs_mod, monkeypatch, dtype):
    """CTAs that sub-allocate arena slabs (forced small here) produce the same
    decoded state, masks and byte totals as exact per-tile reservations; the
    store round-trips through export / import with the slabs' slack."""
    n, B = 16, 9
    c = helpers.optimized(helpers.random_circuit(n, 150, seed=12), B)
    out = []
    for slab in ("1024", "0"):
        monkeypatch.setenv("QOMPSIM_SLAB_BYTES", slab)
        cq = _compressed(qulacs_mod, c, B, 3, dtype=dtype)
        out.append((cq.get_vector(renormalize=False), cq.get_zero_mask(), cq.get_SV_bytes_history(), cq))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]
    blob = out[0][3].export_store()
    out[1][3].import_store(blob)
    assert np.array_equal(out[1][3].get_vector(renormalize=False), out[0][0])


# ------------------------------------------------------------ merged tail
def _dense_then_random(n, seed):
    """H on every qubit (every block stored after the first stages), then a
    random circuit over every gate form, with SWAP / X gates on high qubits."""
    import qulacs
    c = qulacs.QuantumCircuit(n)
    for q in range(n):
        c.add_H_gate(q)
    for g in helpers.perm_heavy_circuit(n, 8, 50, seed)._gates:
        c.add_gate(g)
    return c


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
@pytest.mark.parametrize("n,B,I", [(16, 9, 3), (15, 8, 2)])
def test_merged_tail_matches_per_stage(qulacs_mod, monkeypatch, dtype, n, B, I):
    """Once every block is stored the remaining stages share passes: the
    merged run has the per-stage run's masks, stage list, update count and
    history length, fewer passes, and the same state within the codec's
    error (tight bounds; the two plans quantise at different points), and
    matches csim."""
    c = helpers.optimized(_dense_then_random(n, 31), B)
    ref = csim_ref.run_circuit(n, c._gates)
    kw = dict(dtype=dtype, eps_rel=2.0 ** -22 if dtype == "complex128" else 2.0 ** -20, eps_abs=1e-13)
    runs = []
    for merge in ("1", "0"):
        monkeypatch.setenv("QOMPSIM_MERGE_TAIL", merge)
        cq = _compressed(qulacs_mod, c, B, I, **kw)
        runs.append((cq, cq.get_vector(renormalize=False), cq.get_stats()))
    (m, vm, sm), (u, vu, su) = runs
    assert sm["merged_from"] >= 1 and su["merged_from"] == -1
    assert sm["tail_passes"] > 0 and sm["passes"] < su["passes"]
    assert sm["amp_gate_updates"] == su["amp_gate_updates"]
    assert m.get_stage_list() == u.get_stage_list()
    assert np.array_equal(m.get_zero_mask(), u.get_zero_mask()) and m.get_zero_mask().all()
    assert len(m.get_SV_bytes_history()) == len(u.get_SV_bytes_history())
    tol = 1e-5 if dtype == "complex128" else 5e-5
    assert np.abs(vm - vu).max() < tol
    assert np.abs(vm - ref).max() < tol
    # a second apply from the same start reuses the tail plan and repeats the result
    m.set_zero_state()
    m.apply_circuit()
    assert np.array_equal(m.get_vector(renormalize=False), vm)


# ------------------------------------------------------------ reference gpusim cross-check
@pytest.mark.parametrize("key", ["qft_8", "hea_9", "ghz_10", "qaoa_9", "grover_11"])
def test_reference_gpusim_matches_golden_and_our_dense_paths(qulacs_mod, key):
    """The reference's own plain complex128 GPU kernels (src/gpusim, built
    from source) reproduce the golden csim states, and this package's
    per-gate and fused uncompressed paths match them to 1e-12: the per-gate
    baseline of the speed-up figures is checked against the reference's GPU
    path, not only its CPU kernels."""
    from oracle import gpusim_ref
    if not gpusim_ref.available():
        pytest.skip("oracle/_ref/libgpusim_ref.so not built (the reference is not mounted where it was built)")
    c = helpers.build_circuit(key)
    ref = helpers.golden_states()[key]
    gs = gpusim_ref.GpuState(c.get_qubit_count())
    gs.apply(c._gates)
    g = gs.get_vector()
    assert np.abs(g - ref).max() < F64_TOL
    for pergate in (True, False):
        assert np.abs(_dense_run(qulacs_mod, c, pergate=pergate) - g).max() < F64_TOL


@pytest.mark.parametrize("n,seed", [(12, 51), (16, 52)])
def test_reference_gpusim_matches_random_circuits(qulacs_mod, n, seed):
    from oracle import gpusim_ref
    if not gpusim_ref.available():
        pytest.skip("oracle/_ref/libgpusim_ref.so not built")
    c = helpers.random_circuit(n, 120, seed)
    gs = gpusim_ref.GpuState(n)
    gs.apply(c._gates)
    g = gs.get_vector()
    assert np.abs(g - csim_ref.run_circuit(n, c._gates)).max() < F64_TOL
    assert np.abs(_dense_run(qulacs_mod, c, pergate=True) - g).max() < F64_TOL


# ------------------------------------------------------------ dense k-qubit gates (tensor cores)
def _haar(k, rng):
    z = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


# complex128: the output store's quantisation (relative step 2^-22 of
# amplitudes up to ~0.05); complex64: that at 2^-20 plus the 3xTF32 products
@pytest.mark.parametrize("dtype,tol", [("complex128", 2e-8), ("complex64", 3e-5)])
@pytest.mark.parametrize("targets", [[0, 3, 9, 11, 12], [12, 2, 13, 7], [10, 11, 12, 13, 1]])
def test_dense_gate_pass_matches_csim(qulacs_mod, dtype, tol, targets):
    """One dense 4- or 5-qubit gate over the compressed state
    (qs_apply_dense_gate: complex64 on the tensor cores with a 3xTF32 split,
    complex128 on the CUDA cores), targets below and above the chunk and the
    block, against the reference's csim multi-qubit kernel applied to the
    decoded input state (tight codec bounds); the gate's one-gate stage
    stores the blocks it reaches."""
    from qulacs import gate as G
    n, B = 14, 12
    rng = np.random.default_rng(sum(targets))
    c = helpers.optimized(helpers.random_circuit(n, 40, seed=61), B)
    kw = dict(dtype=dtype, eps_rel=2.0 ** -22 if dtype == "complex128" else 2.0 ** -20, eps_abs=1e-13)
    cq = _compressed(qulacs_mod, c, B, 3, **kw)
    v0 = cq.get_vector(renormalize=False)
    u = _haar(len(targets), rng)
    cq.apply_dense_gate(targets, u)
    got = cq.get_vector(renormalize=False)
    ref = csim_ref.run_circuit(n, [G.DenseMatrix(targets, u)], init=v0)
    assert np.abs(got - ref).max() < tol
    assert cq.get_zero_mask().all()
    assert cq.get_stats()["passes"] == 1


@pytest.mark.parametrize("dtype,tol", [("complex128", 1e-8), ("complex64", 1e-4)])
def test_fused_k_circuit_matches_csim(qulacs_mod, dtype, tol):
    """A random circuit fused by optimize(block_size=5) into gates on up to
    five qubits: apply_gates runs the small gates as registered circuits and
    the fused ones as dense passes; the state matches csim on the same fused
    gates (tight codec bounds)."""
    from qulacs.circuit import QuantumCircuitOptimizer
    n, B = 14, 12
    c = helpers.random_circuit(n, 120, seed=62)
    QuantumCircuitOptimizer(sv_block_size=B).optimize(c, block_size=5)
    big = [g for g in c._gates if len(g.full_qubits()) > 2]
    assert big
    ref = csim_ref.run_circuit(n, c._gates)
    from qulacs import _native
    cq = qulacs_mod.CompressedQuantumState(n, B, dtype=dtype, flags=_native.QS_FLAG_QUIET,
                                           eps_rel=2.0 ** -22 if dtype == "complex128" else 2.0 ** -20,
                                           eps_abs=1e-13)
    try:
        cq.apply_gates(c._gates, inner_size=3)
    except _native.QompsimError as e:
        # a fused gate with more qubits above the chunk than a tile holds
        assert e.status == _native.QS_ERR_UNSUPPORTED_GATE
        pytest.skip(str(e))
    assert np.abs(cq.get_vector(renormalize=False) - ref).max() < tol


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
@pytest.mark.parametrize("circ", ["qft", "random"])
def test_staged_kernel_bit_identical(qulacs_mod, monkeypatch, dtype, circ):
    """The staged pass kernel (QOMPSIM_STAGED_PASS=1: next tile's payloads
    prefetched with bulk copies) runs the same decode, sweeps and quantiser as
    the default kernel: same decoded state, masks and byte totals."""
    from qompsim import circuits as C
    n, B = 16, 9
    c = helpers.optimized(C.qft_basis(n, 5) if circ == "qft" else helpers.random_circuit(n, 120, seed=71), B)
    out = []
    for staged in ("0", "1"):
        monkeypatch.setenv("QOMPSIM_STAGED_PASS", staged)
        cq = _compressed(qulacs_mod, c, B, 3, dtype=dtype)
        out.append((cq.get_vector(renormalize=False), cq.get_zero_mask(), cq.get_SV_bytes_history()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]

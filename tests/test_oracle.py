"""The oracle itself, pinned before it is trusted (CPU only).

* the reference's csim kernels (compiled from the reference sources) against
  analytic states and against the committed golden vectors;
* the codec's C statement: error bound, monotone/continuous code, pack /
  unpack round trip, frame-of-reference widths;
* the compander emulation of the reference against its stated bound.
"""
import math

import numpy as np
import pytest

from oracle import codec as oc
from oracle import csim_ref
from oracle import pipeline, planner

import helpers

pytestmark = pytest.mark.skipif(not csim_ref.available(), reason="oracle/_ref not built")


def test_csim_ghz_analytic():
    from qompsim import circuits as C
    n = 10
    v = csim_ref.run_circuit(n, C.ghz_fanout(n)._gates)
    ref = np.zeros(1 << n, dtype=np.complex128)
    ref[0] = ref[-1] = 1 / math.sqrt(2)
    assert np.abs(v - ref).max() < 1e-15


@pytest.mark.parametrize("n,seed", [(5, 0), (7, 3), (9, 11)])
def test_csim_qft_analytic(n, seed):
    from qompsim import circuits as C
    v = csim_ref.run_circuit(n, C.qft_basis(n, seed)._gates)
    assert np.abs(v - C.qft_expected(n, C.qft_input(n, seed))).max() < 1e-13


@pytest.mark.parametrize("key", sorted(helpers.golden_circuits()))
def test_golden_vectors_reproduce(key):
    c = helpers.build_circuit(key)
    v = csim_ref.run_circuit(c.get_qubit_count(), c._gates)
    assert np.abs(v - helpers.golden_states()[key]).max() == 0.0
    assert abs(csim_ref.norm_squared(v) - 1.0) < 1e-12


def test_csim_matches_dense_matrix_product():
    from qulacs._gates import full_matrix
    n = 6
    c = helpers.random_circuit(n, 40, seed=5)
    v = csim_ref.run_circuit(n, c._gates)
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1
    for g in c._gates:
        m, qs = full_matrix(g)
        t = s.reshape([2] * n)
        axes = [n - 1 - q for q in reversed(qs)]
        k = len(qs)
        mt = m.reshape([2] * (2 * k))
        t = np.tensordot(mt, t, axes=(list(range(k, 2 * k)), axes))
        s = np.moveaxis(t, list(range(k)), axes).reshape(-1)
    assert np.abs(v - s).max() < 1e-12


# ------------------------------------------------------------- codec
@pytest.mark.parametrize("f64", [True, False])
@pytest.mark.parametrize("eps_rel,eps_abs", [(1e-3, 1e-7), (1e-2, 1e-5), (1e-5, 1e-10), (3e-4, 0.0)])
def test_codec_error_bound(f64, eps_rel, eps_abs):
    m, L = oc.params(f64, eps_rel, eps_abs)
    rng = np.random.default_rng(1)
    mags = np.concatenate([10.0 ** rng.uniform(-12, 0, 20000), rng.uniform(0, 1, 5000), [0.0, 1.0, 2 ** -20]])
    x = mags * rng.choice([-1.0, 1.0], size=mags.size)
    dt = np.float64 if f64 else np.float32
    xs = x.astype(dt)
    r = oc.roundtrip(xs, m, L).astype(np.float64)
    x64 = xs.astype(np.float64)
    bound = 0.5 * (eps_rel * np.abs(x64) + eps_abs)
    if not f64 and eps_abs == 0.0:
        bound = bound + 2.0 ** -126
    assert np.all(np.abs(r - x64) <= bound * (1 + 1e-12)), np.max(np.abs(r - x64) - bound)
    assert np.all(r[x64 == 0] == 0)
    assert np.all(np.sign(r[r != 0]) == np.sign(x64[r != 0]))


@pytest.mark.parametrize("f64", [True, False])
def test_codec_code_monotone_and_continuous(f64):
    m, L = oc.params(f64, 1e-3, 1e-7)
    dt = np.float64 if f64 else np.float32
    a = np.sort(10.0 ** np.linspace(-12, 0.3, 4001)).astype(dt)
    q = oc.quantize(a, m, L)
    assert np.all(np.diff(q) >= 0)
    e0 = m - L
    # both sides of the linear / relative seam give the same code
    assert oc.quantize(np.array([2.0 ** e0], dtype=dt), m, L)[0] == 1 << m
    assert oc.quantize(np.array([-(2.0 ** e0)], dtype=dt), m, L)[0] == -(1 << m)


@pytest.mark.parametrize("f64", [True, False])
@pytest.mark.parametrize("C", [4, 6, 8])
def test_codec_chunk_roundtrip(f64, C):
    m, L = oc.params(f64, 1e-3, 1e-7)
    rng = np.random.default_rng(C)
    dt = np.float64 if f64 else np.float32
    for trial in range(6):
        n = 2 << C
        if trial == 0:
            vals = np.zeros(n)
        elif trial == 1:
            vals = np.zeros(n)
            vals[rng.integers(0, n)] = 1.0
        else:
            vals = rng.normal(scale=10.0 ** -rng.uniform(0, 6), size=n)
        vals = vals.astype(dt)
        words, base, width = oc.encode_chunk(vals, C, m, L)
        assert words.size * 4 == oc.payload_bytes(C, width)
        dec = oc.decode_chunk(words, C, base, width, m, L, f64)
        assert np.array_equal(dec, oc.roundtrip(vals, m, L))
        q = oc.quantize(vals, m, L)
        assert base == q.min()
        assert width == int(q.max() - q.min()).bit_length()


def test_compander_emulation_bound():
    eps_rel, eps_abs = 1e-3, 1e-7
    rng = np.random.default_rng(3)
    x = 10.0 ** rng.uniform(-10, 0, 50000) * rng.choice([-1, 1], 50000)
    r = oc.ref_compander_roundtrip(x, eps_rel, eps_abs)
    # round-to-nearest in the log domain: |xhat - x| <= (eps_rel |x| + eps_abs)/2 (to first order)
    assert np.all(np.abs(r - x) <= 0.5 * (eps_rel * np.abs(x) + eps_abs) * 1.01)
    assert oc.ref_compander_roundtrip(np.array([0.0]), eps_rel, eps_abs)[0] == 0.0


# ------------------------------------------------------------- planner oracle
def test_oracle_planner_ghz20_stages():
    from qompsim import circuits as C
    c = helpers.optimized(C.ghz_fanout(20), 12)
    g = planner.describe(c._gates)
    st = planner.partition_circuit(g, 12, 4)
    assert [len(s) for s in st] == [15, 4]
    maps, counts = planner.make_block_groups(g, st, 20, 12)
    assert counts == [16, 16]
    # stage 0: outer qubits 16..19 -> group = block >> 4; stage 1: outer 12..15
    assert maps[0][:32] == [b >> 4 for b in range(32)]
    assert maps[1][:32] == [b & 15 for b in range(32)]


def test_oracle_pipeline_ghz20_masks():
    from qompsim import circuits as C
    c = helpers.optimized(C.ghz_fanout(20), 12)
    g = planner.describe(c._gates)
    st = planner.partition_circuit(g, 12, 4)
    maps, counts = planner.make_block_groups(g, st, 20, 12)
    o = pipeline.CompressedOracle(20, 12)
    o.apply(c._gates, st, maps, counts)
    assert [list(np.nonzero(m)[0]) for m in o.mask_history] == [[0], [0, 15], [0, 15, 255]]
    v = o.vector()
    assert abs(v[0] - 1 / math.sqrt(2)) < 1e-15 and abs(v[-1] - 1 / math.sqrt(2)) < 1e-15


@pytest.mark.parametrize("key", ["ghz_10", "qft_8", "hea_9", "qaoa_9", "wstate_8", "bv_9"])
def test_oracle_pipeline_matches_csim(key):
    c = helpers.optimized(helpers.build_circuit(key), 4)
    n = c.get_qubit_count()
    g = planner.describe(c._gates)
    for B, I in [(4, 1), (5, 2), (4, 4)]:
        st = planner.partition_circuit(g, B, I)
        maps, counts = planner.make_block_groups(g, st, n, B)
        o = pipeline.CompressedOracle(n, B, reference_controls=True)
        o.apply(c._gates, st, maps, counts)
        assert np.abs(o.vector() - helpers.golden_states()[key]).max() < 1e-12

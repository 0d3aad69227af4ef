"""Expectation values and adjoint gradients on the device (run with -m gpu).

* Pauli expectation sums (compressed and uncompressed) against numpy on the
  same vectors, FP64 reductions: 1e-10 (complex128), 1e-5 (complex64).
* Adjoint gradient of <psi(theta)|H|psi(theta)> against central finite
  differences (h = 1e-4) and the +-pi/2 parameter-shift rule of the
  reference's GradCalculator, complex128 to 1e-6, complex64 to 2e-3.
* torch.autograd through CircuitEnergyFunction with parameters shared
  between gates (QAOA), against the same finite differences.
"""
import numpy as np
import pytest

import helpers
from oracle import csim_ref

pytestmark = pytest.mark.gpu


def numpy_pauli_sum(v, xm, zm):
    x = np.arange(v.size, dtype=np.int64)
    sign = np.where(np.vectorize(lambda t: bin(t).count("1") & 1)(x & zm), -1.0, 1.0)
    return np.sum(np.conj(v[x ^ xm]) * sign * v)


def hea_observable(qulacs, n):
    o = qulacs.Observable(n)
    for i in range(n - 1):
        o.add_operator(1.0, f"Z {i} Z {i + 1}")
    for i in range(n):
        o.add_operator(0.5, f"X {i}")
    o.add_operator(0.25, "Y 0 Y 1")
    return o


def numpy_energy(v, obs):
    xs, zs, nys, cs = obs.term_masks()
    return float(np.real(sum(c * (1j ** ny) * numpy_pauli_sum(v, x, z) for x, z, ny, c in zip(xs, zs, nys, cs))))


@pytest.fixture(scope="module")
def qulacs_mod():
    import qulacs
    from qulacs import _native
    _native.load_library()
    return qulacs


@pytest.mark.parametrize("dtype,tol", [("complex128", 1e-10), ("complex64", 1e-5)])
def test_dense_expectation_matches_numpy(qulacs_mod, dtype, tol):
    n = 9
    c = helpers.random_circuit(n, 60, seed=21)
    s = qulacs_mod.QuantumState(n, dtype=dtype)
    c.update_quantum_state(s)
    v = s.get_vector()
    obs = hea_observable(qulacs_mod, n)
    assert abs(obs.get_expectation_value(s) - numpy_energy(v, obs)) < tol
    ref = csim_ref.run_circuit(n, c._gates)
    assert abs(obs.get_expectation_value(s) - numpy_energy(ref, obs)) < (1e-10 if dtype == "complex128" else 1e-4)


@pytest.mark.parametrize("n,B", [(10, 5), (12, 8)])
def test_compressed_expectation_matches_numpy(qulacs_mod, n, B):
    from qulacs import _native
    c = helpers.optimized(helpers.random_circuit(n, 80, seed=n), B)
    cq = qulacs_mod.CompressedQuantumState(n, B, eps_rel=1e-3, eps_abs=1e-7, flags=_native.QS_FLAG_QUIET)
    cq.partition_and_register_circuit(c, 2, 0)
    cq.apply_circuit()
    v = cq.get_vector()   # renormalised, as get_expectation_value divides by the norm
    obs = qulacs_mod.Observable(n)
    for i in range(n - 1):
        obs.add_operator(0.7, f"Z {i} Z {i + 1}")
    for i in range(n):
        obs.add_operator(0.3, f"X {i}")
    obs.add_operator(0.2, f"Y {n - 1} X 0")
    assert abs(obs.get_expectation_value(cq) - numpy_energy(v, obs)) < 1e-9
    # and close to the exact FP64 value of the uncompressed circuit
    ref = csim_ref.run_circuit(n, c._gates)
    assert abs(obs.get_expectation_value(cq) - numpy_energy(ref, obs)) < 5e-3


def _hea_param(qulacs, n, depth, seed):
    from qompsim import circuits as C
    return C.hea(n, depth, seed, parametric=True)


def _fd(circuit, obs, dtype, h=1e-4):
    from qulacs.torch import energy
    c = circuit.copy()
    g = np.zeros(c.get_parameter_count())
    for i in range(len(g)):
        t = c.get_parameter(i)
        c.set_parameter(i, t + h)
        ep = energy(c, obs, dtype)
        c.set_parameter(i, t - h)
        em = energy(c, obs, dtype)
        c.set_parameter(i, t)
        g[i] = (ep - em) / (2 * h)
    return g


@pytest.mark.parametrize("dtype,tol", [("complex128", 1e-6), ("complex64", 2e-3)])
def test_adjoint_gradient_hea(qulacs_mod, dtype, tol):
    from qulacs.torch import energy_and_gradient, parameter_shift_gradient
    n = 8
    circ = _hea_param(qulacs_mod, n, 3, seed=4)
    obs = hea_observable(qulacs_mod, n)
    e, g = energy_and_gradient(circ, obs, dtype)
    ref = csim_ref.run_circuit(n, circ._gates)
    assert abs(e - numpy_energy(ref, obs)) < (1e-10 if dtype == "complex128" else 1e-4)
    fd = _fd(circ, obs, "complex128")
    ps = parameter_shift_gradient(circ, obs, "complex128")
    assert np.max(np.abs(ps - fd)) < 1e-6
    assert np.max(np.abs(g - fd)) < tol
    assert np.max(np.abs(g - ps)) < tol


def test_adjoint_gradient_qaoa_torch(qulacs_mod):
    import torch
    from qompsim import circuits as C
    from qulacs.torch import circuit_energy
    n, p = 8, 2
    edges = C.regular_graph_edges(n, 3, seed=1)

    def builder(params):
        gam, bet = params[:p], params[p:]
        c = qulacs_mod.ParametricQuantumCircuit(n)
        for q in range(n):
            c.add_H_gate(q)
        rows = []
        for layer in range(p):
            for a, b in edges:
                c.add_parametric_multi_Pauli_rotation_gate([a, b], [3, 3], gam[layer])
                rows.append(layer)
            for q in range(n):
                c.add_parametric_RX_gate(q, bet[layer])
                rows.append(p + layer)
        jac = np.zeros((len(rows), 2 * p))
        for i, col in enumerate(rows):
            jac[i, col] = 1.0
        return c, jac

    obs = qulacs_mod.Observable(n)
    for a, b in edges:
        obs.add_operator(0.5, f"Z {a} Z {b}")
    gam, bet = C.qaoa_params(p, seed=3)
    x0 = np.concatenate([gam, bet])
    params = torch.tensor(x0, dtype=torch.float64, requires_grad=True)
    e = circuit_energy(params, builder, obs)
    e.backward()
    from qulacs.torch import energy
    h = 1e-4
    fd = np.zeros_like(x0)
    for j in range(x0.size):
        xp, xm = x0.copy(), x0.copy()
        xp[j] += h
        xm[j] -= h
        fd[j] = (energy(builder(xp)[0], obs) - energy(builder(xm)[0], obs)) / (2 * h)
    assert np.max(np.abs(params.grad.numpy() - fd)) < 1e-6
    assert abs(float(e.detach()) - energy(builder(x0)[0], obs)) < 1e-12


# ------------------------------------------------------------------ compressed adjoint
def _qaoa_param(qulacs, n, p, seed):
    from qompsim import circuits as C
    edges = C.regular_graph_edges(n, 3, seed=seed)
    gam, bet = C.qaoa_params(p, seed=seed)
    c = qulacs.ParametricQuantumCircuit(n)
    for q in range(n):
        c.add_H_gate(q)
    for layer in range(p):
        for a, b in edges:
            c.add_parametric_multi_Pauli_rotation_gate([a, b], [3, 3], gam[layer])
        for q in range(n):
            c.add_parametric_RX_gate(q, bet[layer])
    obs = qulacs.Observable(n)
    for a, b in edges:
        obs.add_operator(0.5, f"Z {a} Z {b}")
    return c, obs


def test_compressed_transition_and_diagonal_sum(qulacs_mod):
    """qs_transition_pauli and qs_apply_diagonal_pauli_sum against numpy on
    the states' own decoded vectors."""
    from qulacs import _native
    n, B = 11, 6
    c1 = helpers.optimized(helpers.random_circuit(n, 60, seed=5), B)
    c2 = helpers.optimized(helpers.random_circuit(n, 60, seed=6), B)
    kw = dict(eps_rel=2.0 ** -20, eps_abs=1e-12, flags=_native.QS_FLAG_QUIET)
    a = qulacs_mod.CompressedQuantumState(n, B, **kw)
    a.partition_and_register_circuit(c1, 2, 0)
    a.apply_circuit()
    b = qulacs_mod.CompressedQuantumState(n, B, **kw)
    b.partition_and_register_circuit(c2, 2, 0)
    b.apply_circuit()
    va, vb = a.get_vector(renormalize=False), b.get_vector(renormalize=False)
    xs = [0, 1 << 3, (1 << 9) | 1, 0, (1 << 10) | (1 << 7)]
    zs = [0, 0, 1 << 2, (1 << 8) | (1 << 1), 1 << 10]
    got = a.transition_pauli_sums(b, xs, zs)   # <b| P |a>
    x = np.arange(1 << n)
    for t, (xm, zm) in enumerate(zip(xs, zs)):
        sign = np.where(np.vectorize(lambda v: bin(v).count("1") & 1)(x & zm), -1.0, 1.0)
        want = np.sum(np.conj(vb[x ^ xm]) * sign * va)
        assert abs(got[t] - want) < 1e-10, t
    # lambda = (0.5 Z1 Z4 - 1.2 Z10 + 0.3) psi
    zsd = [(1 << 1) | (1 << 4), 1 << 10, 0]
    cd = [0.5, -1.2, 0.3]
    lam = qulacs_mod.CompressedQuantumState(n, B, **kw)
    lam.load_diagonal_pauli_sum(a, zsd, cd)
    h = np.zeros(1 << n)
    for zm, cf in zip(zsd, cd):
        h += cf * np.where(np.vectorize(lambda v: bin(v).count("1") & 1)(x & zm), -1.0, 1.0)
    assert np.abs(lam.get_vector(renormalize=False) - h * va).max() < 1e-5
    assert np.array_equal(lam.get_zero_mask(), a.get_zero_mask())


@pytest.mark.parametrize("dtype,checkpoints", [("complex128", False), ("complex128", True), ("complex64", True)])
def test_compressed_adjoint_qaoa(qulacs_mod, dtype, checkpoints):
    """Compressed adjoint gradient of QAOA (layer groups, diagonal H) against
    the dense adjoint and FP64 central differences."""
    from qulacs.torch import compressed_energy_and_gradient, energy_and_gradient
    n, p = 10, 2
    circ, obs = _qaoa_param(qulacs_mod, n, p, seed=2)
    tight = dtype == "complex128"
    e, g = compressed_energy_and_gradient(circ, obs, block_size=5, inner_size=2, dtype=dtype,
                                          eps_rel=2.0 ** -20 if tight else 2.0 ** -16,
                                          eps_abs=1e-12 if tight else 1e-8, checkpoints=checkpoints)
    e_ref, g_ref = energy_and_gradient(circ, obs, "complex128")
    tol = 1e-5 if tight else 2e-3
    assert abs(e - e_ref) < tol
    assert np.max(np.abs(g - g_ref)) < tol
    fd = _fd(circ, obs, "complex128")
    assert np.max(np.abs(g - fd)) < tol + 1e-6


def test_compressed_adjoint_default_bounds(qulacs_mod):
    """At the reference's default error bounds (1e-3 / 1e-7) the compressed
    adjoint stays close to the exact gradient."""
    from qulacs.torch import compressed_energy_and_gradient, energy_and_gradient
    circ, obs = _qaoa_param(qulacs_mod, 12, 2, seed=3)
    e, g = compressed_energy_and_gradient(circ, obs, block_size=6, inner_size=3, dtype="complex64", checkpoints=True)
    e_ref, g_ref = energy_and_gradient(circ, obs, "complex128")
    scale = max(1.0, np.max(np.abs(g_ref)))
    assert abs(e - e_ref) < 2e-2
    assert np.max(np.abs(g - g_ref)) / scale < 5e-2


def test_compressed_circuit_function_torch(qulacs_mod):
    """torch.autograd through the compressed adjoint, QAOA with parameters
    shared across each layer (jacobian mapping), against FP64 differences."""
    import torch
    from qompsim import circuits as C
    from qulacs.torch import compressed_circuit_energy, energy
    n, p = 10, 2
    edges = C.regular_graph_edges(n, 3, seed=4)

    def builder(params):
        gam, bet = params[:p], params[p:]
        c = qulacs_mod.ParametricQuantumCircuit(n)
        for q in range(n):
            c.add_H_gate(q)
        rows = []
        for layer in range(p):
            for a, b in edges:
                c.add_parametric_multi_Pauli_rotation_gate([a, b], [3, 3], gam[layer])
                rows.append(layer)
            for q in range(n):
                c.add_parametric_RX_gate(q, bet[layer])
                rows.append(p + layer)
        jac = np.zeros((len(rows), 2 * p))
        for i, col in enumerate(rows):
            jac[i, col] = 1.0
        return c, jac

    obs = qulacs_mod.Observable(n)
    for a, b in edges:
        obs.add_operator(0.5, f"Z {a} Z {b}")
    x0 = np.concatenate(C.qaoa_params(p, seed=5))
    params = torch.tensor(x0, dtype=torch.float64, requires_grad=True)
    e = compressed_circuit_energy(params, builder, obs, block_size=5, inner_size=2, eps_rel=2.0 ** -20,
                                  eps_abs=1e-12, checkpoints=True)
    e.backward()
    h = 1e-4
    fd = np.zeros_like(x0)
    for j in range(x0.size):
        xp, xm = x0.copy(), x0.copy()
        xp[j] += h
        xm[j] -= h
        fd[j] = (energy(builder(xp)[0], obs) - energy(builder(xm)[0], obs)) / (2 * h)
    assert np.max(np.abs(params.grad.numpy() - fd)) < 1e-5
    assert abs(float(e.detach()) - energy(builder(x0)[0], obs)) < 1e-5


# ------------------------------------------------------------ general compressed adjoint
def _pauli_apply_numpy(v, xm, zm):
    """(P v)[x] = (-1)^{|y & z|} v[y], y = x ^ xm (i^ny left to the coefficient)."""
    x = np.arange(v.size, dtype=np.int64)
    y = x ^ xm
    sign = np.where(np.vectorize(lambda t: bin(t).count("1") & 1)(y & zm), -1.0, 1.0)
    return sign * v[y]


@pytest.mark.parametrize("dtype,tol", [("complex128", 2.0 ** -21), ("complex64", 2.0 ** -18)])
def test_compressed_pauli_sum_matches_numpy(qulacs_mod, dtype, tol):
    """lambda = H psi on compressed stores (qs_apply_pauli_sum) with X, Y and
    Z strings, several of them flipping qubits above the chunk, against numpy
    on the decoded input, to the output store's own quantisation (relative
    steps 2^-22 / 2^-20, so tol = 2 steps of the largest amplitude)."""
    from qulacs import _native
    n, B = 12, 8
    c = helpers.optimized(helpers.random_circuit(n, 60, seed=41), B)
    kw = dict(dtype=dtype, eps_rel=2.0 ** -22 if dtype == "complex128" else 2.0 ** -20, eps_abs=1e-13,
              flags=_native.QS_FLAG_QUIET)
    psi = qulacs_mod.CompressedQuantumState(n, B, **kw)
    psi.partition_and_register_circuit(c, 3, 0)
    psi.apply_circuit()
    obs = hea_observable(qulacs_mod, n)
    obs.add_operator(0.3, "X 9 Y 11 Z 2")
    obs.add_operator(-0.7, "Y 10")
    xs, zs, nys, coefs = obs.term_masks()
    lam = qulacs_mod.CompressedQuantumState(n, B, **kw)
    lam.load_pauli_sum(psi, xs, zs, [cf * (1j ** ny) for cf, ny in zip(coefs, nys)])
    v = psi.get_vector(renormalize=False)
    ref = sum(cf * (1j ** ny) * _pauli_apply_numpy(v, x, z) for x, z, ny, cf in zip(xs, zs, nys, coefs))
    got = lam.get_vector(renormalize=False)
    assert np.abs(got - ref).max() < tol * max(1.0, np.abs(ref).max())
    assert lam.get_zero_mask().all()


@pytest.mark.parametrize("dtype,ckpt", [("complex128", None), ("complex128", 4), ("complex64", None),
                                        ("complex64", 6)])
def test_compressed_adjoint_hea(qulacs_mod, dtype, ckpt):
    """Adjoint gradient with both states compressed (qs_apply_pauli_sum +
    qs_adjoint) on a hardware-efficient ansatz (RY RZ layers + CNOT ladder)
    with H = sum Z_i Z_i+1 + 0.5 sum X_i + 0.25 Y0 Y1, with and without
    device checkpoints: complex128 at tight bounds matches the uncompressed
    FP64 adjoint to 1e-6; complex64 at the reference's default bounds is
    within 3e-3 of FP64 central differences (h = 1e-4)."""
    from qulacs.torch import compressed_adjoint_gradient, energy_and_gradient
    n, B = 10, 6
    circ = _hea_param(qulacs_mod, n, 3, seed=7)
    obs = hea_observable(qulacs_mod, n)
    e_ref, g_ref = energy_and_gradient(circ, obs, "complex128")
    if dtype == "complex128":
        e, g = compressed_adjoint_gradient(circ, obs, B, 3, dtype, eps_rel=2.0 ** -22, eps_abs=1e-13,
                                           checkpoint_every=ckpt)
        assert abs(e - e_ref) < 1e-6
        assert np.max(np.abs(g - g_ref)) < 1e-6
    else:
        e, g = compressed_adjoint_gradient(circ, obs, B, 3, dtype, checkpoint_every=ckpt)
        fd = _fd(circ, obs, "complex128")
        assert abs(e - e_ref) < 3e-3
        assert np.max(np.abs(g - fd)) < 3e-3


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
def test_compressed_adjoint_register_sweeps_match_op_path(qulacs_mod, dtype, monkeypatch):
    """The backward passes as register sweeps over both stores (the default:
    derivative sums inside the sweeps) against one shared-memory sweep per
    gate and per sum (QOMPSIM_DUAL_SWEEPS=0), on a circuit whose generators
    flip one or two qubits (RX, RY, XX, YZ rotations), are diagonal (RZ, ZZ)
    or have Z factors on qubits outside the register bits, and an observable
    with X, Y and Z strings; and both against the FP64 adjoint."""
    from qulacs.torch import compressed_adjoint_gradient, energy_and_gradient
    n, B = 11, 7
    rng = np.random.default_rng(12)
    c = qulacs_mod.ParametricQuantumCircuit(n)
    for q in range(n):
        c.add_H_gate(q)
    for layer in range(2):
        for q in range(n):
            c.add_parametric_RY_gate(q, rng.uniform(0, 2 * np.pi))
            c.add_parametric_RX_gate(q, rng.uniform(0, 2 * np.pi))
        for q in range(0, n - 1, 2):
            c.add_parametric_multi_Pauli_rotation_gate([q, q + 1], [3, 3], rng.uniform(0, 2 * np.pi))
        for q in range(1, n - 1, 2):
            c.add_parametric_multi_Pauli_rotation_gate([q, q + 1], [1, 1], rng.uniform(0, 2 * np.pi))
        for q in range(0, n - 3, 3):
            c.add_parametric_multi_Pauli_rotation_gate([q, q + 3], [2, 3], rng.uniform(0, 2 * np.pi))
            c.add_CNOT_gate(q, q + 2)
        for q in range(n):
            c.add_parametric_RZ_gate(q, rng.uniform(0, 2 * np.pi))
    obs = hea_observable(qulacs_mod, n)
    obs.add_operator(0.3, "X 2 Z 9")
    obs.add_operator(-0.2, "Y 8 Y 10")
    e_ref, g_ref = energy_and_gradient(c, obs, "complex128")
    tight = dtype == "complex128"
    kw = dict(eps_rel=2.0 ** -22, eps_abs=1e-13) if tight else dict(eps_rel=2.0 ** -14, eps_abs=1e-9)
    monkeypatch.setenv("QOMPSIM_DUAL_SWEEPS", "1")
    e1, g1 = compressed_adjoint_gradient(c, obs, B, 3, dtype, checkpoint_every=8, **kw)
    monkeypatch.setenv("QOMPSIM_DUAL_SWEEPS", "0")
    e0, g0 = compressed_adjoint_gradient(c, obs, B, 3, dtype, checkpoint_every=8, **kw)
    tol = 1e-6 if tight else 2e-3
    assert abs(e1 - e0) < 1e-12   # the forward pass is the same; reductions may add in another order
    assert np.max(np.abs(g1 - g0)) < tol
    assert np.max(np.abs(g1 - g_ref)) < tol

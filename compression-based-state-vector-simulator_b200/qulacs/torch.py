"""qulacs.torch -- energies and adjoint gradients of parametric circuits, and
a torch.autograd.Function over them.

energy_and_gradient(circuit, observable) runs the circuit on a device state,
evaluates <psi|H|psi> (FP64 reductions), builds lam = H psi and walks the
circuit backwards with the fused dual-state adjoint pass (qs_dense_adjoint):
for a rotation U_k = exp(i theta_k/2 P_k),
    dE/dtheta_k = 2 Re <lam_k| (i/2) P_k |psi_k> = -Im <lam_k|P_k|psi_k>,
with lam_k = (U_N ... U_{k+1})^dagger H psi_N and psi_k the state after U_k.
This is the reference's state/bistate backprop
(src/vqcsim/parametric_circuit.cpp:180-306) on the GPU; the reference has no
gradient on its compressed state.  Each pass of the backward sweep reads and
writes both states once.

parameter_shift_gradient gives the +-pi/2 shift rule of the reference's
GradCalculator (src/vqcsim/GradCalculator.cpp:8-44) on the same device path,
as an independent check.
"""
from __future__ import annotations

import ctypes as ct
from typing import Callable, Optional, Sequence

import numpy as np

from . import _native as _n
from . import QuantumState, Observable


def _masks_arrays(xs, zs):
    xa = np.ascontiguousarray(np.asarray(xs, dtype=np.uint64))
    za = np.ascontiguousarray(np.asarray(zs, dtype=np.uint64))
    return xa, za


def apply_observable(out: QuantumState, state: QuantumState, observable: Observable) -> None:
    """out := H state (Observable.apply_to_state of the reference)."""
    xs, zs, nys, coefs = observable.term_masks()
    c = np.array([complex(cf) * (1j ** ny) for cf, ny in zip(coefs, nys)], dtype=np.complex128)
    xa, za = _masks_arrays(xs, zs)
    L = _n.lib()
    out._check(L.qs_dense_apply_pauli_sum(out._h, state._h, xa.ctypes.data_as(ct.POINTER(ct.c_uint64)),
                                          za.ctypes.data_as(ct.POINTER(ct.c_uint64)),
                                          c.view(np.float64).ctypes.data_as(ct.POINTER(ct.c_double)), len(xs)))


def energy_and_gradient(circuit, observable: Observable, dtype="complex128"):
    """(E, dE/dtheta) for every parametric gate of `circuit`, in the order of
    circuit parameters (get_parameter(i))."""
    n = circuit.get_qubit_count()
    psi = QuantumState(n, dtype=dtype)
    circuit.update_quantum_state(psi)
    energy = observable.get_expectation_value(psi)
    lam = QuantumState(n, dtype=dtype)
    apply_observable(lam, psi, observable)

    gates = circuit._gates
    param_pos = list(getattr(circuit, "_param_pos", []))
    slot_of = {pos: i for i, pos in enumerate(param_pos)}
    back, slots, gx, gz, gny = [], [], [], [], []
    for k in reversed(range(len(gates))):
        g = gates[k]
        back.append(g.get_inverse())
        if k in slot_of:
            xm, zm, ny = g.generator_masks()
            slots.append(slot_of[k])
            gx.append(xm)
            gz.append(zm)
            gny.append(ny)
        else:
            slots.append(-1)
            gx.append(0)
            gz.append(0)
            gny.append(0)
    nslots = len(param_pos)
    arr = _n.make_gate_array(back)
    sl = np.ascontiguousarray(np.asarray(slots, dtype=np.int32))
    xa, za = _masks_arrays(gx, gz)
    out = np.zeros(2 * max(1, nslots), dtype=np.float64)
    L = _n.lib()
    psi._check(L.qs_dense_adjoint(psi._h, lam._h, arr, sl.ctypes.data_as(ct.POINTER(ct.c_int32)),
                                  xa.ctypes.data_as(ct.POINTER(ct.c_uint64)),
                                  za.ctypes.data_as(ct.POINTER(ct.c_uint64)), len(back),
                                  out.ctypes.data_as(ct.POINTER(ct.c_double)), nslots))
    sums = out[0:2 * nslots:2] + 1j * out[1:2 * nslots:2]
    ny_of_slot = np.zeros(nslots, dtype=np.int64)
    for s_, ny in zip(slots, gny):
        if s_ >= 0:
            ny_of_slot[s_] = ny
    grads = -np.imag((1j ** ny_of_slot) * sums)
    return float(energy), grads


def _support(g):
    return set(g.get_target_index_list()) | set(g.get_control_index_list())


def _is_diagonal(g) -> bool:
    m = np.asarray(g.get_matrix())
    return not np.any(m - np.diag(np.diag(m)))


def _commute(a, b) -> bool:
    """Sufficient test: disjoint qubits, or both diagonal."""
    return not (_support(a) & _support(b)) or (_is_diagonal(a) and _is_diagonal(b))


def commuting_groups(circuit):
    """Maximal runs of consecutive parametric gates that commute pairwise, as
    (start, end) gate-index ranges, last group first."""
    gates = circuit._gates
    pset = set(getattr(circuit, "_param_pos", []))
    out = []
    i = len(gates) - 1
    while i >= 0:
        if i in pset:
            grp = [i]
            j = i - 1
            while j >= 0 and j in pset and all(_commute(gates[j], gates[m]) for m in grp):
                grp.append(j)
                j -= 1
            out.append((j + 1, i + 1))
            i = j
        else:
            i -= 1
    return out


def compressed_energy_and_gradient(circuit, observable: Observable, block_size: int, inner_size: int = 4,
                                   dtype="complex128", eps_rel: float = 1e-3, eps_abs: float = 1e-7,
                                   checkpoints: bool = False, flags: Optional[int] = None,
                                   timings: Optional[dict] = None):
    """(E, dE/dtheta) with both states compressed, for a diagonal observable
    (Z strings only) and circuits whose parametric gates come in groups that
    commute (QAOA cost and mixer layers, layers of single-qubit rotations).

    Forward: psi = U |0> on a CompressedQuantumState.  lambda = H psi by one
    fused diagonal pass.  Backward, group by group from the end: at the group
    boundary every gate k of the group has dE/dtheta_k = -Im <lambda|P_k|psi>
    / <psi|psi> (the group's other gates commute with P_k, so the boundary
    states serve all of them), evaluated by one transition-sum pass over the
    two compressed stores; then the inverse gates back to the previous group
    are applied to psi and lambda as compressed circuits.  With checkpoints,
    psi is stored in device checkpoints at every group boundary during the
    forward pass and restored in the backward pass instead of being
    uncomputed, so its compression error does not accumulate twice.

    timings, when given, receives the wall time (s) of each phase: forward,
    lambda, undo (inverse gates on both states), transition (gradient sums)."""
    import time as _time
    import qulacs
    from . import CompressedQuantumState
    n = circuit.get_qubit_count()
    xs, zs, nys, coefs = observable.term_masks()
    if any(xs):
        raise ValueError("the compressed adjoint needs a diagonal observable (Z strings only)")
    gates = list(circuit._gates)
    param_pos = list(getattr(circuit, "_param_pos", []))
    slot_of = {pos: i for i, pos in enumerate(param_pos)}
    groups = commuting_groups(circuit)
    if flags is None:
        flags = _n.QS_FLAG_QUIET

    def state():
        return CompressedQuantumState(n, block_size, dtype=dtype, eps_rel=eps_rel, eps_abs=eps_abs, flags=flags)

    tm = timings if timings is not None else {}
    for k in ("forward", "lambda", "undo", "transition"):
        tm.setdefault(k, 0.0)

    def run(st, gate_list):
        if not gate_list:
            return
        c = qulacs.QuantumCircuit(n)
        for g in gate_list:
            c.add_gate(g)
        st.partition_and_register_circuit(c, inner_size, 0)
        st.apply_circuit()

    clock = [_time.perf_counter()]

    def lap(key):
        now = _time.perf_counter()
        tm[key] += now - clock[0]
        clock[0] = now

    psi = state()
    if checkpoints:
        bounds = sorted(e for _, e in groups)
        pos = 0
        for k, e in enumerate(bounds):
            run(psi, gates[pos:e])
            psi.checkpoint(k)
            pos = e
        run(psi, gates[pos:])
        slot_at = {e: k for k, e in enumerate(bounds)}
    else:
        run(psi, gates)
    sums = psi._pauli_sums(list(xs) + [0], list(zs) + [0])
    norm2 = sums[-1].real
    energy_value = float(np.real(sum(c * (1j ** ny) * v for c, ny, v in zip(coefs, nys, sums[:-1])) / norm2))
    lap("forward")
    lam = state()
    lam.load_diagonal_pauli_sum(psi, zs, [c * (1j ** ny) for c, ny in zip(coefs, nys)])
    lap("lambda")
    grads = np.zeros(len(param_pos))
    pos = len(gates)
    for start, end in groups:
        back = [g.get_inverse() for g in reversed(gates[end:pos])]
        run(lam, back)
        if checkpoints:
            psi.restore(slot_at[end])
        else:
            run(psi, back)
        lap("undo")
        idx = list(range(start, end))
        masks = [gates[i].generator_masks() for i in idx]
        # <lambda| P |psi>: bra lambda, ket psi
        s = psi.transition_pauli_sums(lam, [m[0] for m in masks], [m[1] for m in masks])
        for i, (xm, zm, ny), v in zip(idx, masks, s):
            grads[slot_of[i]] = -np.imag((1j ** ny) * v) / norm2
        lap("transition")
        pos = end
    if checkpoints:
        for k in range(len(groups)):
            psi.free_checkpoint(k)
    return energy_value, grads


def _backward_lists(gates, start, end, slot_of):
    """Inverse gates of gates[start:end] in reverse order, with the slot and
    generator masks of each parametric one (slot -1 for the others)."""
    back, slots, gx, gz, gny = [], [], [], [], []
    for k in reversed(range(start, end)):
        g = gates[k]
        back.append(g.get_inverse())
        if k in slot_of:
            xm, zm, ny = g.generator_masks()
            slots.append(slot_of[k])
            gx.append(xm)
            gz.append(zm)
            gny.append(ny)
        else:
            slots.append(-1)
            gx.append(0)
            gz.append(0)
            gny.append(0)
    return back, slots, gx, gz, gny


def compressed_adjoint_gradient(circuit, observable: Observable, block_size: int, inner_size: int = 4,
                                dtype="complex128", eps_rel: float = 1e-3, eps_abs: float = 1e-7,
                                checkpoint_every: Optional[int] = None, flags: Optional[int] = None,
                                timings: Optional[dict] = None):
    """(E, dE/dtheta) of any parametric circuit and observable (X, Y, Z
    strings) with both states compressed.

    Forward: psi = U|0> on a CompressedQuantumState (the registered circuit's
    stages and passes), with a device checkpoint of the compressed store after
    every `checkpoint_every` parametric gates when given.  E = <psi|H|psi> /
    <psi|psi> (FP64 reductions); lambda = H psi (qs_apply_pauli_sum).
    Backward, segment by segment from the end: psi is restored from the
    checkpoint at the segment's end (so its compression error does not build
    up over the whole circuit: between checkpoints it is recomputed backwards
    by the inverse gates), then one fused sweep over both compressed stores
    (qs_adjoint) applies the segment's inverse gates to psi and lambda and, at
    each parametric gate k, accumulates <lambda_k|P_k|psi_k>:
    dE/dtheta_k = -Im(i^{ny} <lambda_k|P_k|psi_k>) / <psi|psi>.  This is the
    reference's backprop (src/vqcsim/parametric_circuit.cpp:180-306) on
    compressed states.

    timings, when given, receives device milliseconds (CUDA events on the
    states' stream) of: forward (apply + energy), lambda, backward, each
    window including the host planning between launches; and the same three
    as the engine's own launch spans alone (forward_launches_ms: the applies'
    device time; lambda_launches_ms / backward_launches_ms: the two-store
    calls' device time)."""
    import qulacs
    from . import CompressedQuantumState
    n = circuit.get_qubit_count()
    xs, zs, nys, coefs = observable.term_masks()
    gates = list(circuit._gates)
    param_pos = list(getattr(circuit, "_param_pos", []))
    slot_of = {pos: i for i, pos in enumerate(param_pos)}
    if flags is None:
        flags = _n.QS_FLAG_QUIET
    # segment ends: after every `checkpoint_every` parametric gates
    bounds = []
    if checkpoint_every:
        for k, pos in enumerate(param_pos):
            if (k + 1) % checkpoint_every == 0 and pos + 1 < len(gates):
                bounds.append(pos + 1)
    bounds = sorted(set(bounds))

    ev = None
    try:
        import torch as _t
        if _t.cuda.is_available():
            ev = [_t.cuda.Event(enable_timing=True) for _ in range(4)]
    except ImportError:
        pass

    def rec(i):
        if ev is not None:
            ev[i].record()

    dev = {"forward": 0.0, "lambda": 0.0, "backward": 0.0}

    def run(st, gate_list):
        if not gate_list:
            return
        c = qulacs.QuantumCircuit(n)
        c._gates = list(gate_list)
        st.partition_and_register_circuit(c, inner_size, 0)
        st.apply_circuit()
        dev["forward"] += st.get_stats()["apply_ms"]

    psi = CompressedQuantumState(n, block_size, dtype=dtype, eps_rel=eps_rel, eps_abs=eps_abs, flags=flags)
    rec(0)
    pos = 0
    for k, e in enumerate(bounds):
        run(psi, gates[pos:e])
        psi.checkpoint(k)
        pos = e
    run(psi, gates[pos:])
    sums = psi._pauli_sums(list(xs) + [0], list(zs) + [0])
    norm2 = sums[-1].real
    energy_value = float(np.real(sum(c * (1j ** ny) * v for c, ny, v in zip(coefs, nys, sums[:-1])) / norm2))
    rec(1)
    lam = CompressedQuantumState(n, block_size, dtype=dtype, eps_rel=eps_rel, eps_abs=eps_abs, flags=flags)
    lam.load_pauli_sum(psi, xs, zs, [c * (1j ** ny) for c, ny in zip(coefs, nys)])
    dev["lambda"] = lam.get_stats()["pair_ms"]
    rec(2)
    nslots = len(param_pos)
    acc = np.zeros(2 * max(1, nslots), dtype=np.float64)
    ny_of_slot = np.zeros(max(1, nslots), dtype=np.int64)
    ends = [len(gates)] + list(reversed(bounds))
    starts = list(reversed(bounds)) + [0]
    L = _n.lib()
    for k, (start, end) in enumerate(zip(starts, ends)):
        if k > 0:
            psi.restore(len(bounds) - k)   # the forward state at this segment's end
        back, slots, gx, gz, gny = _backward_lists(gates, start, end, slot_of)
        if not back:
            continue
        for s_, ny in zip(slots, gny):
            if s_ >= 0:
                ny_of_slot[s_] = ny
        arr = _n.make_gate_array(back)
        sl = np.ascontiguousarray(np.asarray(slots, dtype=np.int32))
        xa, za = _masks_arrays(gx, gz)
        out = np.zeros(2 * max(1, nslots), dtype=np.float64)
        psi._check(L.qs_adjoint(psi._h, lam._h, arr, sl.ctypes.data_as(ct.POINTER(ct.c_int32)),
                                xa.ctypes.data_as(ct.POINTER(ct.c_uint64)),
                                za.ctypes.data_as(ct.POINTER(ct.c_uint64)), len(back),
                                out.ctypes.data_as(ct.POINTER(ct.c_double)), nslots))
        dev["backward"] += psi.get_stats()["pair_ms"]
        acc += out
    rec(3)
    for k in range(len(bounds)):
        psi.free_checkpoint(k)
    sums_g = acc[0:2 * nslots:2] + 1j * acc[1:2 * nslots:2]
    grads = -np.imag((1j ** ny_of_slot[:nslots]) * sums_g) / norm2
    if timings is not None and ev is not None:
        import torch as _t
        _t.cuda.synchronize()
        timings["forward_ms"] = ev[0].elapsed_time(ev[1])
        timings["lambda_ms"] = ev[1].elapsed_time(ev[2])
        timings["backward_ms"] = ev[2].elapsed_time(ev[3])
    if timings is not None:
        # device time of the engine's launches alone (no host planning gaps)
        timings["forward_launches_ms"] = dev["forward"]
        timings["lambda_launches_ms"] = dev["lambda"]
        timings["backward_launches_ms"] = dev["backward"]
    return energy_value, grads


def energy(circuit, observable: Observable, dtype="complex128") -> float:
    psi = QuantumState(circuit.get_qubit_count(), dtype=dtype)
    circuit.update_quantum_state(psi)
    return observable.get_expectation_value(psi)


def parameter_shift_gradient(circuit, observable: Observable, dtype="complex128") -> np.ndarray:
    """+-pi/2 shift rule per circuit parameter (GradCalculator.cpp:8-44)."""
    c = circuit.copy()
    out = np.zeros(c.get_parameter_count())
    for i in range(c.get_parameter_count()):
        t = c.get_parameter(i)
        c.set_parameter(i, t + np.pi / 2)
        ep = energy(c, observable, dtype)
        c.set_parameter(i, t - np.pi / 2)
        em = energy(c, observable, dtype)
        c.set_parameter(i, t)
        out[i] = 0.5 * (ep - em)
    return out


try:
    import torch as _torch

    class CircuitEnergyFunction(_torch.autograd.Function):
        """E(params) = <psi(params)|H|psi(params)> with the adjoint gradient.

        builder(params: np.ndarray) -> (ParametricQuantumCircuit, jac) where
        jac[i, j] = d(circuit parameter i)/d(params j), or just the circuit
        when its parameters are `params` themselves."""

        @staticmethod
        def forward(ctx, params, builder: Callable, observable: Observable, dtype: str = "complex128"):
            p = params.detach().cpu().numpy().astype(np.float64)
            built = builder(p)
            circuit, jac = (built if isinstance(built, tuple) else (built, None))
            e, g = energy_and_gradient(circuit, observable, dtype)
            if jac is not None:
                g = np.asarray(jac, dtype=np.float64).T @ g
            ctx.save_for_backward(_torch.as_tensor(g, dtype=_torch.float64))
            return _torch.tensor(e, dtype=_torch.float64)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g.to(grad_out.device), None, None, None

    def circuit_energy(params, builder, observable, dtype="complex128"):
        return CircuitEnergyFunction.apply(params, builder, observable, dtype)

    class CompressedCircuitFunction(_torch.autograd.Function):
        """E(params) on the compressed state, with the compressed adjoint
        gradient (compressed_energy_and_gradient; diagonal observables, commuting
        parametric layers).  builder as for CircuitEnergyFunction; options are
        the keyword arguments of compressed_energy_and_gradient (block_size,
        inner_size, dtype, eps_rel, eps_abs, checkpoints)."""

        @staticmethod
        def forward(ctx, params, builder: Callable, observable: Observable, options: dict):
            p = params.detach().cpu().numpy().astype(np.float64)
            built = builder(p)
            circuit, jac = (built if isinstance(built, tuple) else (built, None))
            e, g = compressed_energy_and_gradient(circuit, observable, **options)
            if jac is not None:
                g = np.asarray(jac, dtype=np.float64).T @ g
            ctx.save_for_backward(_torch.as_tensor(g, dtype=_torch.float64))
            return _torch.tensor(e, dtype=_torch.float64)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g.to(grad_out.device), None, None, None

    def compressed_circuit_energy(params, builder, observable, **options):
        return CompressedCircuitFunction.apply(params, builder, observable, options)
except ImportError:  # torch is optional for the rest of the package
    pass

"""Per-configuration evaluation of the compressed pipeline on one GPU.

    python -m qompsim.evaluate [--only ghz20 qft30 brickwork32 hea24 qaoa34 host_store28] [--quick]

For each configuration of the benchmark suite (seeded synthetic circuits) it
prints one JSON line with the stage list, the compressed size, the apply time
and amplitude-gate updates/s, and the fidelity |<psi_FP64|psi>| of the
renormalised compressed state against an FP64 uncompressed oracle (the
analytic state where one exists, else this package's complex128 QuantumState,
whose amplitudes the GPU tests hold to 1e-12 of the reference's csim
kernels), with the largest amplitude error.  Fidelities are computed in
slices of 2^24 amplitudes, so no full vector is ever held in host memory.
The hardware-efficient-ansatz line times the adjoint gradient against the
forward pass and compares it with FP64 central differences; the QAOA line
runs the compressed adjoint (qulacs.torch.compressed_energy_and_gradient).
--quick shrinks every configuration to n <= 26.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

SLICE = 1 << 24


def _sync():
    try:
        import torch
        if torch.cuda.is_available():
            torch.cuda.synchronize()
    except ImportError:
        pass


def _optimized(circuit, block_size):
    from qulacs.circuit import QuantumCircuitOptimizer
    QuantumCircuitOptimizer(sv_block_size=block_size).optimize(circuit, block_size=2)
    return circuit


def _compressed_run(circuit, n, B, I, dtype, eps_rel=1e-3, eps_abs=1e-7, reps=2, host_store=False):
    import qulacs
    from qulacs import _native
    cq = qulacs.CompressedQuantumState(n, B, dtype=dtype, eps_rel=eps_rel, eps_abs=eps_abs,
                                       flags=_native.QS_FLAG_QUIET | _native.QS_FLAG_PROFILE,
                                       host_store=host_store)
    cq.partition_and_register_circuit(circuit, I, 0)
    times = []
    for _ in range(reps):
        cq.set_computational_basis(0)
        _sync()
        t0 = time.perf_counter()
        cq.apply_circuit()
        _sync()
        times.append(time.perf_counter() - t0)
    st = cq.get_stats()
    info = {"dtype": dtype, "stages": len(cq.get_stage_list()), "passes": int(st["passes"]),
            "apply_ms": round(min(times) * 1e3, 3), "kernel_ms": round(st["kernel_ms"], 3),
            "amp_gate_updates_per_s": st["amp_gate_updates"] / min(times),
            "max_sv_bytes": cq.get_max_SV_bytes(), "dense_bytes": (16 if dtype == "complex128" else 8) << n}
    return cq, info


def _fidelity(cq, n, oracle_slice):
    """|<oracle|psi>| and max |oracle - psi| over slices (psi renormalised)."""
    acc = 0j
    err = 0.0
    for s in range(0, 1 << n, SLICE):
        cnt = min(SLICE, (1 << n) - s)
        a = oracle_slice(s, cnt)
        b = cq.get_amplitudes(s, cnt, renormalize=True)
        acc += np.vdot(a, b)
        err = max(err, float(np.max(np.abs(a - b))))
    return abs(acc), err


def eval_ghz(quick):
    from qompsim import circuits as C
    n, B, I = 20, 12, 4
    c = _optimized(C.ghz_fanout(n), B)
    cq, info = _compressed_run(c, n, B, I, "complex128")
    amp = 1 / math.sqrt(2)

    def oracle(s, cnt):
        v = np.zeros(cnt, dtype=np.complex128)
        if s == 0:
            v[0] = amp
        if s + cnt == 1 << n:
            v[-1] = amp
        return v
    f, e = _fidelity(cq, n, oracle)
    info.update(stage_sizes=[len(x) for x in cq.get_stage_list()],
                stored_blocks=[int(b) for b in np.nonzero(cq.get_zero_mask())[0]], fidelity=f, max_abs_err=e)
    return {"config": "ghz20: n=20 B=12 I=4 fan-out GHZ", **info}


def eval_qft(quick):
    from qompsim import circuits as C
    n = 26 if quick else 30
    B, I = 20, 4
    x = C.qft_input(n, 0)
    out = []
    for dtype in ("complex128", "complex64"):
        c = _optimized(C.qft_basis(n, 0), B)
        cq, info = _compressed_run(c, n, B, I, dtype)

        def oracle(s, cnt):
            k = np.arange(s, s + cnt, dtype=np.int64)
            return np.exp(2j * np.pi * ((x * k) % (1 << n)) / (1 << n)) / math.sqrt(1 << n)
        f, e = _fidelity(cq, n, oracle)
        info.update(fidelity=f, max_abs_err=e)
        # block-wise sampling on the device: |a|^2 = 2^-n, so the per-block
        # counts of 10^6 shots are multinomial with equal cells
        shots = 1_000_000
        t0 = time.perf_counter()
        smp = np.asarray(cq.sampling_blockwise(shots, 7), dtype=np.int64)
        ms = (time.perf_counter() - t0) * 1e3
        cnt = np.bincount(smp >> B, minlength=1 << (n - B))
        e_blk = shots / cnt.size
        info.update(sampling_ms_1e6_shots=ms,
                    sampling_block_chi2_per_dof=float(((cnt - e_blk) ** 2 / e_blk).sum() / (cnt.size - 1)))
        out.append({"config": f"qft{n}: n={n} B={B} I={I} QFT of basis state {x}", **info})
        del cq
    return out


def eval_brickwork(quick):
    import qulacs
    from qompsim import circuits as C
    n = 26 if quick else 32
    B, I = n - 10, 4
    out = []
    ref = qulacs.QuantumState(n, dtype="complex128")
    C.brickwork(n, 20, seed=0).update_quantum_state(ref)
    for dtype in ("complex64", "complex128"):
        c = _optimized(C.brickwork(n, 20, seed=0), B)
        cq, info = _compressed_run(c, n, B, I, dtype, reps=1)
        f, e = _fidelity(cq, n, ref.get_amplitudes)
        info.update(fidelity=f, max_abs_err=e)
        out.append({"config": f"brickwork{n}: n={n} 20 layers B={B} I={I}", **info})
        del cq
    del ref
    return out


def eval_hea(quick):
    import qulacs
    from qompsim import circuits as C
    from qulacs.torch import energy, energy_and_gradient
    n, depth = 24, 8
    circ = C.hea(n, depth, seed=0, parametric=True)
    obs = qulacs.Observable(n)
    for coef, pauli, qubits in C.hea_observable_terms(n):
        obs.add_operator(coef, " ".join(f"{p} {q}" for p, q in zip(pauli, qubits)))
    npar = circ.get_parameter_count()
    # FP64 central differences on every parameter (h = 1e-4)
    h = 1e-4
    fd = np.zeros(npar)
    cc = circ.copy()
    for i in range(npar if not quick else 16):
        t = cc.get_parameter(i)
        cc.set_parameter(i, t + h)
        ep = energy(cc, obs, "complex128")
        cc.set_parameter(i, t - h)
        em = energy(cc, obs, "complex128")
        cc.set_parameter(i, t)
        fd[i] = (ep - em) / (2 * h)
    m = npar if not quick else 16
    out = []
    for dtype in ("complex64", "complex128"):
        energy_and_gradient(circ, obs, dtype)
        t_fwd = t_grad = float("inf")
        for _ in range(3):  # best of three, each call synchronised
            _sync()
            t0 = time.perf_counter()
            energy(circ, obs, dtype)
            _sync()
            t_fwd = min(t_fwd, time.perf_counter() - t0)
            t0 = time.perf_counter()
            e, g = energy_and_gradient(circ, obs, dtype)
            _sync()
            t_grad = min(t_grad, time.perf_counter() - t0)
        out.append({"config": f"hea{n}: n={n} depth={depth} {npar} parameters, uncompressed adjoint",
                    "dtype": dtype, "energy": e, "forward_ms": t_fwd * 1e3, "energy_and_gradient_ms": t_grad * 1e3,
                    "gradient_over_forward": t_grad / t_fwd,
                    "max_grad_err_vs_fd": float(np.max(np.abs(g[:m] - fd[:m]))), "params_checked": m})
    return out


def eval_qaoa(quick):
    import qulacs
    from qompsim import circuits as C
    from qulacs.torch import compressed_energy_and_gradient, energy_and_gradient
    out = []
    p = 4

    def build(n, seed=0):
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
        return c, obs, len(edges)

    # compressed adjoint against the uncompressed FP64 adjoint at a size where both fit
    n_chk = 20
    c, obs, ne = build(n_chk)
    e_ref, g_ref = energy_and_gradient(c, obs, "complex128")
    for ck in (False, True):
        e, g = compressed_energy_and_gradient(c, obs, block_size=n_chk - 8, dtype="complex64", checkpoints=ck)
        out.append({"config": f"qaoa{n_chk}: n={n_chk} p={p} gradient check, complex64 compressed, default bounds",
                    "checkpoints": ck, "energy": e, "energy_fp64": e_ref, "max_grad_err": float(np.max(np.abs(g - g_ref))),
                    "max_grad_fp64": float(np.max(np.abs(g_ref)))})
    # timing at the largest size whose two compressed states fit one GPU
    n = 24 if quick else 32
    c, obs, ne = build(n)
    B = n - 10
    _sync()
    t0 = time.perf_counter()
    from qulacs import CompressedQuantumState, _native
    cq = CompressedQuantumState(n, B, dtype="complex64", flags=_native.QS_FLAG_QUIET)
    plain = qulacs.QuantumCircuit(n)
    for gte in c._gates:
        plain.add_gate(gte)
    cq.partition_and_register_circuit(plain, 4, 0)
    cq.apply_circuit()
    e_fwd = obs.get_expectation_value(cq)
    _sync()
    t_fwd = time.perf_counter() - t0
    size = cq.get_max_SV_bytes()
    del cq
    t0 = time.perf_counter()
    e, g = compressed_energy_and_gradient(c, obs, block_size=B, dtype="complex64", checkpoints=False)
    _sync()
    t_grad = time.perf_counter() - t0
    out.append({"config": f"qaoa{n}: n={n} p={p} {ne} edges, complex64 compressed, default bounds",
                "energy": e, "forward_energy": e_fwd, "forward_ms": t_fwd * 1e3, "energy_and_gradient_ms": t_grad * 1e3,
                "gradient_over_forward": t_grad / t_fwd, "max_sv_bytes": size, "gradient_params": len(g)})
    return out


def eval_host_store(quick):
    """Spill tier: the QFT with its payload arenas in pinned host memory
    (each arena bounded to 4 GiB) against the HBM store, same passes."""
    import os
    from qompsim import circuits as C
    n = 26 if quick else 28
    B, I = 20, 4
    out = []
    first = None
    for host in (False, True):
        old = os.environ.get("QOMPSIM_ARENA_BYTES")
        if host:
            os.environ["QOMPSIM_ARENA_BYTES"] = str(4 << 30)
        try:
            c = _optimized(C.qft_basis(n, 0), B)
            cq, info = _compressed_run(c, n, B, I, "complex128", host_store=host)
        finally:
            if host:
                if old is None:
                    os.environ.pop("QOMPSIM_ARENA_BYTES", None)
                else:
                    os.environ["QOMPSIM_ARENA_BYTES"] = old
        st = cq.get_stats()
        moved = st["bytes_read"] + st["bytes_written"]
        head = cq.get_amplitudes(0, min(SLICE, 1 << n), renormalize=False)
        if first is None:
            first = head
        info.update(host_store=bool(st["host_store"]), payload_and_header_bytes=int(moved),
                    effective_gb_per_s=moved / (info["apply_ms"] * 1e6),
                    first_slice_identical=bool(np.array_equal(head, first)))
        out.append({"config": f"qft{n} spill tier: n={n} B={B} I={I}, payload in "
                              f"{'pinned host memory' if host else 'HBM'}", **info})
        del cq
    return out


EVALS = {"ghz20": eval_ghz, "qft30": eval_qft, "brickwork32": eval_brickwork, "hea24": eval_hea, "qaoa34": eval_qaoa,
         "host_store28": eval_host_store}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=list(EVALS))
    ap.add_argument("--quick", action="store_true")
    a = ap.parse_args(argv)
    for name in a.only:
        try:
            res = EVALS[name](a.quick)
        except Exception as exc:  # one configuration failing does not stop the others
            res = {"config": name, "error": f"{type(exc).__name__}: {exc}"}
        for r in (res if isinstance(res, list) else [res]):
            print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()

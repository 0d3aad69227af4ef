"""One-rank driver mode of the reference's script/run_sim.py.

The reference script exits unless qulacs was built with MPI
(script/run_sim.py:11-17); this engine runs one GPU with no ranks, so this
module provides the same command line and the same flow for one rank:

    python -m qompsim.run_sim -s {qulacs,qompsim,fidelity} -c NAME -n N
           [-o DIR] [-a] [-b B] [-i I] [--factory DIR]

NAME is a circuit of the reference's benchmark/circuit_factory.py (pass the
directory holding it with --factory; it builds its circuits through this
package's qulacs API) or one of this package's workloads (qompsim.circuits:
ghz_fanout, qft_basis, brickwork, hea, qaoa_maxcut).  Block size, inner size,
fusion (optimize(block_size=2)), the printed lines, the JSON records and the
fidelity |<psi_qulacs|psi_qompsim>| follow run_sim.py:60-207.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np


class RunResult:
    def __init__(self):
        self.times: dict = {}
        self.sv_MiB: float = 0.0
        self.fidelity = None


def get_circuit(name: str, nqubits: int, factory: str | None):
    if factory:
        sys.path.insert(0, factory)
        import circuit_factory  # the reference's generator
        return circuit_factory.get_circuit(name, nqubits)
    from . import circuits as C
    builders = {"ghz_fanout": C.ghz_fanout, "qft_basis": C.qft_basis, "brickwork": C.brickwork,
                "hea": lambda n: C.hea(n, 8, 0), "qaoa_maxcut": lambda n: C.qaoa_maxcut(n, 4, 0)}
    if name not in builders:
        raise SystemExit(f"unknown circuit {name!r}: pass --factory <dir of circuit_factory.py> for the "
                         f"reference's circuit names, or use one of {sorted(builders)}")
    return builders[name](nqubits)


def write_result(result: RunResult, outfile: str | None, append: bool) -> None:
    print(f"Simulation time: {result.times['overall']:.3f} seconds")
    print(f"State vector size: {result.sv_MiB:.3f} MiB")
    if result.fidelity is not None:
        print(f"Fidelity: {result.fidelity:.6f}")
    if outfile is not None:
        if not os.path.exists(outfile) or append:
            with open(outfile, "a") as f:
                json.dump(vars(result), f)
                f.write("\n")
        print(outfile)
    else:
        print(vars(result))
    print()


def run_sim(simulator: str, circuit_name: str, nqubits: int, outdir=None, append=False, block_size=None,
            inner_size=None, factory=None):
    import qulacs
    from qulacs import CompressedQuantumState, QuantumState
    from qulacs.circuit import QuantumCircuitOptimizer

    nranks = 1
    if simulator in ("qompsim", "fidelity"):
        if inner_size is None:
            inner_size = 4
        if block_size is None:
            block_size = min(nqubits - max(int(np.log2(nranks)), 1) - inner_size - 1, 26)
    circuit = get_circuit(circuit_name, nqubits, factory)
    QuantumCircuitOptimizer(sv_block_size=block_size or 0).optimize(circuit, block_size=2)
    vectors = {}
    if simulator in ("qulacs", "fidelity"):
        out = f"{outdir}/qulacs_{circuit_name}_{nqubits}qubits_{nranks}ranks.json" if outdir else None
        res = RunResult()
        print("======== Qulacs ========")
        t0 = time.time()
        qs = QuantumState(nqubits)
        t1 = time.time()
        circuit.update_quantum_state(qs)
        t2 = time.time()
        res.times.update(init=t1 - t0, overall=t2 - t1, fused_swap=qs.get_fused_swap_time())
        res.sv_MiB = 2 ** (nqubits + 4) / (1024 ** 2)
        write_result(res, out, append)
        if simulator == "fidelity":
            vectors["qulacs"] = qs.get_vector()
    if simulator in ("qompsim", "fidelity"):
        assert block_size + inner_size + int(np.log2(nranks)) < nqubits, \
            f"{block_size=} and {inner_size=} are too large for the number of qubits and ranks."
        out = (f"{outdir}/qompsim_{circuit_name}_{nqubits}qubits_{nranks}ranks_bs{block_size}_inner{inner_size}.json"
               if outdir else None)
        res = RunResult()
        print("======== QompSim ========")
        print(f"block_size: {block_size}, inner_size: {inner_size}")
        t0 = time.time()
        cqs = CompressedQuantumState(nqubits, block_size)
        cqs.partition_and_register_circuit(circuit, inner_size, verbose=1)
        t1 = time.time()
        cqs.apply_circuit()
        t2 = time.time()
        res.times.update(init=t1 - t0, overall=t2 - t1)
        res.times.update(cqs.get_total_times())
        res.sv_MiB = cqs.get_max_SV_bytes() / (1024 ** 2)
        if simulator == "qompsim":
            write_result(res, out, append)
        else:
            print("Calculating fidelity between Qulacs and QompSim...")
            v = cqs.get_vector()
            print(" Qulacs  sv[0]: ", vectors["qulacs"][0])
            print("QompSim  sv[0]: ", v[0])
            print(" Qulacs sv[-1]: ", vectors["qulacs"][-1])
            print("QompSim sv[-1]: ", v[-1])
            res.fidelity = float(np.abs(np.vdot(vectors["qulacs"], v)))
            write_result(res, out, append)
    return vectors


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("-s", "--simulator", choices=["qulacs", "qompsim", "fidelity"], required=True)
    ap.add_argument("-c", "--circuit_name", required=True)
    ap.add_argument("-n", "--nqubits", type=int, required=True)
    ap.add_argument("-o", "--outdir", default=None)
    ap.add_argument("-a", "--append", action="store_true", default=False)
    ap.add_argument("-b", "--block_size", type=int, default=None)
    ap.add_argument("-i", "--inner_size", type=int, default=None)
    ap.add_argument("--factory", default=None, help="directory holding the reference's circuit_factory.py")
    a = ap.parse_args(argv)
    run_sim(a.simulator, a.circuit_name, a.nqubits, a.outdir, a.append, a.block_size, a.inner_size, a.factory)


if __name__ == "__main__":
    main()

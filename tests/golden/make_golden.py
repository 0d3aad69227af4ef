"""Generate the golden fixtures of tests/golden/ from the reference itself.

Run in a container where the reference is mounted (it does not travel):

    python tests/golden/make_golden.py <reference checkout>

What comes from the reference:
* the circuits: the reference's own generators (benchmark/circuit_factory.py,
  benchmark/grover.py) are imported and executed; they build their circuits
  through this repository's qulacs API, so the fixture records exactly the
  gate sequence (names, qubits, angles, matrices) the reference's scripts
  produce;
* the states: each circuit is applied to |0...0> with the reference's own FP64
  kernels (Qulacs csim, compiled from the reference sources into
  oracle/_ref/libcsim_ref.so) -- the uncompressed result the reference's
  fidelity mode compares against (script/run_sim.py:125-142).

Outputs: reference_circuits.json (gate lists) and reference_states.npz
(complex128 vectors), keyed "<name>_<n>".
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "compression-based-state-vector-simulator_b200"))
sys.path.insert(0, ROOT)

CASES = [
    ("hadamard", 8), ("seq_hadamard", 9), ("ghz", 10), ("qft", 8), ("ising", 8), ("hea", 9),
    ("grover", 11), ("cc", 9), ("bv", 9), ("qsvm", 8), ("qaoa", 9), ("wstate", 8),
]


def gate_record(g):
    m = np.asarray(g.get_matrix(), dtype=np.complex128)
    return {
        "name": g.get_name(),
        "targets": g.get_target_index_list(),
        "target_props": [t.prop for t in g.target_qubit_list],
        "controls": g.get_control_index_list(),
        "control_values": g.get_control_value_list(),
        "gate_property": g.get_property_value(),
        "matrix_re": m.real.tolist(),
        "matrix_im": m.imag.tolist(),
    }


def main(ref: str) -> None:
    import contextlib
    import io

    from oracle import csim_ref

    sys.path.insert(0, os.path.join(ref, "benchmark"))
    import circuit_factory  # the reference's generator

    circuits, states = {}, {}
    for name, n in CASES:
        with contextlib.redirect_stdout(io.StringIO()):
            c = circuit_factory.get_circuit(name, n)
        key = f"{name}_{n}"
        circuits[key] = {"n": n, "gates": [gate_record(g) for g in c._gates]}
        states[key] = csim_ref.run_circuit(n, c._gates)
    with open(os.path.join(HERE, "reference_circuits.json"), "w") as f:
        json.dump(circuits, f)
    np.savez_compressed(os.path.join(HERE, "reference_states.npz"), **states)
    print(f"wrote {len(circuits)} circuits")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout (the directory holding src/ and benchmark/)>")
    main(sys.argv[1])

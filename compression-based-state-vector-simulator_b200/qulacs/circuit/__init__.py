"""qulacs.circuit: QuantumCircuitOptimizer.

Restates QuantumCircuitOptimizer::optimize(circuit, max_block_size, swap_level)
(src/cppsim/circuit_optimizer.cpp:113-168) with its helpers
get_rightmost_commute_index / get_leftmost_commute_index (:35-54),
get_merged_gate_size (:56-100) and is_neighboring (:104-111).  The merge order
and insertion point are the reference's, so the fused gate list -- which
decides the compressed engine's stages -- is the same gate for gate.

swap_level > 0 (SWAP / FusedSWAP insertion, circuit_optimizer.cpp:834+) only
matters with MPI ranks; this build has one GPU and no ranks, so
insert_swap_gates is a no-op here (the reference also skips it when there is
one rank: :851-857), and can_merge_with_swap_insertion is always true.
"""
from __future__ import annotations

from typing import List

from .._gates import QuantumGateBase, merge


class QuantumCircuitOptimizer:
    def __init__(self, mpi_size: int = 0, sv_block_size: int = 0):
        self.mpi_size = int(mpi_size)
        self.sv_block_size = int(sv_block_size)

    # set_qubit_count (circuit_optimizer.cpp:407-423) for one rank.
    def _check_sizes(self, circuit) -> None:
        if self.sv_block_size > circuit.get_qubit_count():
            raise RuntimeError(
                "Error: QuantumCircuitOptimizer::set_qubit_count() "
                "sv_block_size must be less than or equal to local_qc")

    def optimize(self, circuit, block_size: int, swap_level: int = 0) -> None:
        self._check_sizes(circuit)
        if swap_level > 2:
            raise ValueError("invalid swap_level (0, 1 or 2)")
        gl: List[QuantumGateBase] = circuit._gates
        qsets = [set(g.full_qubits()) for g in gl]
        merged_flag = True
        while merged_flag:
            merged_flag = False
            ind1 = 0
            while ind1 < len(gl):
                ind2 = ind1 + 1
                while ind2 < len(gl):
                    if gl[ind1].is_parametric() or gl[ind2].is_parametric():
                        ind2 += 1
                        continue
                    if len(qsets[ind1] | qsets[ind2]) > block_size:
                        ind2 += 1
                        continue
                    if not _is_neighboring(gl, ind1, ind2):
                        ind2 += 1
                        continue
                    merged = merge(gl[ind1], gl[ind2])
                    ind2_left = _leftmost_commute(gl, ind2, floor=ind1 + 1)
                    insert_point = max(ind2_left, ind1 + 1)
                    del gl[ind2]
                    del qsets[ind2]
                    gl.insert(insert_point, merged)
                    qsets.insert(insert_point, set(merged.full_qubits()))
                    del gl[ind1]
                    del qsets[ind1]
                    merged_flag = True
                    # ind2-- then ++ind2 in the reference: ind2 is unchanged
                ind1 += 1

    def optimize_light(self, circuit, swap_level: int = 0) -> None:
        raise NotImplementedError("optimize_light is not on the compressed-state path")

    def merge_all(self, circuit):
        from .._gates import QuantumGateMatrix
        import numpy as np
        cur = QuantumGateMatrix([], np.eye(1, dtype=np.complex128))
        for g in circuit._gates:
            cur = merge(cur, g)
        return cur


def _rightmost_commute(gl, i, ceil):
    """get_rightmost_commute_index, scanning no further than `ceil`."""
    g = gl[i]
    cursor = i + 1
    while cursor < len(gl) and cursor <= ceil:
        if not g.is_commute(gl[cursor]):
            break
        cursor += 1
    return cursor - 1


def _leftmost_commute(gl, i, floor=0):
    """get_leftmost_commute_index, scanning no further down than `floor`."""
    g = gl[i]
    cursor = i - 1
    while cursor >= 0 and cursor >= floor:
        if not g.is_commute(gl[cursor]):
            break
        cursor -= 1
    return cursor + 1


def _is_neighboring(gl, i1, i2) -> bool:
    """ind2_left <= ind1_right + 1 with both scans cut where the answer is
    already decided (the comparison only needs them inside (i1, i2))."""
    r1 = _rightmost_commute(gl, i1, ceil=i2 - 1)
    if r1 >= i2 - 1:
        return True
    l2 = _leftmost_commute(gl, i2, floor=r1 + 1)
    return l2 <= r1 + 1


__all__ = ["QuantumCircuitOptimizer"]

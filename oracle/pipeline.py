"""ORACLE (test infrastructure only): the reference's compressed group loop
restated on the CPU over numpy blocks.

Follows CompressedQuantumState::apply_circuit / process_SV_group
(src/cppsim/compressed_state.hpp:840-1029) and the block-pair gate loops
apply_1q_gate (:1066-1144), apply_cnot (:1146-1264), apply_2q_gate
(:1266-1381):

* blocks are numpy complex128 arrays of 2^B amplitudes, or None for a zero
  block (the reference's nullptr);
* per stage, active groups are the groups holding a stored block, visited in
  ascending group id, their blocks in ascending block id (:791-837);
* every block of an active group is processed, zero blocks as zeros (Q8);
* after the gates only blocks that were zero before the stage are tested
  (Q1): `zero_test` selects the GPU build's exact test
  (cuda_complex_helper.cuh:96-106), ("code", L) -- every component
  quantises to code 0, |x| <= 2^-(L+1) -- or a float threshold (the CPU
  build's ALL_ZERO_THRESHOLD, :939-951);
* then every processed block goes through `codec` (a function on complex128
  arrays) -- the lossy round trip of compression.

`reference_controls=True` reproduces the reference's dispatch (controls
honoured for "CNOT" only, 2x2/4x4 matrices applied uncontrolled with matrix
bit 0 on the lower target, Q3/Q4); False folds controls into the matrix and
keeps csim's target order, which is what the B200 engine does by default.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

import numpy as np

from . import planner


def _pairs_in_block(arr: np.ndarray, t: int):
    a = arr.reshape(-1, 2, 1 << t)
    return a[:, 0, :], a[:, 1, :]


def _apply_1q(m, t, blocks, ids, B):
    if t < B:
        for b in ids:
            x0, x1 = _pairs_in_block(blocks[b], t)
            n0 = m[0, 0] * x0 + m[0, 1] * x1
            n1 = m[1, 0] * x0 + m[1, 1] * x1
            x0[...] = n0
            x1[...] = n1
    else:
        bm = 1 << (t - B)
        pending = list(ids)
        while pending:
            b0 = pending.pop(0)
            b1 = b0 + bm
            pending.remove(b1)
            a0, a1 = blocks[b0], blocks[b1]
            n0 = m[0, 0] * a0 + m[0, 1] * a1
            n1 = m[1, 0] * a0 + m[1, 1] * a1
            a0[...] = n0
            a1[...] = n1


def _apply_2q(m, q0, q1, blocks, ids, B):
    """4x4 with matrix bit 0 on q0 and bit 1 on q1 (any order)."""
    lo, hi = min(q0, q1), max(q0, q1)
    if q0 > q1:  # re-express with bit 0 on the lower qubit
        p = [0, 2, 1, 3]
        m = m[np.ix_(p, p)]
    if hi < B:
        for b in ids:
            a = blocks[b].reshape(-1, 2, 1 << (hi - lo - 1), 2, 1 << lo)
            v = [a[:, 0, :, 0, :], a[:, 0, :, 1, :], a[:, 1, :, 0, :], a[:, 1, :, 1, :]]
            new = [sum(m[r, c] * v[c] for c in range(4)) for r in range(4)]
            for r in range(4):
                v[r][...] = new[r]
    elif lo >= B:
        bm0, bm1 = 1 << (lo - B), 1 << (hi - B)
        pending = list(ids)
        while pending:
            b0 = pending.pop(0)
            b1, b2 = b0 + bm0, b0 + bm1
            b3 = b1 + bm1
            for x in (b1, b2, b3):
                pending.remove(x)
            v = [blocks[b0], blocks[b1], blocks[b2], blocks[b3]]
            new = [sum(m[r, c] * v[c] for c in range(4)) for r in range(4)]
            for r in range(4):
                v[r][...] = new[r]
    else:
        bm1 = 1 << (hi - B)
        pending = list(ids)
        while pending:
            b0 = pending.pop(0)
            b1 = b0 + bm1
            pending.remove(b1)
            x0, x1 = _pairs_in_block(blocks[b0], lo)
            y0, y1 = _pairs_in_block(blocks[b1], lo)
            v = [x0, x1, y0, y1]
            new = [sum(m[r, c] * v[c] for c in range(4)) for r in range(4)]
            for r in range(4):
                v[r][...] = new[r]


def _apply_cnot(c, t, blocks, ids, B):
    X = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    if t < B and c < B:
        for b in ids:
            a = blocks[b]
            idx = np.arange(a.size)
            sel = idx[((idx >> c) & 1 == 1) & ((idx >> t) & 1 == 0)]
            tmp = a[sel].copy()
            a[sel] = a[sel | (1 << t)]
            a[sel | (1 << t)] = tmp
    elif t < B:
        cb = 1 << (c - B)
        for b in ids:
            if b & cb:
                _apply_1q(X, t, blocks, [b], B)
    elif c < B:
        tb = 1 << (t - B)
        pending = list(ids)
        while pending:
            b0 = pending.pop(0)
            b1 = b0 + tb
            pending.remove(b1)
            a0, a1 = blocks[b0], blocks[b1]
            idx = np.arange(a0.size)
            sel = idx[(idx >> c) & 1 == 1]
            tmp = a0[sel].copy()
            a0[sel] = a1[sel]
            a1[sel] = tmp
    else:
        cb, tb = 1 << (c - B), 1 << (t - B)
        pending = [b for b in ids if b & cb]
        while pending:
            b0 = pending.pop(0)
            b1 = b0 + tb
            pending.remove(b1)
            tmp = blocks[b0].copy()
            blocks[b0][...] = blocks[b1]
            blocks[b1][...] = tmp


def _full_matrix(g):
    """Fold controls into the matrix over sorted qubits (bit i <-> qubits[i])."""
    from itertools import product  # noqa: F401
    t = g.get_target_index_list()
    c = g.get_control_index_list()
    cv = g.get_control_value_list()
    nt, nc = len(t), len(c)
    k = nt + nc
    m = np.eye(1 << k, dtype=np.complex128)
    cm = sum((v & 1) << i for i, v in enumerate(cv))
    base = cm << nt
    m[base:base + (1 << nt), base:base + (1 << nt)] = g.get_matrix()
    order = t + c
    srt = sorted(order)
    if order != srt:
        pos = {q: i for i, q in enumerate(order)}
        perm = []
        for x in range(1 << k):
            y = 0
            for j, q in enumerate(srt):
                if (x >> j) & 1:
                    y |= 1 << pos[q]
            perm.append(y)
        m = m[np.ix_(perm, perm)]
    return m, srt


def _apply_gate(g, blocks, ids, B, reference_controls):
    name = g.get_name()
    t = g.get_target_index_list()
    c = g.get_control_index_list()
    if name == "CNOT":
        _apply_cnot(c[0], t[0], blocks, ids, B)
        return
    if reference_controls or not c:
        m = g.get_matrix()
        if m.shape == (2, 2):
            _apply_1q(m, t[0], blocks, ids, B)
        elif m.shape == (4, 4):
            if reference_controls:
                _apply_2q(m, min(t), max(t), blocks, ids, B)
            else:
                _apply_2q(m, t[0], t[1], blocks, ids, B)
        else:
            raise NotImplementedError("only single- or two-qubit gates are implemented")
        return
    m, qs = _full_matrix(g)
    if len(qs) == 1:
        _apply_1q(m, qs[0], blocks, ids, B)
    elif len(qs) == 2:
        _apply_2q(m, qs[0], qs[1], blocks, ids, B)
    else:
        raise NotImplementedError("only single- or two-qubit gates are implemented")


class CompressedOracle:
    """CPU restatement of the compressed state's stage loop."""

    def __init__(self, n: int, block_size: int, codec: Optional[Callable] = None, zero_test="exact",
                 reference_controls: bool = False):
        self.n, self.B = n, block_size
        self.nb = 1 << (n - block_size)
        self.codec = codec or (lambda v: v)
        self.zero_test = zero_test
        self.reference_controls = reference_controls
        self.blocks: List[Optional[np.ndarray]] = [None] * self.nb
        first = np.zeros(1 << block_size, dtype=np.complex128)
        first[0] = 1.0
        self.blocks[0] = self.codec(first)
        self.mask_history: List[np.ndarray] = [self.mask()]

    def set_basis_state(self, x: int):
        self.blocks = [None] * self.nb
        blk = np.zeros(1 << self.B, dtype=np.complex128)
        blk[x & ((1 << self.B) - 1)] = 1.0
        self.blocks[x >> self.B] = self.codec(blk)
        self.mask_history = [self.mask()]

    def mask(self) -> np.ndarray:
        return np.array([b is not None for b in self.blocks], dtype=np.uint8)

    def _is_zero(self, v: np.ndarray) -> bool:
        if self.zero_test == "exact":
            return not np.any((v.real * v.real + v.imag * v.imag) != 0.0)
        if isinstance(self.zero_test, tuple) and self.zero_test[0] == "code":
            # every component quantises to code 0: rint(|x| 2^L) == 0
            thr = 2.0 ** -(self.zero_test[1] + 1)
            return not np.any((np.abs(v.real) > thr) | (np.abs(v.imag) > thr))
        return not np.any((np.abs(v.real) > self.zero_test) | (np.abs(v.imag) > self.zero_test))

    def apply(self, gates: Sequence, stages: Sequence[Sequence[int]], maps, counts) -> None:
        for si, stage in enumerate(stages):
            active, members = planner.execution_plan(maps[si], counts[si], [b is not None for b in self.blocks])
            for gid in active:
                ids = members[gid]
                was_zero = {b: self.blocks[b] is None for b in ids}
                work = {b: (np.zeros(1 << self.B, dtype=np.complex128) if self.blocks[b] is None
                            else self.blocks[b].copy()) for b in ids}
                for gi in stage:
                    _apply_gate(gates[gi], work, ids, self.B, self.reference_controls)
                for b in ids:
                    if was_zero[b] and self._is_zero(work[b]):
                        self.blocks[b] = None
                    else:
                        self.blocks[b] = self.codec(work[b])
            self.mask_history.append(self.mask())

    def vector(self, renormalize: bool = True) -> np.ndarray:
        out = np.concatenate([b if b is not None else np.zeros(1 << self.B, dtype=np.complex128)
                              for b in self.blocks])
        if renormalize:
            nrm = np.sqrt(np.vdot(out, out).real)
            if nrm > 0:
                out = out / nrm
        return out

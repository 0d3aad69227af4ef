"""ORACLE (test infrastructure only): the reference's stage planner restated.

* partition_circuit        -- src/cppsim/compressed_state.hpp:509-583
* make_block_groups        -- compressed_state.hpp:585-671 (one rank)
* execution_plan           -- build_stage_group_execution_plan, :791-837
Gates are described by (name, targets, controls) so the planner is
independent of the product's gate classes.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

GateDesc = Tuple[str, Sequence[int], Sequence[int]]


def describe(gates) -> List[GateDesc]:
    return [(g.get_name(), list(g.get_target_index_list()), list(g.get_control_index_list())) for g in gates]


def partition_circuit(gates: Sequence[GateDesc], block_size: int, inner_size: int) -> List[List[int]]:
    stages: List[List[int]] = []
    current: List[int] = []
    global_indices: List[int] = []
    global_targets: List[int] = []
    threshold = max(inner_size, 2)
    for i, (name, targets, controls) in enumerate(gates):
        if name == "FusedSWAP":
            if current:
                stages.append(current)
            stages.append([i])
            current = []
            global_indices = []
            continue
        for t in targets:
            if t >= block_size:
                global_targets.append(t)
        for c in controls:
            if c >= block_size:
                global_targets.append(c)
        tmp = list(global_indices)
        for gt in global_targets:
            if gt not in tmp:
                tmp.append(gt)
        if len(tmp) > threshold:
            stages.append(current)
            current = []
            tmp = list(global_targets)
            global_indices = []
            global_targets = []
        global_indices = tmp
        global_targets = []
        current.append(i)
    if current:
        stages.append(current)
    return stages


def make_block_groups(gates: Sequence[GateDesc], stages: Sequence[Sequence[int]], n: int, block_size: int):
    """-> (block_to_group per stage, num_groups per stage)."""
    nb = 1 << (n - block_size)
    maps, counts = [], []
    for stage in stages:
        inner = set(range(block_size))
        for gi in stage:
            _, targets, controls = gates[gi]
            inner.update(q for q in targets if q >= block_size)
            inner.update(q for q in controls if q >= block_size)
        outer = [q for q in range(n) if q not in inner]
        m = []
        for b in range(nb):
            gid = 0
            for i, oq in enumerate(outer):
                gid |= ((b >> (oq - block_size)) & 1) << i
            m.append(gid)
        maps.append(m)
        counts.append(1 << len(outer))
    return maps, counts


def execution_plan(block_to_group: Sequence[int], num_groups: int, nonzero: Sequence[bool]):
    """-> (active group ids ascending, {group: ascending block ids})."""
    counts = [0] * num_groups
    for b, g in enumerate(block_to_group):
        if nonzero[b]:
            counts[g] += 1
    active = [g for g in range(num_groups) if counts[g] > 0]
    members = {g: [] for g in range(num_groups)}
    for b, g in enumerate(block_to_group):
        members[g].append(b)
    return active, members

"""Compressed state vector sharded over ranks (the reference's multi-rank mode).

The reference distributes a state of n qubits over P = 2^g MPI ranks: rank r
holds the blocks [r nb/P, (r+1) nb/P), so the top g qubits are "global"
(src/cppsim/state.hpp:86-124, compressed_state.hpp:156-160, 630-638), and
its optimizer inserts FusedSWAP gates that bring global qubits into the
local range before any gate that needs them; the compressed engine then
exchanges compressed blocks between rank pairs (apply_fused_swap,
compressed_state.hpp:1396-1546).

Here every rank runs this package's engine on its local store of n - g
qubits, and the layout is managed at run time instead of by inserted gates:

* a gate is applied locally when every global qubit it touches is one it
  does not mix (controls, phases, Z-type factors): the gate restricted to
  the rank's fixed value of those qubits acts on local qubits only;
* a gate that mixes a global qubit first swaps that qubit with a local one
  (>= the chunk bits): each rank sends the half of its store whose local bit
  differs from its own global bit to the partner rank across that bit and
  receives the partner's half into the same positions.  The halves are
  compressed chunks (headers and payloads, `qs_export_half` /
  `qs_import_half`), never decoded; SWAP and FusedSWAP gates of the circuit
  only relabel qubits;
* after the circuit the qubits are put back in order (global qubits by
  exchanges, local ones by local SWAPs), so the store layout is the
  reference's.

Every rank makes the same layout decisions from the gate list alone, so the
exchanges pair up.  The transport is `torch.distributed` point-to-point
(NCCL over NVLink for CUDA buffers; gloo for the CPU tests), or
`ThreadExchange` for ranks run as threads of one process.
"""
from __future__ import annotations

import threading
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as _n

__all__ = ["ShardedCompressedQuantumState", "TorchExchange", "ThreadExchange", "CompressedShard", "NumpyShard",
           "gate_as_dense"]


# ---------------------------------------------------------------- transports
class TorchExchange:
    """Point-to-point exchange over a torch.distributed process group."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self._dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def _peer(self, r: int) -> int:
        return self._dist.get_global_rank(self.group, r) if self.group is not None else r

    def sendrecv(self, peer: int, buf):
        """Send `buf` (a 1-D uint8 tensor) to `peer` and return what `peer`
        sent (same device), with one size exchange first."""
        import torch
        dist = self._dist
        p = self._peer(peer)
        n_out = torch.tensor([buf.numel()], dtype=torch.int64, device=buf.device)
        n_in = torch.empty_like(n_out)
        for r in dist.batch_isend_irecv([dist.P2POp(dist.isend, n_out, p, self.group),
                                        dist.P2POp(dist.irecv, n_in, p, self.group)]):
            r.wait()
        out = torch.empty(int(n_in.item()), dtype=torch.uint8, device=buf.device)
        for r in dist.batch_isend_irecv([dist.P2POp(dist.isend, buf, p, self.group),
                                        dist.P2POp(dist.irecv, out, p, self.group)]):
            r.wait()
        return out

    def allgather(self, arr: np.ndarray) -> List[np.ndarray]:
        import torch
        t = torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).copy())
        if self._dist.get_backend(self.group) == "nccl":
            t = t.cuda()
        outs = [torch.empty_like(t) for _ in range(self.size)]
        self._dist.all_gather(outs, t, group=self.group)
        return [o.cpu().numpy().view(arr.dtype) for o in outs]


class ThreadExchange:
    """Ranks run as threads of one process: `endpoint(r)` is rank r's view.
    Buffers are handed over as objects (the receiver copies them)."""

    def __init__(self, size: int, timeout: float = 120.0):
        self.size = size
        self._timeout = timeout
        self._cv = threading.Condition()
        self._box: Dict[Tuple[int, int, int], object] = {}
        self._seq: Dict[Tuple[int, int], int] = {}

    def endpoint(self, rank: int) -> "_ThreadEndpoint":
        return _ThreadEndpoint(self, rank)

    def _post(self, key, obj):
        with self._cv:
            self._box[key] = obj
            self._cv.notify_all()

    def _take(self, key):
        with self._cv:
            if not self._cv.wait_for(lambda: key in self._box, timeout=self._timeout):
                raise TimeoutError(f"exchange {key} timed out")
            return self._box.pop(key)


class _ThreadEndpoint:
    def __init__(self, hub: ThreadExchange, rank: int):
        self.hub = hub
        self.rank = rank
        self.size = hub.size

    def _next(self, a: int, b: int) -> int:
        with self.hub._cv:
            k = self.hub._seq.get((a, b), 0)
            self.hub._seq[(a, b)] = k + 1
        return k

    def sendrecv(self, peer: int, buf):
        k_out = self._next(self.rank, peer)
        self.hub._post((self.rank, peer, k_out), buf.clone() if hasattr(buf, "clone") else np.array(buf))
        k_in = self._next(-1 - peer, self.rank)   # receive counter, separate from the send one
        return self.hub._take((peer, self.rank, k_in))

    def allgather(self, arr: np.ndarray) -> List[np.ndarray]:
        out = []
        k = self._next(self.rank, -1)
        # the posted copy carries how many other ranks still have to read it
        self.hub._post((self.rank, -1, k), [np.array(arr), self.size - 1])
        for r in range(self.size):
            if r == self.rank:
                out.append(np.array(arr))
                continue
            with self.hub._cv:
                key = (r, -1, k)
                if not self.hub._cv.wait_for(lambda: key in self.hub._box, timeout=self.hub._timeout):
                    raise TimeoutError(f"allgather {key} timed out")
                entry = self.hub._box[key]
                out.append(np.array(entry[0]))
                entry[1] -= 1
                if entry[1] == 0:
                    del self.hub._box[key]
        return out


# ---------------------------------------------------------------- gate algebra
def gate_as_dense(g) -> Tuple[List[int], np.ndarray]:
    """(qubits, matrix) of a gate: its targets then its controls, matrix
    index bit i <-> qubits[i]; the control pattern selects the target matrix,
    every other pattern is the identity."""
    t = list(g.get_target_index_list())
    c = list(g.get_control_index_list())
    cv = list(g.get_control_value_list())
    m = np.asarray(g.get_matrix(), dtype=np.complex128)
    if not c:
        return t, m
    nt, k = len(t), len(t) + len(c)
    dim_t = 1 << nt
    full = np.eye(1 << k, dtype=np.complex128)
    on = sum(v << (nt + i) for i, v in enumerate(cv))
    full[on:on + dim_t, on:on + dim_t] = m
    return t + c, full


def _mixes(m: np.ndarray, i: int) -> bool:
    """Whether matrix m couples index patterns that differ in bit i."""
    dim = m.shape[0]
    x = np.arange(dim)
    cross = ((x[:, None] ^ x[None, :]) >> i) & 1
    return bool(np.any((cross == 1) & (m != 0)))


def _restrict(qubits: List[int], m: np.ndarray, fixed: Dict[int, int]) -> Tuple[List[int], np.ndarray]:
    """The matrix on the remaining qubits when qubits[i] = fixed[i] (for a
    bit the matrix does not mix)."""
    keep = [i for i in range(len(qubits)) if i not in fixed]
    base = sum(v << i for i, v in fixed.items())
    idx = []
    for y in range(1 << len(keep)):
        x = base
        for j, i in enumerate(keep):
            if (y >> j) & 1:
                x |= 1 << i
        idx.append(x)
    idx = np.array(idx)
    return [qubits[i] for i in keep], m[np.ix_(idx, idx)]


_SWAP = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=np.complex128)


# ---------------------------------------------------------------- local stores
class CompressedShard:
    """A rank's local store: this package's compressed engine on n_local qubits."""

    def __init__(self, n_local: int, block_size: int, dtype=None, eps_rel=None, eps_abs=None, flags=None,
                 inner_size: int = 4):
        from . import CompressedQuantumState
        kw = {}
        if flags is not None:
            kw["flags"] = flags
        self.state = CompressedQuantumState(n_local, block_size, dtype=dtype, eps_rel=eps_rel, eps_abs=eps_abs, **kw)
        self.n_local = n_local
        self.inner_size = inner_size
        self.chunk_bits = int(self.state.get_stats()["chunk_log2"])

    def set_basis(self, x: int) -> None:
        self.state.set_computational_basis(x)

    def set_zero(self) -> None:
        self.state._check(_n.lib().qs_set_zero_vector(self.state._h))

    def apply(self, gates: Sequence[Tuple[List[int], np.ndarray]]) -> None:
        if not gates:
            return
        from . import QuantumCircuit, gate
        c = QuantumCircuit(self.n_local)
        for q, m in gates:
            c.add_gate(gate.DenseMatrix(q, m))
        self.state.partition_and_register_circuit(c, self.inner_size, 0)
        self.state.apply_circuit()

    def export_half(self, qubit: int, value: int):
        import torch
        L = _n.lib()
        size = _n.ct.c_uint64()
        self.state._check(L.qs_export_half(self.state._h, qubit, value, None, 0, _n.ct.byref(size)))
        buf = torch.empty(size.value, dtype=torch.uint8, device="cuda")
        self.state._check(L.qs_export_half(self.state._h, qubit, value, _n.ct.c_void_p(buf.data_ptr()),
                                           size.value, _n.ct.byref(size)))
        return buf

    def import_half(self, qubit: int, value: int, buf) -> None:
        import torch
        if buf.device.type != "cuda":
            buf = buf.cuda()
        torch.cuda.synchronize(buf.device)
        self.state._check(_n.lib().qs_import_half(self.state._h, qubit, value, _n.ct.c_void_p(buf.data_ptr()),
                                                  buf.numel()))

    def vector(self) -> np.ndarray:
        return self.state.get_vector(renormalize=False)


class NumpyShard:
    """A dense complex128 local store (the orchestration's CPU test double)."""

    def __init__(self, n_local: int, chunk_bits: int = 0):
        self.n_local = n_local
        self.chunk_bits = chunk_bits
        self.v = np.zeros(1 << n_local, dtype=np.complex128)

    def set_basis(self, x: int) -> None:
        self.v[:] = 0
        self.v[x] = 1

    def set_zero(self) -> None:
        self.v[:] = 0

    def apply(self, gates) -> None:
        n = self.n_local
        for q, m in gates:
            k = len(q)
            t = self.v.reshape([2] * n)
            axes = [n - 1 - qq for qq in reversed(q)]   # matrix bit i <-> q[i]; tensor axis 0 = top qubit
            t = np.moveaxis(t, axes, list(range(k)))
            sh = t.shape
            t = (m @ t.reshape(1 << k, -1)).reshape(sh)
            self.v = np.moveaxis(t, list(range(k)), axes).reshape(-1)

    def _half(self, qubit: int, value: int) -> np.ndarray:
        x = np.arange(1 << self.n_local)
        return np.nonzero(((x >> qubit) & 1) == value)[0]

    def export_half(self, qubit: int, value: int):
        import torch
        if not self.chunk_bits <= qubit < self.n_local:
            raise ValueError("exchanged qubit must lie in [chunk bits, n)")
        return torch.from_numpy(self.v[self._half(qubit, value)].copy().view(np.uint8))

    def import_half(self, qubit: int, value: int, buf) -> None:
        self.v[self._half(qubit, value)] = buf.numpy().view(np.complex128)

    def vector(self) -> np.ndarray:
        return self.v.copy()


# ---------------------------------------------------------------- sharded state
class ShardedCompressedQuantumState:
    """CompressedQuantumState(n, B) over P = 2^g ranks (see the module text).

    exchange: a TorchExchange (default: the default process group) or a
    ThreadExchange endpoint; shard: the local store (default: a
    CompressedShard of n - g qubits with this block size)."""

    def __init__(self, qubit_count: int, block_size: int, dtype=None, eps_rel: Optional[float] = None,
                 eps_abs: Optional[float] = None, flags: Optional[int] = None, exchange=None, shard=None,
                 lookahead: int = 64):
        self.ex = exchange if exchange is not None else TorchExchange()
        P = self.ex.size
        g = P.bit_length() - 1
        if P <= 0 or (1 << g) != P:
            raise ValueError("the number of ranks must be a power of two")
        self.n = int(qubit_count)
        self.g = g
        self.n_local = self.n - g
        self.rank = self.ex.rank
        self.shard = shard if shard is not None else CompressedShard(self.n_local, block_size, dtype, eps_rel, eps_abs,
                                                                     flags)
        if self.shard.n_local != self.n_local:
            raise ValueError("local store size does not match n - log2(ranks)")
        if g and self.n_local <= self.shard.chunk_bits:
            raise ValueError("each rank needs a local qubit above its chunk bits to exchange through")
        self.lookahead = lookahead
        self._gates: List = []
        self._inner = 4
        self.exchanges = 0
        self.exchanged_bytes = 0
        self.set_zero_state()

    # ---- layout
    def _identity(self) -> None:
        self.l2p = list(range(self.n))   # logical qubit -> physical position
        self.p2l = list(range(self.n))

    def set_zero_state(self) -> None:
        self.set_computational_basis(0)

    def set_computational_basis(self, basis: int) -> None:
        self._identity()
        if (basis >> self.n_local) == self.rank:
            self.shard.set_basis(basis & ((1 << self.n_local) - 1))
        else:
            self.shard.set_zero()

    def _rank_bit(self, phys: int) -> int:
        return (self.rank >> (phys - self.n_local)) & 1

    def _swap_global(self, G: int, l: int) -> None:
        """Exchange physical global qubit G with physical local qubit l."""
        b = self._rank_bit(G)
        peer = self.rank ^ (1 << (G - self.n_local))
        buf = self.shard.export_half(l, 1 - b)
        got = self.ex.sendrecv(peer, buf)
        self.shard.import_half(l, 1 - b, got)
        self.exchanges += 1
        self.exchanged_bytes += int(buf.numel())
        a, c = self.p2l[G], self.p2l[l]
        self.p2l[G], self.p2l[l] = c, a
        self.l2p[a], self.l2p[c] = l, G

    def _swap_local(self, p: int, l: int) -> None:
        """Exchange the qubits at local positions p and l (a local SWAP)."""
        self.shard.apply([([p, l], _SWAP)])
        a, c = self.p2l[p], self.p2l[l]
        self.p2l[p], self.p2l[l] = c, a
        self.l2p[a], self.l2p[c] = l, p

    def _pick_local(self, busy: Sequence[int], upcoming: Sequence[int]) -> int:
        """A local position >= the chunk bits for an incoming global qubit: not
        one the current gate uses, preferring one whose qubit no upcoming gate
        uses, then the highest."""
        lo = self.shard.chunk_bits
        cands = [p for p in range(self.n_local - 1, lo - 1, -1) if p not in busy]
        if not cands:
            raise RuntimeError("no local qubit left to exchange through")
        soon = set(upcoming)
        for p in cands:
            if self.p2l[p] not in soon:
                return p
        return cands[0]

    # ---- circuit
    def partition_and_register_circuit(self, circuit, inner_size: int = 4, verbose: int = 0) -> None:
        self._gates = list(circuit._gates)
        self._inner = int(inner_size)
        if hasattr(self.shard, "inner_size"):
            self.shard.inner_size = self._inner

    def apply_circuit(self) -> None:
        gates = self._gates
        seg: List[Tuple[List[int], np.ndarray]] = []
        for gi, gt in enumerate(gates):
            name = gt.get_name()
            if name in ("SWAP", "FusedSWAP"):
                # relabelling only: exchange the logical qubits' positions
                t = list(gt.get_target_index_list())
                w = len(t) // 2
                for a, c in zip(t[:w], t[w:]):
                    pa, pc = self.l2p[a], self.l2p[c]
                    self.l2p[a], self.l2p[c] = pc, pa
                    self.p2l[pa], self.p2l[pc] = c, a
                continue
            qubits, m = gate_as_dense(gt)
            while True:
                phys = [self.l2p[q] for q in qubits]
                mix = [i for i, p in enumerate(phys) if p >= self.n_local and _mixes(m, i)]
                if not mix:
                    break
                self.shard.apply(seg)
                seg = []
                upcoming = []
                for g2 in gates[gi + 1: gi + 1 + self.lookahead]:
                    upcoming += list(g2.get_target_index_list()) + list(g2.get_control_index_list())
                l = self._pick_local([p for p in phys if p < self.n_local], upcoming)
                self._swap_global(phys[mix[0]], l)
            fixed = {i: self._rank_bit(p) for i, p in enumerate(phys) if p >= self.n_local}
            lq, lm = _restrict(phys, m, fixed)
            if not lq:   # a phase on this rank's amplitudes: any local qubit carries it
                lq, lm = [0], lm[0, 0] * np.eye(2, dtype=np.complex128)
            seg.append((lq, lm))
        self.shard.apply(seg)
        self._restore_layout()

    def _restore_layout(self) -> None:
        """Physical position p back to logical qubit p for every p."""
        nl = self.n_local
        for G in range(nl, self.n):
            if self.l2p[G] == G:
                continue
            p = self.l2p[G]
            if p >= nl:   # logical G sits at another global position: bring it local first
                l = self._pick_local([], [])
                self._swap_global(p, l)
                p = l
            elif p < self.shard.chunk_bits:   # exchanges go through qubits above the chunk bits
                l = self._pick_local([p], [])
                self._swap_local(p, l)
                p = l
            self._swap_global(G, p)
        swaps = []
        for q in range(nl):
            p = self.l2p[q]
            if p != q:
                swaps.append(([p, q], _SWAP))
                o = self.p2l[q]
                self.l2p[q], self.l2p[o] = q, p
                self.p2l[q], self.p2l[p] = q, o
        self.shard.apply(swaps)

    # ---- readout
    def get_local_vector(self) -> np.ndarray:
        """This rank's 2^(n - g) amplitudes (global qubits = the rank)."""
        return self.shard.vector()

    def get_vector(self) -> np.ndarray:
        """The whole state on every rank (gathered; small n only)."""
        parts = self.ex.allgather(self.get_local_vector())
        return np.concatenate(parts)

"""Host logic of the engine on the CPU (tests/engine_host_check.cpp, built
with engine.cpp by the host compiler; no GPU):

* imported stores: chunk headers of stored blocks are checked before any
  upload (misaligned offsets, widths above 32 and payloads past the arena are
  rejected; headers of unstored blocks are never read and are ignored);
* the planner: the QFT's bit-reversal SWAPs between chunk bits and outer
  qubits become code-domain passes while the QFT's own passes carry values,
  and every tile is padded to the largest tile of its precision when the
  block has the qubits for it.
"""
import os
import shutil
import struct
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "compression-based-state-vector-simulator_b200", "csrc")
CUDA = "/usr/local/cuda"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None or not os.path.isdir(os.path.join(CUDA, "include")):
        pytest.skip("no host C++ compiler or CUDA headers")
    exe = tmp_path_factory.mktemp("engine") / "engine_host_check"
    cmd = [gxx, "-O1", "-std=c++17", "-w", "-pthread", "-I", CSRC, "-I", os.path.join(CUDA, "include"),
           "-o", str(exe), os.path.join(HERE, "engine_host_check.cpp"), "-L", os.path.join(CUDA, "lib64"),
           "-lcudart", "-Wl,--unresolved-symbols=ignore-all", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    env = dict(os.environ)
    env.pop("CXX", None)
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    return str(exe)


def test_store_header_check(checker):
    r = subprocess.run([checker, "headers"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "0 failures" in r.stdout, r.stdout + r.stderr


def test_selector_run_encoding(checker):
    """Ops whose selector bits form at most two runs are re-encoded with their
    matrix variants permuted so that the two-shift rule of the device picks
    what the per-bit rule picked; other ops are left as they were."""
    r = subprocess.run([checker, "selruns"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "selruns ok" in r.stdout, r.stdout + r.stderr


def test_pass_planner_order_and_tiles(checker):
    """Both pass planners place every gate once, give each pass a tile that
    holds the qubits its gates mix (at most jmax, padded to jmin) and at most
    the allowed outer selectors, and keep every non-commuting pair of gates
    in order; the reordering planner does move commuting gates."""
    r = subprocess.run([checker, "dagplan"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "dagplan ok" in r.stdout, r.stdout + r.stderr


def test_chunk_permutation_folding(checker):
    """SWAP and X gates on qubits above the chunk bits folded into one chunk
    permutation, the other gates relabelled through it: the relabelled gates
    and then the permutation's chunk moves give the original circuit's state
    (dense vectors of up to 10 qubits, random gates, CNOTs left unfolded)."""
    r = subprocess.run([checker, "chunkperm"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "chunkperm ok" in r.stdout, r.stdout + r.stderr


def test_op_compiler_against_direct_application(checker):
    """Random circuits of dense, diagonal, block-diagonal and permutation
    gates compiled to register ops by the fused path's host steps; the ops,
    interpreted tile by tile by a host restatement of the tile pass, give
    the state of the gates applied one by one (within 1e-9)."""
    r = subprocess.run([checker, "opcompile"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "opcompile ok" in r.stdout, r.stdout + r.stderr


def test_two_store_op_compiler_sums_and_states(checker):
    """The adjoint's two-store passes compiled by plan_dual_sweeps: on random
    unitary circuits with parametric gates (X, Y, Z generators on their own
    qubits), the interpreted ops give every derivative sum
    sum_x conj(lambda[x ^ gx]) (-1)^{|x & gz|} psi[x] just before its gate and
    both final states, at 3 (complex128) and 4 (complex64) register bits."""
    r = subprocess.run([checker, "dualcompile"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "dualcompile ok" in r.stdout, r.stdout + r.stderr


def test_half_diagonal_chain_fusion(checker):
    """Runs of half-diagonals on one register bit fused into pending factors
    and one application give every register group the unfused result, and
    no pending factor outlives its sweep."""
    r = subprocess.run([checker, "halfchains"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "halfchains ok" in r.stdout, r.stdout + r.stderr


def _plan(checker, tmp_path, circuit, n, B, I, f64):
    import ctypes as ct
    from qulacs import _native
    from qulacs.circuit import QuantumCircuitOptimizer
    QuantumCircuitOptimizer(sv_block_size=B).optimize(circuit, block_size=2)
    arr = _native.make_gate_array(circuit._gates)
    path = tmp_path / "gates.bin"
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", len(circuit._gates)))
        f.write(ct.string_at(ct.addressof(arr), ct.sizeof(_native.qs_gate) * len(circuit._gates)))
    r = subprocess.run([checker, "plan", str(path), str(n), str(B), str(I), "1" if f64 else "0"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    passes = []
    for line in r.stdout.splitlines():
        if line.startswith("pass kind"):
            t = line.split()
            passes.append(dict(kind=int(t[2]), j=int(t[4]), codes=int(t[6]), jmax=int(t[8])))
    return passes


@pytest.mark.parametrize("f64", [True, False])
def test_plan_code_domain_and_header_passes(checker, tmp_path, f64):
    from qompsim import circuits as C
    passes = _plan(checker, tmp_path, C.qft_basis(16, 5), 16, 9, 3, f64)
    assert passes
    assert any(p["kind"] == 0 and p["codes"] for p in passes)      # chunk bit <-> outer qubit SWAPs
    assert not all(p["codes"] for p in passes if p["kind"] == 0)   # the QFT's own passes carry values


@pytest.mark.parametrize("f64", [True, False])
def test_plan_tiles_padded_to_largest(checker, tmp_path, f64):
    import helpers
    passes = _plan(checker, tmp_path, helpers.random_circuit(16, 80, seed=3), 16, 14, 3, f64)
    tiles = [p for p in passes if p["kind"] == 0]
    assert tiles
    assert all(p["j"] == p["jmax"] for p in tiles), tiles
    assert tiles[0]["jmax"] == (4 if f64 else 5)


def _tail(checker, tmp_path, circuit, n, B, I, f64):
    import ctypes as ct
    from qulacs import _native
    from qulacs.circuit import QuantumCircuitOptimizer
    QuantumCircuitOptimizer(sv_block_size=B).optimize(circuit, block_size=2)
    arr = _native.make_gate_array(circuit._gates)
    path = tmp_path / "gates.bin"
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", len(circuit._gates)))
        f.write(ct.string_at(ct.addressof(arr), ct.sizeof(_native.qs_gate) * len(circuit._gates)))
    r = subprocess.run([checker, "tail", str(path), str(n), str(B), str(I), "1" if f64 else "0"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = []
    for line in r.stdout.splitlines():
        t = line.split()
        if t and t[0] == "tail":
            out.append(dict(s0=int(t[1]), per_stage=int(t[3]), merged=int(t[5]), ends=[int(x) for x in t[7:]]))
    return out


@pytest.mark.parametrize("f64", [True, False])
def test_merged_tail_plan(checker, tmp_path, f64):
    """Brickwork n=20 (a dense state after its first stages): planned as one
    gate sequence with commuting gates reordered, the stages from any start
    need fewer passes than stage by stage (a third fewer from stage 2 on);
    every stage ends in a tail pass, in order, the last stage in the last
    pass."""
    from qompsim import circuits as C
    tails = _tail(checker, tmp_path, C.brickwork(20, 20, seed=0), 20, 12, 4, f64)
    assert tails
    for t in tails:
        assert 1 <= t["merged"] <= t["per_stage"]
        assert all(b >= a for a, b in zip(t["ends"], t["ends"][1:]))
        assert t["ends"][-1] == t["merged"] - 1
    assert tails[2]["merged"] * 3 < tails[2]["per_stage"] * 2

"""Benchmark of the compressed state-vector stage pipeline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload qft30]

Workload (default): QFT of a seeded random basis state on n=30 qubits,
complex128, block_size B=20, inner_size I=4, BITCOMP_REL_EB 1e-3 /
BITCOMP_ABS_EB 1e-7, fused with QuantumCircuitOptimizer(block_size=2) as
script/run_sim.py does.  One step = apply_circuit over every stage, from the
input state already resident in HBM (reset to |0...0> before each step; the
circuit's X gates prepare the basis input).

Metric: amplitude-gate updates/s = sum_s gates(s) * amplitudes in the active
groups of stage s, per second (the reference processes every amplitude of
every active group for every gate of the stage).  value aggregates all ranks
(N ranks run independent replicas: weak scaling).

Also reported: roofline of the fused pass kernel (compressed bytes read +
written per launch / per-launch device time, against the measured HBM copy
bandwidth), the end-to-end figure through the C ABI with the compressed store
imported from and exported to pinned host memory every step, and the CPU
baseline (the reference's csim FP64 kernels on the host cores).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "compression-based-state-vector-simulator_b200")
for _p in (PKG, ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "amplitude-gate updates/s"
UNIT = "updates/s"


def workload_spec(name: str):
    from qompsim import circuits as C
    spec = dict(C.WORKLOADS[name])
    spec["name"] = name
    return spec


def build_circuit(spec):
    from qulacs.circuit import QuantumCircuitOptimizer
    c = spec["builder"]()
    QuantumCircuitOptimizer(sv_block_size=spec["block_size"]).optimize(c, block_size=2)
    return c


def describe(spec) -> str:
    return (f"{spec['name']}: n={spec['n']} {spec['dtype']} compressed, block_size={spec['block_size']}, "
            f"inner_size={spec['inner_size']}, eps_rel={spec['eps_rel']}, eps_abs={spec['eps_abs']}")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def ncu_traffic_ratio():
    """DRAM bytes / algorithmic bytes of the fused pass, from the committed
    ncu capture (profiles/pass_kernel_traffic.json), if present."""
    p = os.path.join(ROOT, "profiles", "pass_kernel_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["dram_to_algorithmic_ratio"])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        rows = [r.strip().split(",") for r in self.f.read().splitlines() if r.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def barrier(pg, torch):
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()


def max_over_ranks(pg, torch, x: float, device: str = "cuda") -> float:
    """The largest x over all ranks (timings are taken as the max over ranks)."""
    if pg is None:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def aggregate(pg, torch, local_ms: float, updates_per_step: int, steps: int, world: int, device: str = "cuda"):
    """Whole-job figure of N replicas: every rank applied `steps` circuits of
    `updates_per_step` amplitude-gate updates; the job took the slowest
    rank's time.  Returns (ms, updates/s)."""
    ms = max_over_ranks(pg, torch, local_ms, device)
    return ms, world * updates_per_step * steps / (ms * 1e-3)


# ----------------------------------------------------------------- CPU baseline
def cpu_sample(spec, budget_s: float = 12.0):
    """The reference's csim FP64 kernels (oracle/_ref) applying the fused
    gate list uncompressed on the host cores, on a bounded sample: the first
    gates of the same QFT construction on a smaller register (2^ncpu
    amplitudes), timed until ~budget_s.  Returns (updates/s, cores, sample)."""
    import numpy as np
    from oracle import csim_ref
    from qompsim import circuits as C
    from qulacs.circuit import QuantumCircuitOptimizer

    try:
        mem = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES")
    except (ValueError, OSError):
        mem = 0
    ncpu = 28 if mem >= (64 << 30) else 24
    c = C.qft_basis(ncpu, seed=0)
    QuantumCircuitOptimizer(sv_block_size=spec["block_size"]).optimize(c, block_size=2)
    state = csim_ref.zero_state(ncpu)
    t0 = time.perf_counter()
    done = 0
    for g in c._gates:
        csim_ref.apply_gate(state, g)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    rate = done * float(1 << ncpu) / dt
    cores = csim_ref.max_threads()
    sample = (f"csim FP64 uncompressed (reference kernels, OpenMP {cores} threads): first {done} of "
              f"{len(c._gates)} fused gates of QFT n={ncpu} on 2^{ncpu} amplitudes, {dt:.1f} s")
    return rate, cores, sample


def run_reference(args, spec):
    # under torchrun only rank 0 runs the CPU baseline; the others exit at once
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from oracle import csim_ref
    if not csim_ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libcsim_ref.so not built"}))
        return
    for _ in range(args.warmup):
        cpu_sample(spec, budget_s=1.0)
    rates = []
    t0 = time.perf_counter()
    sample = ""
    cores = 1
    for _ in range(args.steps):
        r, cores, sample = cpu_sample(spec, budget_s=max(2.0, 60.0 / max(1, args.steps)))
        rates.append(r)
    wall = time.perf_counter() - t0
    value = statistics.median(rates)
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * wall / max(1, args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": describe(spec)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


# ----------------------------------------------------------------- our arm
def complex64_leg(spec, circuit, updates_per_step, torch, steps: int = 3):
    """The same fused gate list through the complex64 compressed pipeline
    (FP32 gate arithmetic and stored amplitudes, FP64 reductions)."""
    import qulacs
    from qulacs import _native
    cq = qulacs.CompressedQuantumState(spec["n"], spec["block_size"], dtype="complex64", eps_rel=spec["eps_rel"],
                                       eps_abs=spec["eps_abs"], flags=_native.QS_FLAG_QUIET)
    cq.partition_and_register_circuit(circuit, spec["inner_size"], 0)
    for _ in range(3):
        cq.set_computational_basis(0)
        cq.apply_circuit()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        cq.set_computational_basis(0)
        cq.apply_circuit()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    out = {"ms_per_step": ms, "value": updates_per_step / (ms * 1e-3), "unit": UNIT, "steps": steps,
           "max_sv_bytes": cq.get_max_SV_bytes()}
    del cq
    return out


def adjoint_leg(torch, n: int = 24, depth: int = 8, reps: int = 5):
    """Hardware-efficient ansatz n=24, depth 8 (RY RZ per qubit + CNOT ladder,
    384 parameters), H = sum Z_i Z_i+1 + 0.5 sum X_i: wall time of the energy
    alone and of energy + adjoint gradient through the public API, each call
    synchronised; the best of `reps` calls of each (the calls include host
    planning, whose time varies with the host's load)."""
    import qulacs
    from qompsim import circuits as C
    from qulacs.torch import energy, energy_and_gradient
    circ = C.hea(n, depth, seed=0, parametric=True)
    obs = qulacs.Observable(n)
    for coef, pauli, qubits in C.hea_observable_terms(n):
        obs.add_operator(coef, " ".join(f"{p} {q}" for p, q in zip(pauli, qubits)))
    res = {"workload": f"hea: n={n} depth={depth}, {circ.get_parameter_count()} parameters"}
    for dtype in ("complex64", "complex128"):
        energy_and_gradient(circ, obs, dtype)
        energy(circ, obs, dtype)
        torch.cuda.synchronize()

        def best(fn):
            ts = []
            for _ in range(reps):
                t0 = time.perf_counter()
                fn(circ, obs, dtype)
                torch.cuda.synchronize()
                ts.append(time.perf_counter() - t0)
            return min(ts)
        fwd = best(energy)
        grad = best(energy_and_gradient)
        res[dtype] = {"energy_ms": fwd * 1e3, "energy_and_gradient_ms": grad * 1e3, "ratio": grad / fwd}
    return res


def run_ours(args, spec):
    import numpy as np
    import torch

    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    import qulacs
    from qulacs import _native

    circuit = build_circuit(spec)
    flags = _native.QS_FLAG_QUIET | _native.QS_FLAG_PROFILE
    cq = qulacs.CompressedQuantumState(spec["n"], spec["block_size"], dtype=spec["dtype"],
                                       eps_rel=spec["eps_rel"], eps_abs=spec["eps_abs"], flags=flags)
    cq.partition_and_register_circuit(circuit, spec["inner_size"], 0)

    def step():
        cq.set_computational_basis(0)
        cq.apply_circuit()

    for _ in range(max(3, args.warmup)):
        step()
    st = cq.get_stats()
    updates_per_step = int(st["amp_gate_updates"])

    # ---- device-resident timing
    barrier(pg, torch)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pass_ms, pass_bytes, passes = 0.0, 0, 0
    with ClockSampler(local) as clk:
        start.record()
        for _ in range(args.steps):
            step()
            s = cq.get_stats()
            pass_ms += s["kernel_ms"]                         # tile passes (pass_kernel) only
            pass_bytes += int(s["bytes_read"]) + int(s["bytes_written"])
            passes += int(s["passes"]) - int(s["perm_passes"])
        end.record()
        torch.cuda.synchronize()
    ms, value = aggregate(pg, torch, start.elapsed_time(end), updates_per_step, args.steps, world)
    barrier(pg, torch)
    clocks = clk.summary()

    # ---- end to end through the C ABI with host buffers
    cq.set_computational_basis(0)
    blob_in = cq.export_store()
    h_in = torch.frombuffer(bytearray(blob_in), dtype=torch.uint8).pin_memory()
    step()
    out_size = len(cq.export_store())
    h_out = torch.empty(out_size + (1 << 20), dtype=torch.uint8).pin_memory()
    L = _native.lib()
    import ctypes as ct

    def e2e_step():
        _native.check(L.qs_import_store(cq._h, ct.c_void_p(h_in.data_ptr()), len(blob_in)), cq._h)
        cq.apply_circuit()
        sz = ct.c_uint64()
        _native.check(L.qs_export_store(cq._h, ct.c_void_p(h_out.data_ptr()), h_out.numel(), ct.byref(sz)), cq._h)
        return sz.value

    e2e_step()
    barrier(pg, torch)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d2h = 0
    e0.record()
    for _ in range(args.steps):
        d2h = e2e_step()
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(pg, torch, e0.elapsed_time(e1))

    # ---- the plain uncompressed per-gate path on the same gates (rank 0, N=1 only): one kernel per gate
    # over the whole complex128 vector, and this package's fused uncompressed tile passes beside it
    dense = None
    if rank == 0 and world == 1 and not args.no_dense:
        gates = list(circuit._gates)
        ds = qulacs.QuantumState(spec["n"], dtype="complex128")
        legs = {}
        for name, pergate in (("pergate_c128", True), ("fused_dense_c128", False)):
            ds.set_computational_basis(0)
            ds._apply_gates(gates, pergate=pergate)       # warm-up
            torch.cuda.synchronize()
            d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            d0.record()
            ds.set_computational_basis(0)
            ds._apply_gates(gates, pergate=pergate)
            d1.record()
            torch.cuda.synchronize()
            dms = d0.elapsed_time(d1)
            legs[name] = {"ms_per_step": dms, "value": updates_per_step / (dms * 1e-3), "unit": UNIT,
                          "launches_per_step": len(gates) if pergate else None}
        del ds
        dense = legs
        dense["compressed_speedup_vs_pergate_c128"] = legs["pergate_c128"]["ms_per_step"] / (ms / args.steps)

    # ---- the same circuit in the complex64 pipeline, and the adjoint gradient of the
    # hardware-efficient ansatz against its forward pass (rank 0, N=1 only)
    extra = {}
    max_sv = cq.get_max_SV_bytes()
    if rank == 0 and world == 1 and not args.no_legs:
        del cq  # frees the complex128 store's arena for the complex64 state
        extra["complex64"] = complex64_leg(spec, circuit, updates_per_step, torch)
        if dense is not None:
            extra["complex64"]["speedup_vs_pergate_c128"] = (dense["pergate_c128"]["ms_per_step"]
                                                             / extra["complex64"]["ms_per_step"])
        extra["adjoint"] = adjoint_leg(torch)

    # ---- CPU baseline (rank 0, N=1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import csim_ref
        if csim_ref.available():
            rate, cores, sample = cpu_sample(spec)
            cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample}

    if rank == 0:
        peak, peak_kind = measured_peaks()
        achieved = (pass_bytes / max(1, passes)) / (pass_ms / max(1, passes) * 1e-3) / 1e9 if pass_ms > 0 else None
        ratio = ncu_traffic_ratio()
        traffic = ratio * pass_bytes / max(1, passes) if ratio is not None else None
        launches_per_step = int(st["passes"]) + 4 * int(st["stages"]) + 1
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if spec["dtype"] == "complex128" else "f32",
            "data": "synthetic",
            "config": {"workload": describe(spec), "n": spec["n"], "block_size": spec["block_size"],
                       "inner_size": spec["inner_size"], "stages": int(st["stages"]), "passes": int(st["passes"]),
                       "header_only_passes": int(st["perm_passes"]),
                       "gates": circuit.get_gate_count(), "amp_gate_updates_per_step": updates_per_step,
                       "parallelism": f"replicas x{world}",
                       "l2": "compressed store larger than L2 (126 MB); no flush between steps",
                       "max_sv_bytes": max_sv},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6.65 TB/s",
                         "traffic_source": "ncu DRAM/algorithmic ratio of QFT n=26 (profiles/) x bytes per launch",
                         "kernel": f"pass_kernel<{'double' if spec['dtype'] == 'complex128' else 'float'}, 4, *> "
                                   "(value and code-domain tile passes)",
                         "pass_ms_per_step": pass_ms / args.steps,
                         "bytes_per_launch": pass_bytes / max(1, passes)},
            "e2e": {"value": world * updates_per_step * args.steps / (e2e_ms * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": len(blob_in), "d2h_bytes_per_step": int(d2h),
                    "ms_per_step": e2e_ms / args.steps},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "uncompressed": dense,
        }
        out.update(extra)
        print(json.dumps(out))
    if pg is not None:
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="qft30")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-dense", action="store_true", help="skip the uncompressed per-gate comparison leg")
    ap.add_argument("--no-legs", action="store_true", help="skip the complex64 and adjoint-gradient legs")
    args = ap.parse_args()
    spec = workload_spec(args.workload)
    if args.impl == "reference":
        run_reference(args, spec)
    else:
        run_ours(args, spec)


if __name__ == "__main__":
    main()

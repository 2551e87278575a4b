#!/usr/bin/env python
"""Benchmark of the state-vector gate-pass path on B200.

Workload (default): the 30-qubit complex128 brick-wall circuit of depth 40
(U3 on every qubit per layer + CX brick pairs, 1780 gates, seeded), planned by
the library into tile passes.  One step = reset the 16 GiB state to |0...0>
and run the whole circuit.  Inputs (the planned passes and their matrices) are
resident on the device before the timed region; the state (16 GiB) is far
larger than L2 (126 MB), so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value     = gate-pass bytes (2 x 16 B x 2^n per pass, summed over passes and
            ranks) / device time of the K steps (max over ranks), in GB/s.
e2e       = the same metric through the C ABI a reference user calls
            (iq_statevector_reset / apply_1q / apply_2q with host matrices,
            then <Z_i> for every qubit read back), wall clock per step.
roofline  = the tile-pass kernel: 2 x 16 x 2^n bytes per launch / mean launch
            time (CUDA events on the library's stream) against the measured HBM
            copy bandwidth.
cpu_baseline = the reference's own OpenMP core (oracle/_ref, built from the
            reference sources) on this host's cores, on the first gates of the
            same circuit.
With --gpus N > 1 (torchrun) every rank simulates its own replica (the state
vector is not sharded): weak scaling, no collective on the data path.
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
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "30q c128 gate-pass GB/s vs HBM peak; batched adjoint grads/sec vs param-shift"
UNIT = "GB/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--depth", type=int, default=40)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--tile-bits", type=int, default=None)
    ap.add_argument("--chunk-bits", type=int, default=None)
    ap.add_argument("--budget", type=float, default=None)
    ap.add_argument("--max-stages", type=int, default=None)
    ap.add_argument("--nbuf", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-gates", type=int, default=4, help="gates per step of the reference arm")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the batched adjoint-gradient measurement")
    ap.add_argument("--adjoint-circuits", type=int, default=256)
    ap.add_argument("--adjoint-sets", type=int, default=16)
    ap.add_argument("--adjoint-steps", type=int, default=2)
    ap.add_argument("--adjoint-streams", type=int, default=0)
    ap.add_argument("--ps-stride", type=int, default=16,
                    help="parameter-shift baseline on every k-th circuit (one parameter set each)")
    return ap.parse_args()


def pass_bytes(n: int) -> float:
    return 2.0 * 16.0 * float(1 << n)


def circuit_gates(n, depth, seed):
    from invariantq_b200.circuits import brickwall
    c = brickwall(n, depth, seed)
    return [([c.get_qubit_index(q) for q in op.qubits], np.asarray(op.matrix, np.complex128)) for op in c.ops]


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_record(n):
    """DRAM bytes per tile-pass launch from the committed ncu summary
    (profiles/tile_pass_traffic.txt: `qubits Q` and `bytes_per_launch B`),
    scaled to n qubits by the amplitudes per launch."""
    p = REPO / "profiles" / "tile_pass_traffic.txt"
    if not p.exists():
        return None
    try:
        kv = dict(line.split()[:2] for line in p.read_text().splitlines() if line.strip() and not line.startswith("#"))
        q, b = int(kv["qubits"]), float(kv["bytes_per_launch"])
        return b * (2.0 ** (n - q))
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu_id}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def gpu_uuid(dev: int):
    import torch
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(dev)


# ---------------------------------------------------------------- CPU baseline

def cpu_reference_run(gates, n_target, seconds, max_gates=None):
    """Time the reference OpenMP core gate by gate on the first gates of the circuit.
    Returns (gb_per_s, gates_done, qubits, kind, threads)."""
    from oracle.oracle import Port, RefCore
    avail = 0
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable"):
                avail = int(line.split()[1]) * 1024
    except Exception:
        pass
    n = n_target
    while n > 20 and (1 << n) * 16 * 1.3 > avail:
        n -= 1
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    try:
        core = RefCore()
        sv = core.sv(n)
        kind = "reference"
        apply1 = sv.apply_1q
        apply2 = sv.apply_2q
    except FileNotFoundError:
        port = Port()
        st = port.zero_state(n)
        kind, threads = "port", 1
        apply1 = lambda q, U: port.apply_1q(st, n, q, U)  # noqa: E731
        apply2 = lambda a, b, U: port.apply_2q(st, n, a, b, U)  # noqa: E731
    done = 0
    t0 = time.perf_counter()
    for qs, U in gates:
        if max_gates is not None and done >= max_gates:
            break
        (apply1(qs[0], U) if len(qs) == 1 else apply2(qs[0], qs[1], U))
        done += 1
        if max_gates is None and time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return done * pass_bytes(n) / dt / 1e9, done, n, kind, threads, dt


def reference_arm(args, rank):
    if rank != 0:
        return
    gates = circuit_gates(args.qubits, args.depth, args.seed)
    g = args.ref_gates
    times, n_used, kind, threads = [], args.qubits, "reference", 1
    from oracle.oracle import RefCore
    try:
        core = RefCore()
    except FileNotFoundError:
        print(json.dumps({"impl": "reference", "unavailable": "reference core not built (make -C oracle ref)"}))
        return
    # reuse one handle for all steps (create zero-fills the state; not timed)
    avail = 0
    for line in open("/proc/meminfo"):
        if line.startswith("MemAvailable"):
            avail = int(line.split()[1]) * 1024
    n = args.qubits
    while n > 20 and (1 << n) * 16 * 1.3 > avail:
        n -= 1
    n_used = n
    sv = core.sv(n)
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    pos = 0
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for _ in range(g):
            qs, U = gates[pos % len(gates)]
            pos += 1
            (sv.apply_1q(qs[0], U) if len(qs) == 1 else sv.apply_2q(qs[0], qs[1], U))
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = args.steps * g * pass_bytes(n_used) / total / 1e9
    sample = (f"{g} gates per step of the {n_used}-qubit depth-{args.depth} brick-wall through the reference C ABI "
              f"(iq_statevector_apply_1q/2q, OpenMP, {threads} threads); one pass of 2*16*2^n bytes per gate")
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total / args.steps * 1e3, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
           "data": "synthetic: seeded brick-wall U3+CX circuit",
           "config": {"workload": f"statevector {args.qubits}q brick-wall U3+CX depth {args.depth}, complex128",
                      "qubits": n_used, "depth": args.depth, "parallelism": "host OpenMP"},
           "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
           "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


# ------------------------------------------------------- batched adjoint gradients

def gradient_jobs(ncirc, nsets, seed=1234):
    """256 circuits with n ~ U{10..22}, L ~ U{4..12}; per layer RY and RZ on every
    qubit then a CZ ring; 16 parameter sets of angles ~ U[0, 2 pi); H = TFIM,
    h = 1.0, open boundary."""
    from invariantq_b200.gradients import Ansatz, PauliHamiltonian
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(ncirc):
        n = int(rng.integers(10, 23))
        L = int(rng.integers(4, 13))
        a = Ansatz.hardware_efficient(n, L)
        jobs.append((a, PauliHamiltonian.tfim(n, 1.0), rng.uniform(0, 2 * np.pi, (nsets, a.num_params))))
    return jobs


def adjoint_section(args, rank, world):
    """grads/s of the batch API on this rank's share of the circuits (weak:
    circuits split across ranks, no collective on the data path) and the plain
    one-circuit-at-a-time parameter-shift path on a sample of the same circuits."""
    import torch
    from invariantq_b200.gradients import adjoint_gradient_batch, adjoint_stats, parameter_shift_gradient
    jobs = gradient_jobs(args.adjoint_circuits, args.adjoint_sets)
    mine = jobs[rank::world]
    grads = sum(P.shape[0] for _, _, P in mine)
    partials = sum(P.shape[0] * P.shape[1] for _, _, P in mine)
    adjoint_gradient_batch(mine, args.adjoint_streams)            # warm-up (allocations, first plans)
    times = []
    for _ in range(max(args.adjoint_steps, 1)):
        t0 = time.perf_counter()
        out = adjoint_gradient_batch(mine, args.adjoint_streams)
        times.append(time.perf_counter() - t0)
    st = adjoint_stats()
    t = float(np.median(times))
    if world > 1:
        x = torch.tensor([t], dtype=torch.float64, device=f"cuda:{int(os.environ.get('LOCAL_RANK', 0))}")
        torch.distributed.all_reduce(x, op=torch.distributed.ReduceOp.MAX)
        t = float(x.item())
    # parameter-shift baseline on every k-th circuit of this rank (first parameter set)
    ps_t, ps_n, err = 0.0, 0, 0.0
    for i in range(0, len(mine), max(args.ps_stride, 1)):
        a, h, P = mine[i]
        t0 = time.perf_counter()
        g = parameter_shift_gradient(a, h, P[0])
        ps_t += time.perf_counter() - t0
        ps_n += 1
        err = max(err, float(np.max(np.abs(g - out[i][1][0]))))
    ps_rate = ps_n / ps_t
    ns = [a.num_qubits for a, _, _ in mine]
    return {
        "metric": "batched adjoint grads/s", "value": round(world * grads / t, 2), "unit": "gradients/s",
        "partials_per_s": round(world * partials / t, 1), "batch_s": round(t, 4), "steps": len(times),
        "warmup": 1, "gradients": world * grads, "streams": int(st["streams"]),
        "passes": {"forward": int(st["forward_passes"]), "backward": int(st["backward_passes"])},
        "achieved_gbs": round(st["bytes"] / t / 1e9, 1), "host_prep_ms": round(st["host_ms"], 1),
        "workload": f"{args.adjoint_circuits} circuits n~U{{10..22}} (here {min(ns)}..{max(ns)}), L~U{{4..12}}, "
                    f"RY+RZ per qubit + CZ ring per layer, {args.adjoint_sets} parameter sets each, TFIM h=1.0, "
                    "complex128; timed through iq_adjoint_gradient_batch (host parameters in, host gradients out)",
        "param_shift": {"grads_per_s": round(world * ps_rate, 3), "sample": f"{ps_n} circuits (every "
                        f"{args.ps_stride}th, first parameter set), 2P plain forward simulations + energy each",
                        "seconds": round(ps_t, 2)},
        "speedup_vs_param_shift": round((grads / t) / ps_rate, 1),
        "max_abs_diff_vs_param_shift": err,
    }


# ---------------------------------------------------------------- our arm

def our_arm(args, rank, world, local_rank):
    import torch
    from invariantq_b200 import _lib
    from invariantq_b200.binding import NativeStateVector
    from invariantq_b200.simulator import apply_gate_matrix

    dist = world > 1
    lib = _lib.load()
    n = args.qubits
    gates = circuit_gates(n, args.depth, args.seed)
    sv = NativeStateVector(n)
    for key, val in (("tile_bits", args.tile_bits), ("chunk_bits", args.chunk_bits), ("budget", args.budget),
                     ("max_stages", args.max_stages), ("nbuf", args.nbuf)):
        if val is not None:
            sv.set_option(key, val)
    with sv.record() as rec:
        for qs, U in gates:
            apply_gate_matrix(sv, qs, U)
    prog = rec.program
    stream = torch.cuda.ExternalStream(sv.stream(), device=torch.device("cuda", local_rank))

    def step():
        sv.reset()
        prog.run(sv)

    for _ in range(max(args.warmup, 1)):
        step()
    sv.sync()
    sv.set_option("profile", 1)
    sv.profile_read()

    def barrier():
        if dist:
            torch.distributed.barrier()

    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(gpu_uuid(local_rank)) if rank == 0 else None
    time.sleep(0.3 if clocks else 0)
    l0 = lib.iq_kernel_launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    sv.sync()
    e1.synchronize()
    launches = lib.iq_kernel_launches() - l0
    ms = e0.elapsed_time(e1)
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    pass_ms = sv.profile_read()
    sv.set_option("profile", 0)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local_rank}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())

    # e2e through the reference-facing C ABI (host matrices every step, <Z_i> read back)
    e2e = None
    if not args.no_e2e:
        e2e_times, h2d0 = [], sv.stats()["h2d_bytes"]
        for i in range(args.warmup + args.steps):
            if i == args.warmup:
                h2d0 = sv.stats()["h2d_bytes"]
            t0 = time.perf_counter()
            sv.reset()
            for qs, U in gates:
                apply_gate_matrix(sv, qs, U)
            z = sv.expval_z_all()
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                e2e_times.append(dt)
        h2d = (sv.stats()["h2d_bytes"] - h2d0) / args.steps
        e2e_ms = sum(e2e_times) / len(e2e_times) * 1e3
        if dist:
            t = torch.tensor([e2e_ms], dtype=torch.float64, device=f"cuda:{local_rank}")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": round(world * prog.passes * pass_bytes(n) / (e2e_ms / 1e3) / 1e9, 3), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(8 * n + 4),
               "ms_per_step": round(e2e_ms, 3)}
        assert np.all(np.abs(z) <= 1.0 + 1e-9)

    adj = adjoint_section(args, rank, world) if not args.no_adjoint else None
    if rank != 0:
        return
    peak, peak_kind = measured_peaks()
    mean_pass = float(np.mean(pass_ms)) if len(pass_ms) else None
    achieved = pass_bytes(n) / (mean_pass / 1e3) / 1e9 if mean_pass else None
    traffic = traffic_record(n)
    value = world * args.steps * prog.passes * pass_bytes(n) / (ms / 1e3) / 1e9
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic: seeded brick-wall U3+CX circuit (default_rng angles)",
        "config": {"workload": f"statevector {n}q brick-wall U3+CX depth {args.depth} ({len(gates)} gates), "
                               f"complex128, planned into tile passes",
                   "qubits": n, "depth": args.depth, "gates": len(gates), "passes": prog.passes,
                   "gates_per_pass": round(len(gates) / prog.passes, 2),
                   "tile_bits": sv.get_option("tile_bits"), "chunk_bits": sv.get_option("chunk_bits"),
                   "budget": sv.get_option("budget"), "max_stages": sv.get_option("max_stages"),
                   "nbuf": sv.get_option("nbuf"),
                   "l2": "state (16 B x 2^n) larger than the 126 MB L2; no flush between steps",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "circuit_ms": round(ms / args.steps, 3),
        "gates_per_s": round(world * args.steps * len(gates) / (ms / 1e3), 1),
        "passes_per_s": round(world * args.steps * prog.passes / (ms / 1e3), 2),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None, "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4) if achieved else None,
                     "traffic": traffic, "peak_kind": peak_kind, "kernel": "tile_pass_kernel<4>",
                     "per_launch_bytes": pass_bytes(n), "launch_ms": round(mean_pass, 4) if mean_pass else None},
        "gpu_launches": int(launches),
        "e2e": e2e,
        "clocks": clk,
    }
    if adj is not None:
        out["adjoint"] = adj
    if world == 1 and not args.no_cpu_baseline:
        gbs, done, nq, kind, threads, dt = cpu_reference_run(gates, n, args.cpu_seconds)
        out["cpu_baseline"] = {"value": round(gbs, 3), "unit": UNIT, "cores": threads, "kind": kind,
                               "sample": f"first {done} gates of the {nq}-qubit depth-{args.depth} brick-wall, one "
                                         f"pass per gate through the C ABI, {dt:.1f} s"}
    print(json.dumps(out))


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    import torch
    os.environ["IQ_CUDA_DEVICE"] = str(local_rank)
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local_rank))
    try:
        our_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()

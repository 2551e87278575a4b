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
    ap.add_argument("--reg-slots", type=int, default=None, help="register slots R of the tile kernel (3, 4, 5)")
    ap.add_argument("--ctas-per-sm", type=int, default=None, help="resident tile-pass CTAs per SM")
    ap.add_argument("--jit-threads", type=int, default=None, help="CTA size of the specialised kernels")
    ap.add_argument("--jit", type=int, default=None, choices=[0, 1, 2],
                    help="specialised pass kernels: 0 off, 1 library default, 2 always")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-gates", type=int, default=4, help="gates per step of the reference arm")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the batched adjoint-gradient measurement")
    ap.add_argument("--adjoint-circuits", type=int, default=256)
    ap.add_argument("--adjoint-sets", type=int, default=16)
    ap.add_argument("--adjoint-steps", type=int, default=2)
    ap.add_argument("--adjoint-streams", type=int, default=0)
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the 20q, fusion-sweep, density-matrix and 30q-adjoint sections")
    ap.add_argument("--dm-cpu-seconds", type=float, default=10.0)
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

def _omp_set_threads(k):
    """Thread count of the OpenMP team the reference core's kernels use (calls
    from this thread); returns False where libgomp cannot be reached."""
    import ctypes
    try:
        ctypes.CDLL("libgomp.so.1").omp_set_num_threads(int(k))
        return True
    except OSError:
        return False


def cpu_reference_run(gates, n_target, seconds, repeats=5):
    """Time the reference OpenMP core gate by gate on the first gates of the
    circuit: `repeats` samples with all host threads (the gate count per sample
    sized to ~seconds/repeats) and `repeats` one-gate samples on one thread;
    medians of each.  Returns a dict."""
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
    pos = [0]

    def run(count):
        t0 = time.perf_counter()
        for _ in range(count):
            qs, U = gates[pos[0] % len(gates)]
            pos[0] += 1
            (apply1(qs[0], U) if len(qs) == 1 else apply2(qs[0], qs[1], U))
        return time.perf_counter() - t0

    if kind == "reference":
        _omp_set_threads(threads)
    first = run(1)                                          # warm-up gate (first touch, thread start)
    per = max(1, int((seconds / repeats) / max(first, 1e-3)))
    rates = []
    for _ in range(repeats):
        rates.append(per * pass_bytes(n) / run(per) / 1e9)
    out = {"gbs": statistics.median(rates), "n": n, "kind": kind, "threads": threads, "gates_per_sample": per,
           "samples": repeats, "samples_gbs": [round(r, 2) for r in rates]}
    if kind == "reference" and threads > 1 and _omp_set_threads(1):
        one = [pass_bytes(n) / run(1) / 1e9 for _ in range(repeats)]
        _omp_set_threads(threads)
        out["one_thread_gbs"] = statistics.median(one)
        out["one_thread_samples_gbs"] = [round(r, 2) for r in one]
    return out


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
    from invariantq_b200.replicas import max_over_ranks, shard
    import tempfile as _tf
    from invariantq_b200.autotune import AdjointAutotuner, adjoint_settings
    jobs = gradient_jobs(args.adjoint_circuits, args.adjoint_sets)
    mine = shard(jobs, rank, world)
    grads = sum(P.shape[0] for _, _, P in mine)
    partials = sum(P.shape[0] * P.shape[1] for _, _, P in mine)
    # executor settings picked by the project's autotuner on every 16th circuit (not timed; each
    # candidate compiles the kernels of its pass structures, so the search is kept short)
    tuner = AdjointAutotuner(Path(_tf.mkdtemp()) / "autotune.json", stride=16, rounds=1,
                             candidates={"tile_bits": (12,), "chunk_bits": (4, 5), "budget": (160, 200),
                                         "schedule": ((3, 1), (2, 1))})
    t_tune = time.perf_counter()
    choice = tuner.choose(mine)
    tune_s = time.perf_counter() - t_tune
    with adjoint_settings(choice):
        adjoint_gradient_batch(mine, args.adjoint_streams)            # warm-up (allocations, first plans)
        times = []
        for _ in range(max(args.adjoint_steps, 1)):
            t0 = time.perf_counter()
            out = adjoint_gradient_batch(mine, args.adjoint_streams)
            times.append(time.perf_counter() - t0)
        st = adjoint_stats()
    t = max_over_ranks(float(np.median(times)), device=f"cuda:{int(os.environ.get('LOCAL_RANK', 0))}")
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
        "resident_sets": int(st.get("resident_sets", 0)),
        "workload": f"{args.adjoint_circuits} circuits n~U{{10..22}} (here {min(ns)}..{max(ns)}), L~U{{4..12}}, "
                    f"RY+RZ per qubit + CZ ring per layer, {args.adjoint_sets} parameter sets each, TFIM h=1.0, "
                    "complex128; timed through iq_adjoint_gradient_batch (host parameters in, host gradients out)",
        "param_shift": {"grads_per_s": round(world * ps_rate, 3), "sample": f"{ps_n} circuits (every "
                        f"{args.ps_stride}th, first parameter set), 2P plain forward simulations + energy each",
                        "seconds": round(ps_t, 2)},
        "speedup_vs_param_shift": round((grads / t) / ps_rate, 1),
        "max_abs_diff_vs_param_shift": err,
        "settings": {"choice_id": choice["choice_id"], "tile_bits": choice["tile_bits"],
                     "chunk_bits": choice["chunk_bits"], "budget": choice["budget"],
                     "ctas_per_sm": choice["schedule"][0], "nbuf": choice["schedule"][1],
                     "autotune": {"candidates_ms": choice["candidates_ms"], "measured": tuner.measured,
                                  "sample_circuits": choice["sample_jobs"], "tune_s": round(tune_s, 1)}},
    }


# --------------------------------------------------------------- other configs

def cuda_ms(stream, fn, reps=1):
    """Device time of fn() on `stream` (CUDA events), averaged over reps."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def brickwall20_section(args):
    """20-qubit depth-20 brick-wall with every output the workload asks for
    (statevector, 2^20 probabilities, <Z_i>, 8192 shots) through the C ABI,
    wall clock per run; beside it the reference core doing the same on the
    host, and the agreement of the two."""
    from invariantq_b200.binding import NativeStateVector
    from invariantq_b200.simulator import apply_gate_matrix
    from oracle.oracle import RefCore
    n, depth = 20, 20
    gates = circuit_gates(n, depth, args.seed)
    sv = NativeStateVector(n)

    def gpu_run():
        sv.reset()
        for qs, U in gates:
            apply_gate_matrix(sv, qs, U)
        return sv.get_amplitudes(), sv.get_probabilities(), sv.expval_z_all(), sv.sample(8192, seed=7)

    gpu_run()
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        amps, probs, z, shots = gpu_run()
        ts.append(time.perf_counter() - t0)
    sv.close()
    out = {"workload": f"statevector {n}q brick-wall U3+CX depth {depth} ({len(gates)} gates) + all probabilities, "
                       "<Z_i> for every qubit, 8192 shots", "gpu_ms": round(1e3 * float(np.median(ts)), 3)}
    try:
        core = RefCore()
    except FileNotFoundError:
        out["cpu"] = "reference core not built"
        return out
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    ref = core.sv(n)
    t0 = time.perf_counter()
    for qs, U in gates:
        (ref.apply_1q(qs[0], U) if len(qs) == 1 else ref.apply_2q(qs[0], qs[1], U))
    ramps = ref.amplitudes()
    rprobs = ref.probabilities()
    rz = np.array([ref.expval_pauli("Z", [q]).real for q in range(n)])
    rshots = ref.sample(8192, 7)
    cpu_s = time.perf_counter() - t0
    out.update({"cpu_ms": round(cpu_s * 1e3, 1), "cpu_kind": "reference", "cpu_cores": threads,
                "speedup_vs_cpu": round(cpu_s * 1e3 / out["gpu_ms"], 1),
                "max_abs_amp_diff": float(np.max(np.abs(amps - ramps))),
                "max_abs_prob_diff": float(np.max(np.abs(probs - rprobs))),
                "max_abs_z_diff": float(np.max(np.abs(z - rz))),
                "shots_identical_frac": float(np.mean(np.asarray(shots) == np.asarray(rshots)))})
    return out


def fusion_sweep_section(args, sv, n, stream):
    """The 30-qubit circuit through GateFusionPass at k = 2..5: blocks, tile
    passes after planning, passes/s and GB/s (2 x 16 B x 2^n per pass), with
    each block applied as the driver does ('cost': its dense matrix, or its
    original gates where those need less FP64 work per amplitude) and, beside
    it, every block as its dense 2^k x 2^k matrix ('dense')."""
    from invariantq_b200.circuits import brickwall
    from invariantq_b200.fusion import GateFusionPass
    from invariantq_b200.simulator import apply_fused_op, apply_gate_matrix
    c = brickwall(n, args.depth, seed=args.seed)
    out = {}
    for k in (2, 3, 4, 5):
        f = GateFusionPass(k).run(c)
        row = {"blocks": len(f.ops)}
        for policy in ("cost", "dense"):
            how = {"dense": 0, "originals": 0}
            with sv.record() as rec:
                for op in f.ops:
                    qs = [f.get_qubit_index(q) for q in op.qubits]
                    if type(op).__name__ == "FusedGateOp":
                        how[apply_fused_op(sv, f, op, policy)] += 1
                    else:
                        apply_gate_matrix(sv, qs, op.matrix)
            prog = rec.program

            def step():
                sv.reset()
                prog.run(sv)

            step()
            sv.sync()
            ms = cuda_ms(stream, step)
            sv.sync()
            row[policy] = {"fused_blocks_dense": how["dense"], "fused_blocks_as_original_gates": how["originals"],
                           "passes": prog.passes, "circuit_ms": round(ms, 2),
                           "passes_per_s": round(prog.passes / (ms / 1e3), 2),
                           "GBs": round(prog.passes * pass_bytes(n) / (ms / 1e3) / 1e9, 1)}
            del prog
        out[str(k)] = row
    return out


def plan_section(args, sv, n, gates, stream, opts, label):
    """The 30-qubit circuit recorded with other handle options (`opts`),
    timed on the device; its amplitudes' <Z_q> against the headline run's
    (`ref_z`).  Options stay set on the handle, so run it after the headline."""
    from invariantq_b200.simulator import apply_gate_matrix
    for k, v in opts.items():
        sv.set_option(k, v)
    with sv.record() as rec:
        for qs, U in gates:
            apply_gate_matrix(sv, qs, U)
    prog = rec.program

    def step():
        sv.reset()
        prog.run(sv)

    step()
    sv.sync()
    ms = cuda_ms(stream, step)
    sv.sync()
    z = sv.expval_z_all()
    return {"plan": label, "options": opts, "passes": prog.passes, "circuit_ms": round(ms, 2),
            "passes_per_s": round(prog.passes / (ms / 1e3), 2),
            "GBs_per_pass": round(prog.passes * pass_bytes(n) / (ms / 1e3) / 1e9, 1), "z": z}


def autotune_section(args, sv, n, gates, stream, ref_z):
    """The project's autotuner on the 30-qubit circuit (coordinate search over
    tile bits, chunk bits, budget, register slots and CTAs per SM on the
    circuit's first quarter; fusion width fixed at the runtime's own two-qubit
    fusion), then the whole circuit timed with its choice."""
    import tempfile as _tf
    from invariantq_b200.autotune import Autotuner
    from invariantq_b200.circuits import brickwall
    c = brickwall(n, args.depth, seed=args.seed)
    cache = Path(_tf.mkdtemp()) / "autotune.json"
    tuner = Autotuner(cache, candidates={"k": (2,), "tile_bits": (11, 12), "chunk_bits": (3, 4, 5),
                                         "budget": (120, 160, 200), "reg_slots": (4,), "ctas_per_sm": (2, 3, 4)})
    t0 = time.perf_counter()
    ch = tuner.choose(c)
    tune_s = time.perf_counter() - t0
    opts = {k: ch[k] for k in ("tile_bits", "chunk_bits", "budget", "reg_slots", "ctas_per_sm")}
    run = plan_section(args, sv, n, gates, stream, opts, "autotuned")
    z = run.pop("z")
    run.update({"choice_id": ch["choice_id"], "candidates_measured": tuner.measured, "tune_s": round(tune_s, 1),
                "probe_ms": ch["probe_ms"], "candidates_ms": ch["candidates_ms"],
                "max_abs_z_diff_vs_headline": float(np.max(np.abs(z - ref_z)))})
    return run


def density_matrix_section(args):
    """14-qubit noisy brick-wall of depth 12 as a density matrix (4 GiB):
    depolarizing(1e-3) after every U3, amplitude (2e-3) and phase (1e-3)
    damping on both qubits after every CX, thermal relaxation (100 us, 80 us,
    50 ns) on every qubit at each layer end.  Outputs trace, purity,
    <Z_i Z_i+1>.  GPU: the whole circuit as a recorded program, wall clock of
    reset + program + trace readback (best of 2 after a warm-up); CPU: the
    reference core on the first operations of the same circuit."""
    from invariantq_b200.binding import NativeDensityMatrix
    from invariantq_b200.channels import build_kraus_channel
    from invariantq_b200.circuits import noisy_brickwall
    from oracle.oracle import RefCore
    n, depth = 14, 12
    c = noisy_brickwall(n, depth, seed=args.seed)
    dep = build_kraus_channel("depolarizing", [1e-3])
    ops = []
    for op in c.ops:
        qs = [c.get_qubit_index(q) for q in op.qubits]
        if type(op).__name__ == "GateOp":
            if len(qs) == 1:
                ops += [("u1", qs, op.matrix), ("k1", qs, dep)]
            else:
                ops.append(("u2", qs, op.matrix))
        else:
            K = build_kraus_channel(op.channel_name, op.params)
            ops += [("k1", [q], K) for q in qs]

    def apply(target, o):
        kind, qs, m = o
        if kind == "u1":
            target.apply_1q_unitary(qs[0], m)
        elif kind == "u2":
            target.apply_2q_unitary(qs[0], qs[1], m)
        else:
            target.apply_1q_kraus(qs[0], m)

    def apply_ref(target, o):       # the reference core's wrapper names
        kind, qs, m = o
        if kind == "u1":
            target.apply_1q(qs[0], m)
        elif kind == "u2":
            target.apply_2q(qs[0], qs[1], m)
        else:
            target.apply_kraus_1q(qs[0], m)

    dm = NativeDensityMatrix(n)
    with dm.record() as rec:
        for o in ops:
            apply(dm, o)
    prog = rec.program

    def step():
        dm.reset()
        prog.run(dm)
        return dm.trace()            # waits for the stream

    step()
    ts = []
    for _ in range(2):
        t0 = time.perf_counter()
        step()
        ts.append(time.perf_counter() - t0)
    ms = 1e3 * min(ts)
    d = dm.get_diagonal()
    bits = (np.arange(1 << n)[:, None] >> np.arange(n)[None, :]) & 1
    zz = [float((d * (1 - 2 * bits[:, i]) * (1 - 2 * bits[:, i + 1])).sum()) for i in range(n - 1)]
    op_bytes = 2.0 * 16.0 * float(4 ** n)
    out = {"workload": f"density matrix {n}q noisy brick-wall depth {depth} ({len(ops)} unitary / Kraus operations), "
                       "complex128", "ops": len(ops), "passes": prog.passes, "circuit_ms": round(ms, 2),
           "ops_per_s": round(len(ops) / (ms / 1e3), 1),
           "GBs_per_pass": round(prog.passes * op_bytes / (ms / 1e3) / 1e9, 1),
           "trace": dm.trace(), "purity": dm.purity(), "zz_mean": float(np.mean(zz)), "zz_first": zz[:3]}
    del prog
    dm.close()
    try:
        core = RefCore()
    except FileNotFoundError:
        out["cpu"] = "reference core not built"
        return out
    avail = 0
    for line in open("/proc/meminfo"):
        if line.startswith("MemAvailable"):
            avail = int(line.split()[1]) * 1024
    if avail < 3 * 16 * 4 ** n:
        out["cpu"] = "not enough host memory for the 4 GiB reference density matrix and its temporaries"
        return out
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    ref = core.dm(n)
    done, t0 = 0, time.perf_counter()
    for o in ops:
        apply_ref(ref, o)
        done += 1
        if time.perf_counter() - t0 > args.dm_cpu_seconds:
            break
    cpu_s = time.perf_counter() - t0
    rate = done / cpu_s
    out.update({"cpu_ops_per_s": round(rate, 3), "cpu_kind": "reference", "cpu_cores": threads,
                "cpu_sample": f"first {done} operations of the circuit, {cpu_s:.1f} s",
                "cpu_circuit_s_estimate": round(len(ops) / rate, 1),
                "speedup_vs_cpu": round((len(ops) / rate) / (ms / 1e3), 1)})
    return out


def adjoint30_section(args):
    """One 30-qubit adjoint gradient: 16 layers of RY and RZ on every qubit
    plus a CZ ring (960 parameters), TFIM H with h = 0.7, complex128; the
    gradient is checked against the parameter-shift rule on 4 parameters.  The
    same gradient again with complex64 states, and its error against complex128."""
    from invariantq_b200.gradients import Ansatz, PauliHamiltonian, adjoint_gradient, adjoint_stats, ansatz_energies
    from invariantq_b200.gradients import shifted_parameter_sets
    n, L = 30, 16
    a, h = Ansatz.hardware_efficient(n, L), PauliHamiltonian.tfim(n, 0.7)
    rng = np.random.default_rng(30)
    th = rng.uniform(0, 2 * np.pi, a.num_params)
    adjoint_gradient(a, h, th)                     # warm-up: planning, workspace
    times = []
    for _ in range(3):                             # median of 3 timed gradients
        t0 = time.perf_counter()
        e, g = adjoint_gradient(a, h, th)
        times.append(time.perf_counter() - t0)
    t = float(np.median(times))
    st = adjoint_stats()
    idx = rng.choice(a.num_params, 4, replace=False)
    sets = shifted_parameter_sets(th)
    rows = np.concatenate([[2 * j, 2 * j + 1] for j in idx])
    es = ansatz_energies(a, h, sets[rows])
    ps = 0.5 * (es[0::2] - es[1::2])
    from invariantq_b200.gradients import adjoint_gradient_c64, adjoint_release
    adjoint_release()                              # the complex128 workspace
    adjoint_gradient_c64(a, h, th)                 # warm-up: its kernels and workspace
    times32 = []
    for _ in range(3):
        t0 = time.perf_counter()
        e32, g32 = adjoint_gradient_c64(a, h, th)
        times32.append(time.perf_counter() - t0)
    t32 = float(np.median(times32))
    adjoint_release()
    return {"workload": f"{n}q, {L} layers RY+RZ per qubit + CZ ring ({a.num_params} parameters), TFIM h=0.7, complex128; "
                        "state memory: one [psi | lambda] array of 2^(n+1) amplitudes (two state-sized buffers)",
            "gradient_s": round(t, 3), "gradient_s_runs": [round(x, 3) for x in times], "timing": "median of 3 after a warm-up",
            "energy": e, "passes": {"forward": int(st["forward_passes"]),
                                                              "backward": int(st["backward_passes"])},
            "achieved_gbs": round(st["bytes"] / t / 1e9, 1),
            "max_abs_diff_vs_param_shift": float(np.max(np.abs(ps - g[idx]))), "checked_parameters": [int(i) for i in idx],
            "complex64": {"gradient_s": round(t32, 3), "gradient_s_runs": [round(x, 3) for x in times32],
                          "energy_abs_err": abs(e32 - e),
                          "grad_max_abs_err": float(np.max(np.abs(g32 - g))),
                          "grad_rel_err": float(np.max(np.abs(g32 - g)) / max(np.max(np.abs(g)), 1e-300)),
                          "speedup_vs_complex128": round(t / t32, 3),
                          "states": "psi and lambda as complex64 (2 x 8 GiB), FP64 arithmetic and sums"}}


def adjoint32_section(args):
    """One 32-qubit adjoint gradient (4 layers of RY and RZ on every qubit plus
    a CZ ring: 256 parameters; TFIM h = 0.7; complex128): the joint array
    [psi | lambda] of 2^33 amplitudes (128 GiB) is the only state memory.
    Checked against the parameter-shift rule on 2 parameters."""
    import torch
    from invariantq_b200.gradients import Ansatz, PauliHamiltonian, adjoint_gradient, adjoint_release, \
        adjoint_stats, ansatz_energies, shifted_parameter_sets
    free, _ = torch.cuda.mem_get_info()
    if free < 140 * (1 << 30):
        return {"skipped": f"needs ~130 GiB of free device memory ({free / 2**30:.0f} GiB free)"}
    n, L = 32, 4
    a, h = Ansatz.hardware_efficient(n, L), PauliHamiltonian.tfim(n, 0.7)
    rng = np.random.default_rng(32)
    th = rng.uniform(0, 2 * np.pi, a.num_params)
    adjoint_gradient(a, h, th)                     # warm-up: planning, kernels, workspace
    times = []
    for _ in range(3):                             # median of 3 timed gradients
        t0 = time.perf_counter()
        e, g = adjoint_gradient(a, h, th)
        times.append(time.perf_counter() - t0)
    t = float(np.median(times))
    st = adjoint_stats()
    adjoint_release()
    idx = rng.choice(a.num_params, 2, replace=False)
    sets = shifted_parameter_sets(th)
    rows = np.concatenate([[2 * j, 2 * j + 1] for j in idx])
    es = ansatz_energies(a, h, sets[rows])
    ps = 0.5 * (es[0::2] - es[1::2])
    return {"workload": f"{n}q, {L} layers RY+RZ per qubit + CZ ring ({a.num_params} parameters), TFIM h=0.7, "
                        "complex128; state memory: one [psi | lambda] array of 2^33 amplitudes (128 GiB)",
            "gradient_s": round(t, 3), "gradient_s_runs": [round(x, 3) for x in times],
            "timing": "median of 3 after a warm-up", "energy": e,
            "passes": {"forward": int(st["forward_passes"]), "backward": int(st["backward_passes"])},
            "achieved_gbs": round(st["bytes"] / t / 1e9, 1),
            "max_abs_diff_vs_param_shift": float(np.max(np.abs(ps - g[idx]))),
            "checked_parameters": [int(i) for i in idx]}


# ---------------------------------------------------------------- our arm

def our_arm(args, rank, world, local_rank):
    import torch
    from invariantq_b200 import _lib
    from invariantq_b200.binding import NativeStateVector, jit_info, jit_wait
    from invariantq_b200.simulator import apply_gate_matrix
    from invariantq_b200.replicas import max_over_ranks

    dist = world > 1
    lib = _lib.load()
    n = args.qubits
    gates = circuit_gates(n, args.depth, args.seed)
    sv = NativeStateVector(n)
    for key, val in (("tile_bits", args.tile_bits), ("chunk_bits", args.chunk_bits), ("budget", args.budget),
                     ("max_stages", args.max_stages), ("nbuf", args.nbuf), ("reg_slots", args.reg_slots),
                     ("ctas_per_sm", args.ctas_per_sm), ("jit_threads", args.jit_threads), ("jit", args.jit)):
        if val is not None:
            sv.set_option(key, val)
    t_rec = time.perf_counter()
    with sv.record() as rec:
        for qs, U in gates:
            apply_gate_matrix(sv, qs, U)
    prog = rec.program
    record_s = time.perf_counter() - t_rec
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
    j0 = sv.stats()["jit_passes"]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    sv.sync()
    e1.synchronize()
    launches = lib.iq_kernel_launches() - l0
    jit_passes = sv.stats()["jit_passes"] - j0
    ms = e0.elapsed_time(e1)
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    pass_ms = sv.profile_read()
    sv.set_option("profile", 0)
    ref_z = sv.expval_z_all()          # <Z_q> after the last timed step (the whole circuit from |0...0>)
    ms = max_over_ranks(ms, device=f"cuda:{local_rank}")

    # e2e through the reference-facing C ABI (host matrices every step, <Z_i> read back)
    e2e = None
    if not args.no_e2e:
        e2e_times, h2d0 = [], sv.stats()["h2d_bytes"]
        for i in range(args.warmup + args.steps):
            if i == args.warmup:
                # kernels the warm-up flushes queued for compilation finish before timing
                jit_wait(600.0)
                h2d0 = sv.stats()["h2d_bytes"]
                ej0 = sv.stats()["jit_passes"]
            t0 = time.perf_counter()
            sv.reset()
            for qs, U in gates:
                apply_gate_matrix(sv, qs, U)
            z = sv.expval_z_all()
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                e2e_times.append(dt)
        h2d = (sv.stats()["h2d_bytes"] - h2d0) / args.steps
        e2e_jit = (sv.stats()["jit_passes"] - ej0) / args.steps
        e2e_ms = sum(e2e_times) / len(e2e_times) * 1e3
        e2e_ms = max_over_ranks(e2e_ms, device=f"cuda:{local_rank}")
        e2e = {"value": round(world * prog.passes * pass_bytes(n) / (e2e_ms / 1e3) / 1e9, 3), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(8 * n + 4),
               "ms_per_step": round(e2e_ms, 3), "specialised_passes_per_step": e2e_jit,
               "max_abs_z_diff_vs_recorded_program": float(np.max(np.abs(z - ref_z)))}
        assert np.all(np.abs(z) <= 1.0 + 1e-9)

    adj = adjoint_section(args, rank, world) if not args.no_adjoint else None
    opts = {k: sv.get_option(k) for k in ("tile_bits", "chunk_bits", "budget", "max_stages", "nbuf", "reg_slots",
                                          "ctas_per_sm", "jit")}
    configs = None
    if world == 1 and not args.no_configs:
        configs = {"fusion_sweep_30q": fusion_sweep_section(args, sv, n, stream)}
        configs["autotune_30q"] = autotune_section(args, sv, n, gates, stream, ref_z)
        other = plan_section(args, sv, n, gates, stream,
                             {"tile_bits": 11, "chunk_bits": 5, "budget": 120, "ctas_per_sm": 4},
                             "more passes: the interpreting kernel's tile shape (2^11, 5 chunk qubits), budget 120")
        other["max_abs_z_diff_vs_headline"] = float(np.max(np.abs(other.pop("z") - ref_z)))
        configs["plan_comparison_30q"] = other
        configs["brickwall_20q"] = brickwall20_section(args)
        sv.close()
        configs["density_matrix_14q"] = density_matrix_section(args)
        configs["adjoint_30q"] = adjoint30_section(args)
        configs["adjoint_32q"] = adjoint32_section(args)
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
                   **opts,
                   "l2": "state (16 B x 2^n) larger than the 126 MB L2; no flush between steps",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "circuit_ms": round(ms / args.steps, 3),
        "gates_per_s": round(world * args.steps * len(gates) / (ms / 1e3), 1),
        "passes_per_s": round(world * args.steps * prog.passes / (ms / 1e3), 2),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None, "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4) if achieved else None,
                     "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "iq_jit_pass (specialised per pass)" if jit_passes else "tile_pass_kernel<4>",
                     "per_launch_bytes": pass_bytes(n), "launch_ms": round(mean_pass, 4) if mean_pass else None},
        "gpu_launches": int(launches),
        "specialised_passes": int(jit_passes),
        "record_s": round(record_s, 2),
        "jit": jit_info(),
        "e2e": e2e,
        "clocks": clk,
    }
    if adj is not None:
        out["adjoint"] = adj
    if configs is not None:
        out["configs"] = configs
    if world == 1 and not args.no_cpu_baseline:
        cb = cpu_reference_run(gates, n, args.cpu_seconds)
        out["cpu_baseline"] = {
            "value": round(cb["gbs"], 3), "unit": UNIT, "cores": cb["threads"], "kind": cb["kind"],
            "sample": f"median of {cb['samples']} samples of {cb['gates_per_sample']} consecutive gates of the "
                      f"{cb['n']}-qubit depth-{args.depth} brick-wall (from its first gate), one pass per gate "
                      f"through the C ABI, all {cb['threads']} host threads",
            "samples_gbs": cb["samples_gbs"]}
        if "one_thread_gbs" in cb:
            out["cpu_baseline"]["one_core"] = {"value": round(cb["one_thread_gbs"], 3), "unit": UNIT, "cores": 1,
                                               "sample": f"median of {cb['samples']} single-gate samples, 1 thread",
                                               "samples_gbs": cb["one_thread_samples_gbs"]}
    print(json.dumps(out))


def main():
    from invariantq_b200.replicas import env_ranks
    args = parse()
    rank, world, local_rank = env_ranks()
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

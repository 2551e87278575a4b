"""Autotuner for the state-vector path: picks the fusion width k of
``GateFusionPass`` and the tile-pass settings -- tile bits M, chunk bits c (the
contiguous low qubits every tile holds), arithmetic budget per pass, register
slots, and the block-to-CTA schedule (resident CTAs per SM) -- for a circuit,
and records its choice.

A choice is measured once per circuit structure and GPU: candidates run the
circuit's first gates (``probe_fraction`` of them, at least one) as a recorded
program on a state of the circuit's own size, the fastest wins, and the result
-- winner, its choice ID and every candidate's time -- is written to a JSON
cache (``IQ_AUTOTUNE_CACHE``, default ``~/.cache/invariantq_b200/autotune.json``).
Later calls with the same key read the cache.  The key hashes the number of
qubits, the gate names and wires (not the angles: the settings depend on
structure) and the GPU name.

Search: ``"grid"`` times every combination of the candidate values;
``"coordinate"`` (the default: the full space has hundreds of points) starts
from ``start`` and sweeps one setting at a time with the others at the best
values found so far, for up to ``rounds`` rounds or until a round finds
nothing faster.  A candidate the library rejects is recorded as infinite.

k = 2 leaves two-qubit fusion to the runtime (it folds one-qubit gates into
the two-qubit gate between them); k >= 3 runs ``GateFusionPass`` first, its
blocks applied as the driver applies them (dense, or as their original gates
where those cost less).
"""
from __future__ import annotations

import hashlib
import itertools
import json
import os
import time
from pathlib import Path
from typing import Callable, Dict, Iterable, List, Optional, Tuple

import numpy as np

from .fusion import GateFusionPass
from .ir import CircuitIR, op_kind

SETTINGS = ("k", "tile_bits", "chunk_bits", "budget", "reg_slots", "ctas_per_sm")
# handle options a choice sets (k is applied by fusing before recording)
HANDLE_OPTIONS = ("tile_bits", "chunk_bits", "budget", "reg_slots", "ctas_per_sm")
DEFAULT_START = {"k": 2, "tile_bits": 12, "chunk_bits": 4, "budget": 160, "reg_slots": 4, "ctas_per_sm": 3}
DEFAULT_CANDIDATES = {"k": (2, 3, 4), "tile_bits": (11, 12), "chunk_bits": (3, 4, 5), "budget": (120, 160, 200),
                      "reg_slots": (4,), "ctas_per_sm": (2, 3, 4)}


def default_cache_path() -> Path:
    p = os.environ.get("IQ_AUTOTUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "invariantq_b200" / "autotune.json"


def choice_id(c: Dict) -> str:
    return (f"k{c['k']}-m{c['tile_bits']}-c{c['chunk_bits']}-b{int(c['budget'])}-r{c['reg_slots']}"
            f"-a{c['ctas_per_sm']}")


def circuit_key(circuit, device: str) -> str:
    h = hashlib.sha1()
    h.update(f"{circuit.num_qubits}|{device}".encode())
    for op in circuit.ops:
        kind = op_kind(op)
        wires = ",".join(str(circuit.get_qubit_index(q)) for q in op.qubits)
        h.update(f"|{kind}:{getattr(op, 'name', '')}:{wires}".encode())
    return h.hexdigest()[:24]


def device_name() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name()
    except Exception:
        pass
    return "cuda"


def prefix(circuit, fraction: float) -> CircuitIR:
    """The circuit cut after its first `fraction` of gate operations."""
    gates = [op for op in circuit.ops if op_kind(op) in ("GateOp", "FusedGateOp")]
    keep = max(1, int(round(len(gates) * fraction)))
    out = CircuitIR(getattr(circuit, "name", "circuit") + "_probe")
    for name, size in circuit.qubit_regs.items():
        out.add_qubit_register(name, size)
    for op in gates[:keep]:
        out.ops.append(op)
    return out


def apply_circuit(sv, circuit) -> None:
    from .simulator import apply_fused_op, apply_gate_matrix
    for op in circuit.ops:
        kind = op_kind(op)
        qs = [circuit.get_qubit_index(q) for q in op.qubits]
        if kind == "FusedGateOp":
            apply_fused_op(sv, circuit, op)
        elif kind == "GateOp":
            apply_gate_matrix(sv, qs, np.asarray(op.matrix, np.complex128))


def time_candidate(circuit, cand: Dict, reps: int = 2) -> float:
    """Milliseconds per run of `circuit` as a recorded program with settings `cand`."""
    from .binding import NativeStateVector
    c = GateFusionPass(cand["k"]).run(circuit) if cand["k"] > 2 else circuit
    sv = NativeStateVector(circuit.num_qubits)
    try:
        for key in HANDLE_OPTIONS:
            sv.set_option(key, cand[key])
        with sv.record() as rec:
            apply_circuit(sv, c)
        prog = rec.program
        sv.reset()
        prog.run(sv)
        sv.sync()
        t0 = time.perf_counter()
        for _ in range(reps):
            sv.reset()
            prog.run(sv)
        sv.sync()
        return (time.perf_counter() - t0) * 1e3 / reps
    finally:
        sv.close()


class Autotuner:
    """``choose(circuit)`` returns the recorded or newly measured best settings."""

    def __init__(self, cache_path: Optional[os.PathLike] = None, candidates: Optional[Dict[str, Iterable]] = None,
                 probe_fraction: float = 0.25, timer: Optional[Callable[[CircuitIR, Dict], float]] = None,
                 search: str = "coordinate", start: Optional[Dict] = None, rounds: int = 2):
        if search not in ("grid", "coordinate"):
            raise ValueError("search must be 'grid' or 'coordinate'")
        self.cache_path = Path(cache_path) if cache_path else default_cache_path()
        self.start = dict(DEFAULT_START, **(start or {}))
        cands = {k: tuple(v) for k, v in (candidates or DEFAULT_CANDIDATES).items()}
        # a setting without candidates keeps its start value
        self.candidates = {k: cands.get(k, (self.start[k],)) for k in SETTINGS}
        for k in SETTINGS:
            if self.start[k] not in self.candidates[k]:
                self.start[k] = self.candidates[k][0]
        self.probe_fraction = float(probe_fraction)
        self.timer = timer or time_candidate
        self.search = search
        self.rounds = int(rounds)
        self.measured = 0          # candidates timed by this instance

    def _load(self) -> Dict:
        try:
            return json.loads(self.cache_path.read_text())
        except (OSError, ValueError):
            return {}

    def _store(self, key: str, entry: Dict) -> None:
        data = self._load()
        data[key] = entry
        self.cache_path.parent.mkdir(parents=True, exist_ok=True)
        tmp = self.cache_path.with_suffix(self.cache_path.suffix + f".{os.getpid()}.tmp")
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        os.replace(tmp, self.cache_path)

    def grid(self) -> List[Dict]:
        return [dict(zip(SETTINGS, vals)) for vals in itertools.product(*(self.candidates[n] for n in SETTINGS))]

    def _measure(self, probe, cand: Dict, times: Dict) -> float:
        cid = choice_id(cand)
        if cid not in times:
            try:
                ms = float(self.timer(probe, cand))
            except (ValueError, RuntimeError, MemoryError):
                ms = float("inf")      # a combination the library rejects
            self.measured += 1
            times[cid] = round(ms, 4) if ms != float("inf") else None
        v = times[cid]
        return float("inf") if v is None else v

    def _search(self, probe, times: Dict) -> Dict:
        if self.search == "grid":
            best, best_ms = None, float("inf")
            for cand in self.grid():
                ms = self._measure(probe, cand, times)
                if best is None or ms < best_ms:
                    best, best_ms = cand, ms
            return best
        best = dict(self.start)
        best_ms = self._measure(probe, best, times)
        for _ in range(max(self.rounds, 1)):
            improved = False
            for name in SETTINGS:
                for v in self.candidates[name]:
                    cand = dict(best, **{name: v})
                    ms = self._measure(probe, cand, times)
                    if ms < best_ms:
                        best, best_ms, improved = cand, ms, True
            if not improved:
                break
        return best

    def choose(self, circuit, device: Optional[str] = None) -> Dict:
        device = device or device_name()
        key = circuit_key(circuit, device)
        hit = self._load().get(key)
        if hit is not None:
            return dict(hit, cached=True)
        probe = prefix(circuit, self.probe_fraction)
        times: Dict[str, Optional[float]] = {}
        best = self._search(probe, times)
        best_ms = times[choice_id(best)]
        entry = dict(best, choice_id=choice_id(best), probe_ms=best_ms, candidates_ms=times, search=self.search,
                     probe_gates=sum(1 for op in probe.ops), num_qubits=circuit.num_qubits, device=device,
                     measured_at=time.strftime("%Y-%m-%dT%H:%M:%S"))
        self._store(key, entry)
        return dict(entry, cached=False)


# ------------------------------------------------------------------ adjoint

ADJOINT_SETTINGS = ("tile_bits", "chunk_bits", "budget", "schedule")
# schedule = (resident CTAs per SM, tile buffers per CTA)
ADJOINT_START = {"tile_bits": 12, "chunk_bits": 4, "budget": 200, "schedule": (3, 1)}
ADJOINT_CANDIDATES = {"tile_bits": (11, 12), "chunk_bits": (3, 4, 5), "budget": (120, 160, 200),
                      "schedule": ((3, 1), (2, 1), (4, 1), (2, 3))}


def adjoint_env(choice: Dict) -> Dict[str, str]:
    """The executor settings of a choice, as the environment variables
    iq_adjoint_gradient_batch reads at each call."""
    ctas, nbuf = choice["schedule"]
    return {"IQ_TILE_BITS": str(int(choice["tile_bits"])), "IQ_CHUNK_BITS": str(int(choice["chunk_bits"])),
            "IQ_ADJOINT_BUDGET": str(float(choice["budget"])), "IQ_CTAS_PER_SM": str(int(ctas)),
            "IQ_NBUF": str(int(nbuf))}


class adjoint_settings:
    """Context manager: the adjoint executor runs with a choice's settings."""

    def __init__(self, choice: Optional[Dict]):
        self.env = adjoint_env(choice) if choice else {}
        self.saved: Dict[str, Optional[str]] = {}

    def __enter__(self):
        for k, v in self.env.items():
            self.saved[k] = os.environ.get(k)
            os.environ[k] = v
        return self

    def __exit__(self, *exc):
        for k, v in self.saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
        return False


def adjoint_choice_id(c: Dict) -> str:
    return f"m{c['tile_bits']}-c{c['chunk_bits']}-b{int(c['budget'])}-a{c['schedule'][0]}x{c['schedule'][1]}"


def time_adjoint_candidate(jobs, cand: Dict, reps: int = 1) -> float:
    """Milliseconds per adjoint_gradient_batch(jobs) with settings `cand` (after
    one untimed call that plans the circuits and compiles their kernels)."""
    from .gradients import adjoint_gradient_batch
    with adjoint_settings(cand):
        adjoint_gradient_batch(jobs)
        t0 = time.perf_counter()
        for _ in range(reps):
            adjoint_gradient_batch(jobs)
        return (time.perf_counter() - t0) * 1e3 / reps


def jobs_key(jobs, device: str) -> str:
    h = hashlib.sha1()
    h.update(f"adjoint|{device}".encode())
    for a, ham, params in jobs:
        h.update(f"|{a.num_qubits}:{len(a)}:{np.asarray(params).shape[0]}:{len(ham.coeffs)}".encode())
        h.update(np.asarray(a.kinds).tobytes() + np.asarray(a.q0).tobytes() + np.asarray(a.q1).tobytes())
    return h.hexdigest()[:24]


class AdjointAutotuner:
    """Picks the adjoint executor's tile bits, chunk bits, pass budget and
    CTA schedule for a batch of gradient jobs by coordinate search on a sample
    of the jobs (every ``stride``-th), and records the choice in the same cache
    file as ``Autotuner``."""

    def __init__(self, cache_path: Optional[os.PathLike] = None, candidates: Optional[Dict[str, Iterable]] = None,
                 stride: int = 8, timer: Optional[Callable] = None, start: Optional[Dict] = None, rounds: int = 2):
        self.cache_path = Path(cache_path) if cache_path else default_cache_path()
        self.start = dict(ADJOINT_START, **(start or {}))
        cands = {k: tuple(v) for k, v in (candidates or ADJOINT_CANDIDATES).items()}
        self.candidates = {k: cands.get(k, (self.start[k],)) for k in ADJOINT_SETTINGS}
        for k in ADJOINT_SETTINGS:
            if self.start[k] not in self.candidates[k]:
                self.start[k] = self.candidates[k][0]
        self.stride = max(1, int(stride))
        self.timer = timer or time_adjoint_candidate
        self.rounds = int(rounds)
        self.measured = 0

    def choose(self, jobs, device: Optional[str] = None) -> Dict:
        device = device or device_name()
        sample = list(jobs)[::self.stride]
        key = jobs_key(sample, device)
        store = Autotuner(self.cache_path)
        hit = store._load().get(key)
        if hit is not None:
            hit = dict(hit)
            hit["schedule"] = tuple(hit["schedule"])
            return dict(hit, cached=True)
        times: Dict[str, Optional[float]] = {}

        def measure(cand):
            cid = adjoint_choice_id(cand)
            if cid not in times:
                try:
                    if not times:
                        # the process's first batches also grow the workers' buffers to
                        # their sizes: one more untimed run, so the first candidate is not
                        # charged for it
                        self.timer(sample, cand)
                    ms = float(self.timer(sample, cand))
                except (ValueError, RuntimeError, MemoryError):
                    ms = float("inf")
                self.measured += 1
                times[cid] = round(ms, 4) if ms != float("inf") else None
            v = times[cid]
            return float("inf") if v is None else v

        best = dict(self.start)
        best_ms = measure(best)
        for _ in range(max(self.rounds, 1)):
            improved = False
            for name in ADJOINT_SETTINGS:
                for v in self.candidates[name]:
                    cand = dict(best, **{name: v})
                    ms = measure(cand)
                    if ms < best_ms:
                        best, best_ms, improved = cand, ms, True
            if not improved:
                break
        entry = dict(best, schedule=list(best["schedule"]), choice_id=adjoint_choice_id(best), probe_ms=best_ms,
                     candidates_ms=times, sample_jobs=len(sample), device=device,
                     measured_at=time.strftime("%Y-%m-%dT%H:%M:%S"))
        store._store(key, entry)
        return dict(entry, schedule=tuple(best["schedule"]), cached=False)

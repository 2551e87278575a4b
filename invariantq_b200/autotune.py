"""Autotuner for the state-vector path: picks the fusion width k of
``GateFusionPass`` and the tile-pass settings (tile bits, arithmetic budget per
pass, register slots) for a circuit, and records its choice.

A choice is measured once per circuit structure and GPU: every candidate runs
the circuit's first gates (``probe_fraction`` of them, at least one) as a
recorded program on a state of the circuit's own size, the fastest wins, and
the result -- winner, its choice ID and every candidate's time -- is written to
a JSON cache (``IQ_AUTOTUNE_CACHE``, default
``~/.cache/invariantq_b200/autotune.json``).  Later calls with the same key
read the cache.  The key hashes the number of qubits, the gate names and
wires (not the angles: the settings depend on structure) and the GPU name.

k = 2 leaves two-qubit fusion to the runtime (it folds one-qubit gates into
the two-qubit gate between them); k >= 3 runs ``GateFusionPass`` first.
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

DEFAULT_CANDIDATES = {"k": (2, 3, 4), "tile_bits": (11, 12), "budget": (80, 120, 160), "reg_slots": (4,)}


def default_cache_path() -> Path:
    p = os.environ.get("IQ_AUTOTUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "invariantq_b200" / "autotune.json"


def choice_id(c: Dict) -> str:
    return f"k{c['k']}-m{c['tile_bits']}-b{int(c['budget'])}-r{c['reg_slots']}"


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
    from .simulator import apply_gate_matrix
    for op in circuit.ops:
        kind = op_kind(op)
        qs = [circuit.get_qubit_index(q) for q in op.qubits]
        if kind == "FusedGateOp":
            sv.apply_fused(qs, op.fused_matrix)
        elif kind == "GateOp":
            apply_gate_matrix(sv, qs, np.asarray(op.matrix, np.complex128))


def time_candidate(circuit, cand: Dict, reps: int = 2) -> float:
    """Milliseconds per run of `circuit` as a recorded program with settings `cand`."""
    from .binding import NativeStateVector
    c = GateFusionPass(cand["k"]).run(circuit) if cand["k"] > 2 else circuit
    sv = NativeStateVector(circuit.num_qubits)
    try:
        for key in ("tile_bits", "budget", "reg_slots"):
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
                 probe_fraction: float = 0.25, timer: Optional[Callable[[CircuitIR, Dict], float]] = None):
        self.cache_path = Path(cache_path) if cache_path else default_cache_path()
        self.candidates = {k: tuple(v) for k, v in (candidates or DEFAULT_CANDIDATES).items()}
        self.probe_fraction = float(probe_fraction)
        self.timer = timer or time_candidate
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
        names = ("k", "tile_bits", "budget", "reg_slots")
        return [dict(zip(names, vals)) for vals in itertools.product(*(self.candidates[n] for n in names))]

    def choose(self, circuit, device: Optional[str] = None) -> Dict:
        device = device or device_name()
        key = circuit_key(circuit, device)
        hit = self._load().get(key)
        if hit is not None:
            return dict(hit, cached=True)
        probe = prefix(circuit, self.probe_fraction)
        times = {}
        best, best_ms = None, float("inf")
        for cand in self.grid():
            ms = float(self.timer(probe, cand))
            self.measured += 1
            times[choice_id(cand)] = round(ms, 4)
            if ms < best_ms:
                best, best_ms = cand, ms
        entry = dict(best, choice_id=choice_id(best), probe_ms=round(best_ms, 4), candidates_ms=times,
                     probe_gates=sum(1 for op in probe.ops), num_qubits=circuit.num_qubits, device=device,
                     measured_at=time.strftime("%Y-%m-%dT%H:%M:%S"))
        self._store(key, entry)
        return dict(entry, cached=False)

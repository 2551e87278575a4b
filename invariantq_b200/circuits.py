"""Seeded synthetic workloads (no public dataset is involved).

* ``brickwall``   -- the U3 + CX brick-wall circuit: per layer U3(theta, phi,
  lambda) on every qubit, angles i.i.d. U[0, 2 pi) drawn in (layer, qubit,
  [theta, phi, lambda]) order from ``np.random.default_rng(seed)`` (the
  generator pattern of invariantq/benchmarks/suite.py:41-59), then CX on
  (0,1),(2,3),... in even layers and (1,2),(3,4),... in odd layers, control
  first.  20 qubits / depth 20 = 590 gates; 30 qubits / depth 40 = 1780 gates.
* ``noisy_brickwall`` -- the same with depolarizing(p) after every U3 (as a
  per-gate noise model), amplitude (2e-3) and phase (1e-3) damping on both
  qubits after every CX, and thermal relaxation (T1, T2, t_gate) on every qubit
  at the end of each layer.
* ``tfim_ansatz`` -- RY then RZ on every qubit per layer, then a CZ ring
  (i, i+1 mod n); the transverse-field Ising Hamiltonian
  H = -sum_{i<n-1} Z_i Z_{i+1} - h sum_i X_i (open boundary).
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from .ir import CircuitIR, GateOp, NoiseOp, QWire


def brickwall_angles(n: int, depth: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 2.0 * np.pi, size=(depth, n, 3))


def brickwall(n: int, depth: int, seed: int = 0) -> CircuitIR:
    ang = brickwall_angles(n, depth, seed)
    c = CircuitIR(name=f"brickwall_{n}q_d{depth}")
    c.add_qubit_register("q", n)
    c.add_clbit_register("c", n)
    for layer in range(depth):
        for q in range(n):
            c.add_op(GateOp(name="u3", qubits=[QWire("q", q)], params=[float(a) for a in ang[layer, q]]))
        for q in range(layer % 2, n - 1, 2):
            c.add_op(GateOp(name="cx", qubits=[QWire("q", q), QWire("q", q + 1)]))
    return c


def noisy_brickwall(n: int, depth: int, seed: int = 0, amp: float = 2e-3, phase: float = 1e-3,
                    thermal=(100e-6, 80e-6, 50e-9), angles=None) -> CircuitIR:
    ang = brickwall_angles(n, depth, seed) if angles is None else angles
    c = CircuitIR(name=f"noisy_brickwall_{n}q_d{depth}")
    c.add_qubit_register("q", n)
    for layer in range(depth):
        for q in range(n):
            c.add_op(GateOp(name="u3", qubits=[QWire("q", q)], params=[float(a) for a in ang[layer, q]]))
        for q in range(layer % 2, n - 1, 2):
            pair = [QWire("q", q), QWire("q", q + 1)]
            c.add_op(GateOp(name="cx", qubits=list(pair)))
            c.add_op(NoiseOp(qubits=list(pair), channel_name="amp_damping", params=[amp]))
            c.add_op(NoiseOp(qubits=list(pair), channel_name="phase_damping", params=[phase]))
        c.add_op(NoiseOp(qubits=[QWire("q", q) for q in range(n)], channel_name="thermal_relaxation",
                         params=list(thermal)))
    return c


def tfim_ansatz_ops(n: int, layers: int) -> List[Tuple[str, Tuple[int, ...], int]]:
    """(gate, qubits, parameter index or -1) for the RY/RZ + CZ-ring ansatz."""
    ops = []
    p = 0
    for _ in range(layers):
        for q in range(n):
            ops.append(("ry", (q,), p))
            p += 1
        for q in range(n):
            ops.append(("rz", (q,), p))
            p += 1
        if n > 1:
            for q in range(n if n > 2 else 1):
                ops.append(("cz", (q, (q + 1) % n), -1))
    return ops


def tfim_terms(n: int, h: float = 1.0) -> Tuple[np.ndarray, List[str]]:
    """Coefficients and n-character Pauli strings (character q acts on qubit q)."""
    coeffs, strs = [], []
    for i in range(n - 1):
        s = ["I"] * n
        s[i] = s[i + 1] = "Z"
        coeffs.append(-1.0)
        strs.append("".join(s))
    for i in range(n):
        s = ["I"] * n
        s[i] = "X"
        coeffs.append(-h)
        strs.append("".join(s))
    return np.array(coeffs), strs

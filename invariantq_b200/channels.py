"""Kraus sets of the CPTP noise channels, following the reference's
``build_kraus_channel`` (invariantq/noise/channels.py:11-103) and
``compute_choi_matrix`` (channels.py:116-134).  Pinned against the reference by
tests/golden/gates.npz."""
from __future__ import annotations

import math
from typing import List, Sequence

import numpy as np

_I = np.eye(2, dtype=np.complex128)
_X = np.array([[0, 1], [1, 0]], dtype=np.complex128)
_Y = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
_Z = np.array([[1, 0], [0, -1]], dtype=np.complex128)


def _clip01(p: float) -> float:
    return min(1.0, max(0.0, p))


def build_kraus_channel(name: str, params: Sequence[float]) -> List[np.ndarray]:
    """Kraus operators {K_k} with sum_k K_k^dagger K_k = I (channels.py:11-103)."""
    name = name.lower()
    params = list(params)
    p = params[0] if params else 0.0
    if name in ("depolarizing", "depol"):
        pv = _clip01(p)
        return [math.sqrt(max(0.0, 1.0 - 0.75 * pv)) * _I, math.sqrt(pv / 4.0) * _X,
                math.sqrt(pv / 4.0) * _Y, math.sqrt(pv / 4.0) * _Z]
    if name in ("amplitude_damping", "amp_damping", "t1"):
        g = _clip01(p)
        return [np.array([[1.0, 0.0], [0.0, math.sqrt(1.0 - g)]], dtype=np.complex128),
                np.array([[0.0, math.sqrt(g)], [0.0, 0.0]], dtype=np.complex128)]
    if name in ("phase_damping", "dephasing", "t2"):
        lam = _clip01(p)
        return [np.array([[1.0, 0.0], [0.0, math.sqrt(1.0 - lam)]], dtype=np.complex128),
                np.array([[0.0, 0.0], [0.0, math.sqrt(lam)]], dtype=np.complex128)]
    if name in ("bit_flip", "bitflip"):
        pv = _clip01(p)
        return [math.sqrt(1.0 - pv) * _I, math.sqrt(pv) * _X]
    if name in ("phase_flip", "phaseflip"):
        pv = _clip01(p)
        return [math.sqrt(1.0 - pv) * _I, math.sqrt(pv) * _Z]
    if name in ("thermal_relaxation", "thermal"):
        t1 = params[0] if len(params) > 0 else 50e-6
        t2 = params[1] if len(params) > 1 else 70e-6
        tg = params[2] if len(params) > 2 else 50e-9
        t2 = min(t2, 2.0 * t1)
        gamma = 1.0 - math.exp(-tg / t1) if t1 > 0 else 0.0
        inv_tphi = (1.0 / t2) - (1.0 / (2.0 * t1)) if (t1 > 0 and t2 > 0) else 0.0
        lam = 1.0 - math.exp(-tg * max(0.0, inv_tphi))
        ka = build_kraus_channel("amp_damping", [gamma])
        kp = build_kraus_channel("phase_damping", [lam])
        return [b @ a for b in kp for a in ka]
    if name in ("depolarizing_2q", "depol_2q"):
        pv = _clip01(p)
        paulis = [_I, _X, _Y, _Z]
        ops = []
        for i in range(4):
            for j in range(4):
                w = math.sqrt(max(0.0, 1.0 - (15.0 / 16.0) * pv)) if (i == 0 and j == 0) else math.sqrt(pv / 16.0)
                ops.append(w * np.kron(paulis[i], paulis[j]))
        return ops
    return [np.eye(2, dtype=np.complex128)]


def depolarizing_2q(p: float) -> List[np.ndarray]:
    return build_kraus_channel("depolarizing_2q", [p])


def thermal_relaxation(t1: float, t2: float, gate_time: float) -> List[np.ndarray]:
    return build_kraus_channel("thermal_relaxation", [t1, t2, gate_time])


def compute_choi_matrix(kraus_ops: List[np.ndarray], dim: int = 2) -> np.ndarray:
    """J(E) = sum_k (I (x) K_k) |Phi+><Phi+| (I (x) K_k)^dagger (channels.py:116-134)."""
    phi = np.zeros(dim * dim, dtype=np.complex128)
    for i in range(dim):
        phi[i * dim + i] = 1.0 / math.sqrt(dim)
    proj = np.outer(phi, phi.conj())
    eye = np.eye(dim, dtype=np.complex128)
    choi = np.zeros((dim * dim, dim * dim), dtype=np.complex128)
    for k in kraus_ops:
        op = np.kron(eye, k)
        choi += op @ proj @ op.conj().T
    return choi


def superoperator(kraus_ops: List[np.ndarray]) -> np.ndarray:
    """S = sum_k K_k (x) conj(K_k): vec_row(K rho K^dagger) = S vec_row(rho)."""
    return sum(np.kron(k, k.conj()) for k in kraus_ops)

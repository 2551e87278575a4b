"""Gate matrices, following the reference's single source of gate matrices
(``GateOp._compute_matrix``, invariantq/ir/qir.py:67-208).

Multi-qubit matrices use the reference IR convention: the first listed wire is
the most significant bit of the local index (so ``cx`` on [c, t] has the
control first).  Pinned against the reference by tests/golden/gates.npz.
"""
from __future__ import annotations

import math
from typing import Sequence

import numpy as np

_S2 = 1.0 / math.sqrt(2.0)

TWO_QUBIT = {"cx", "cnot", "cy", "cz", "ch", "iswap", "crx", "cry", "crz", "cp", "cphase", "swap"}
THREE_QUBIT = {"ccx", "toffoli", "cswap", "fredkin"}
PARAMETRIC = {"rx": 1, "ry": 1, "rz": 1, "p": 1, "phase": 1, "u3": 3, "crx": 1, "cry": 1, "crz": 1, "cp": 1,
              "cphase": 1}


def gate_arity(name: str) -> int:
    name = name.lower()
    if name in TWO_QUBIT:
        return 2
    if name in THREE_QUBIT:
        return 3
    return 1


def _ctrl(u: np.ndarray) -> np.ndarray:
    m = np.eye(4, dtype=np.complex128)
    m[2:, 2:] = u
    return m


def gate_matrix(name: str, params: Sequence[float] = (), nqubits: int | None = None) -> np.ndarray:
    """Matrix of gate ``name`` (qir.py:67-208); unknown names give the identity
    on ``nqubits`` wires (qir.py:208)."""
    n = name.lower()
    p = [float(x) for x in params]
    if n in ("i", "id"):
        return np.eye(2, dtype=np.complex128)
    if n == "x":
        return np.array([[0, 1], [1, 0]], dtype=np.complex128)
    if n == "y":
        return np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
    if n == "z":
        return np.array([[1, 0], [0, -1]], dtype=np.complex128)
    if n == "h":
        return np.array([[_S2, _S2], [_S2, -_S2]], dtype=np.complex128)
    if n == "s":
        return np.array([[1, 0], [0, 1j]], dtype=np.complex128)
    if n == "sdg":
        return np.array([[1, 0], [0, -1j]], dtype=np.complex128)
    if n == "t":
        return np.array([[1, 0], [0, np.exp(1j * math.pi / 4)]], dtype=np.complex128)
    if n == "tdg":
        return np.array([[1, 0], [0, np.exp(-1j * math.pi / 4)]], dtype=np.complex128)
    if n == "rx":
        th = p[0] if p else 0.0
        c, s = math.cos(th / 2.0), math.sin(th / 2.0)
        return np.array([[c, -1j * s], [-1j * s, c]], dtype=np.complex128)
    if n == "ry":
        th = p[0] if p else 0.0
        c, s = math.cos(th / 2.0), math.sin(th / 2.0)
        return np.array([[c, -s], [s, c]], dtype=np.complex128)
    if n == "rz":
        th = p[0] if p else 0.0
        return np.array([[np.exp(-1j * th / 2.0), 0], [0, np.exp(1j * th / 2.0)]], dtype=np.complex128)
    if n in ("p", "phase"):
        th = p[0] if p else 0.0
        return np.array([[1, 0], [0, np.exp(1j * th)]], dtype=np.complex128)
    if n == "u3":
        th = p[0] if len(p) > 0 else 0.0
        ph = p[1] if len(p) > 1 else 0.0
        lam = p[2] if len(p) > 2 else 0.0
        c, s = math.cos(th / 2.0), math.sin(th / 2.0)
        return np.array([[c, -np.exp(1j * lam) * s],
                         [np.exp(1j * ph) * s, np.exp(1j * (ph + lam)) * c]], dtype=np.complex128)
    if n in ("cx", "cnot"):
        return _ctrl(np.array([[0, 1], [1, 0]], dtype=np.complex128))
    if n == "cy":
        return _ctrl(np.array([[0, -1j], [1j, 0]], dtype=np.complex128))
    if n == "cz":
        return np.diag([1, 1, 1, -1]).astype(np.complex128)
    if n == "ch":
        return _ctrl(np.array([[_S2, _S2], [_S2, -_S2]], dtype=np.complex128))
    if n == "iswap":
        return np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]], dtype=np.complex128)
    if n == "crx":
        th = p[0] if p else 0.0
        c, s = math.cos(th / 2.0), math.sin(th / 2.0)
        return _ctrl(np.array([[c, -1j * s], [-1j * s, c]], dtype=np.complex128))
    if n == "cry":
        th = p[0] if p else 0.0
        c, s = math.cos(th / 2.0), math.sin(th / 2.0)
        return _ctrl(np.array([[c, -s], [s, c]], dtype=np.complex128))
    if n == "crz":
        th = p[0] if p else 0.0
        return np.diag([1, 1, np.exp(-1j * th / 2.0), np.exp(1j * th / 2.0)]).astype(np.complex128)
    if n in ("cp", "cphase"):
        th = p[0] if p else 0.0
        return np.diag([1, 1, 1, np.exp(1j * th)]).astype(np.complex128)
    if n == "swap":
        return np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=np.complex128)
    if n in ("ccx", "toffoli"):
        m = np.eye(8, dtype=np.complex128)
        m[6, 6] = m[7, 7] = 0
        m[6, 7] = m[7, 6] = 1
        return m
    if n in ("cswap", "fredkin"):
        m = np.eye(8, dtype=np.complex128)
        m[5, 5] = m[6, 6] = 0
        m[5, 6] = m[6, 5] = 1
        return m
    return np.eye(2 ** (nqubits if nqubits is not None else 1), dtype=np.complex128)


# generators of the rotation gates: G(theta) = exp(-i theta P / 2)
ROTATION_GENERATORS = {"rx": "X", "ry": "Y", "rz": "Z"}

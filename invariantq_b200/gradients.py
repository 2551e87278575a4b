"""Gradients of E(theta) = <psi(theta)|H|psi(theta)> on the GPU.

* ``adjoint_gradient`` / ``adjoint_gradient_batch`` -- the adjoint method
  (Jones & Gacon, arXiv:2009.02823) in the CUDA library: one forward pass over
  the circuit, lambda = H psi, and one backward sweep that un-applies every
  gate on psi and lambda together and accumulates Im<lambda|P|psi> per
  rotation in FP64.  The batch call runs many circuits and parameter sets
  concurrently on several CUDA streams.
* ``ansatz_energies`` / ``parameter_shift_gradient`` -- the plain path: one
  forward simulation and energy per parameter set, one set at a time, and the
  parameter-shift rule built on it (2 P energies per gradient).
* ``AdjointExpectation`` -- a ``torch.autograd.Function`` whose forward returns
  the energies and whose backward uses the adjoint gradients.

The reference has no gradient code; the energy is its TFIM expectation
(invariantq/algorithms/vqe.py:44-79) for any ansatz of RX/RY/RZ/U3/P rotations
and H/X/SX/CZ/CX gates.  Gate matrices follow invariantq/core/gates.py
(U3 = e^{i(phi+lambda)/2} Rz(phi) Ry(theta) Rz(lambda); the global phase does
not change E)."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from . import _lib

GATE_KINDS = {"rx": 1, "ry": 2, "rz": 3, "u3": 4, "p": 5, "cz": 6, "cx": 7, "h": 8, "x": 9, "sx": 10}
_NPARAM = {1: 1, 2: 1, 3: 1, 4: 3, 5: 1}


class Ansatz:
    """A parametrised circuit from |0...0>.  ``ops`` holds (gate, qubits,
    parameter index) with gate a name of ``GATE_KINDS`` (or its number), qubits
    a tuple (control, target for cx) and the first parameter index the gate
    reads (-1 for fixed gates; u3 reads p, p+1, p+2 as theta, phi, lambda)."""

    def __init__(self, num_qubits: int, ops: Sequence[Tuple]):
        self.num_qubits = int(num_qubits)
        k, a, b, p = [], [], [], []
        for g, qs, pi in ops:
            kind = GATE_KINDS[g.lower()] if isinstance(g, str) else int(g)
            qs = tuple(int(q) for q in qs)
            k.append(kind)
            a.append(qs[0])
            b.append(qs[1] if len(qs) > 1 else -1)
            p.append(int(pi))
        self.kinds = np.ascontiguousarray(k, np.int32)
        self.q0 = np.ascontiguousarray(a, np.int32)
        self.q1 = np.ascontiguousarray(b, np.int32)
        self.param_index = np.ascontiguousarray(p, np.int32)
        n = 0
        for kind, pi in zip(k, p):
            if kind in _NPARAM:
                n = max(n, pi + _NPARAM[kind])
        self.num_params = n

    def __len__(self) -> int:
        return len(self.kinds)

    @classmethod
    def hardware_efficient(cls, n: int, layers: int) -> "Ansatz":
        """RY then RZ on every qubit per layer, then a CZ ring (i, i+1 mod n)."""
        from .circuits import tfim_ansatz_ops
        return cls(n, tfim_ansatz_ops(n, layers))

    def rotation_counts(self) -> np.ndarray:
        """How many rotation angles read each parameter (the shift rule is exact
        when every count is 1)."""
        c = np.zeros(self.num_params, np.int64)
        for kind, pi in zip(self.kinds, self.param_index):
            if kind in _NPARAM:
                c[pi:pi + _NPARAM[kind]] += 1
        return c


class PauliHamiltonian:
    """H = sum_t coeffs[t] P_t with P_t an n-character string over I, X, Y, Z
    (character q acts on qubit q)."""

    def __init__(self, num_qubits: int, coeffs: Sequence[float], paulis: Sequence[str]):
        self.num_qubits = int(num_qubits)
        self.coeffs = np.ascontiguousarray(coeffs, np.float64)
        if len(paulis) != len(self.coeffs):
            raise ValueError("one Pauli string per coefficient")
        for s in paulis:
            if len(s) != self.num_qubits:
                raise ValueError(f"Pauli string {s!r} does not have {self.num_qubits} characters")
        self.paulis = list(paulis)
        self._packed = "".join(self.paulis).encode("ascii")

    @classmethod
    def tfim(cls, n: int, h: float = 1.0) -> "PauliHamiltonian":
        """-sum Z_i Z_{i+1} (open boundary) - h sum X_i."""
        from .circuits import tfim_terms
        c, s = tfim_terms(n, h)
        return cls(n, c, s)


@dataclass
class _Job:
    ansatz: Ansatz
    ham: PauliHamiltonian
    params: np.ndarray        # num_sets x num_params
    energies: np.ndarray
    grads: np.ndarray


def _params2d(ansatz: Ansatz, params) -> np.ndarray:
    p = np.ascontiguousarray(params, np.float64)
    if p.ndim == 1:
        p = p[None, :]
    if p.ndim != 2 or p.shape[1] < ansatz.num_params:
        raise ValueError(f"parameters must have {ansatz.num_params} columns")
    return p


def _struct(job: _Job) -> _lib.AdjointCircuit:
    a, h = job.ansatz, job.ham
    if h.num_qubits != a.num_qubits:
        raise ValueError("the Hamiltonian and the ansatz have different qubit counts")
    ip = lambda x: x.ctypes.data_as(_lib.c_ip)
    dp = lambda x: x.ctypes.data_as(_lib.c_dp)
    return _lib.AdjointCircuit(a.num_qubits, len(a), ip(a.kinds), ip(a.q0), ip(a.q1), ip(a.param_index),
                               job.params.shape[1], job.params.shape[0], dp(job.params), len(h.coeffs),
                               dp(h.coeffs), h._packed, dp(job.energies), dp(job.grads))


def _make_job(ansatz, ham, params) -> _Job:
    p = _params2d(ansatz, params)
    return _Job(ansatz, ham, p, np.zeros(p.shape[0]), np.zeros(p.shape))


def adjoint_gradient_batch(jobs: Sequence[Tuple[Ansatz, PauliHamiltonian, np.ndarray]], num_streams: int = 0
                           ) -> List[Tuple[np.ndarray, np.ndarray]]:
    """Energies (num_sets) and gradients (num_sets x num_params) of every
    (ansatz, Hamiltonian, parameter sets) job, computed concurrently."""
    lib = _lib.load()
    js = [_make_job(a, h, p) for a, h, p in jobs]
    arr = (_lib.AdjointCircuit * max(len(js), 1))(*[_struct(j) for j in js])
    rc = lib.iq_adjoint_gradient_batch(arr, len(js), int(num_streams))
    _lib.check(lib)
    if rc != 0:
        raise _lib.IQError("iq_adjoint_gradient_batch failed")
    return [(j.energies, j.grads) for j in js]


def adjoint_gradient(ansatz: Ansatz, ham: PauliHamiltonian, params) -> Tuple[float, np.ndarray]:
    """Energy and gradient for one parameter vector."""
    (e, g), = adjoint_gradient_batch([(ansatz, ham, np.asarray(params, np.float64)[None, :])], 1)
    return float(e[0]), g[0]


def adjoint_gradient_c64(ansatz: Ansatz, ham: PauliHamiltonian, params) -> Tuple[float, np.ndarray]:
    """Energy and gradient with the states stored as complex64 (FP64 arithmetic
    and sums): half the memory of ``adjoint_gradient``, rounding ~1e-7 relative."""
    lib = _lib.load()
    job = _make_job(ansatz, ham, np.asarray(params, np.float64)[None, :])
    a, h = ansatz, ham
    ip = lambda x: x.ctypes.data_as(_lib.c_ip)
    dp = lambda x: x.ctypes.data_as(_lib.c_dp)
    rc = lib.iq_adjoint_gradient_c64(a.num_qubits, len(a), ip(a.kinds), ip(a.q0), ip(a.q1), ip(a.param_index),
                                     job.params.shape[1], dp(job.params), len(h.coeffs), dp(h.coeffs), h._packed,
                                     dp(job.energies), dp(job.grads))
    _lib.check(lib)
    if rc != 0:
        raise _lib.IQError("iq_adjoint_gradient_c64 failed")
    return float(job.energies[0]), job.grads[0]


def ansatz_energies(ansatz: Ansatz, ham: PauliHamiltonian, params) -> np.ndarray:
    """E for each row of ``params``, one forward simulation after another."""
    lib = _lib.load()
    job = _make_job(ansatz, ham, params)
    s = _struct(job)
    rc = lib.iq_ansatz_energy(ctypes.byref(s))
    _lib.check(lib)
    if rc != 0:
        raise _lib.IQError("iq_ansatz_energy failed")
    return job.energies


def shifted_parameter_sets(params) -> np.ndarray:
    """The 2 P rows theta +- pi/2 e_j (row 2j: +, row 2j+1: -)."""
    p = np.asarray(params, np.float64)
    P = p.shape[0]
    sets = np.repeat(p[None, :], 2 * P, axis=0)
    idx = np.arange(P)
    sets[2 * idx, idx] += np.pi / 2
    sets[2 * idx + 1, idx] -= np.pi / 2
    return sets


def parameter_shift_gradient(ansatz: Ansatz, ham: PauliHamiltonian, params) -> np.ndarray:
    """dE/dtheta_j = [E(theta + pi/2 e_j) - E(theta - pi/2 e_j)] / 2 from 2 P
    plain forward simulations.  Exact when each parameter is read by one
    rotation exp(-i t P / 2) (see ``Ansatz.rotation_counts``)."""
    e = ansatz_energies(ansatz, ham, shifted_parameter_sets(params))
    return 0.5 * (e[0::2] - e[1::2])


def adjoint_release() -> int:
    """Free the workspaces the adjoint calls keep between calls."""
    return int(_lib.load().iq_adjoint_release())


def adjoint_stats() -> dict:
    """Counters of this thread's last adjoint / energy call."""
    lib = _lib.load()
    out = (ctypes.c_double * 10)()
    lib.iq_adjoint_stats(out, 10)
    keys = ["jobs", "forward_passes", "backward_passes", "launches", "bytes", "host_ms", "wall_ms", "streams",
            "specialised_passes", "resident_sets"]
    return dict(zip(keys, list(out)))


try:
    import torch

    class AdjointExpectation(torch.autograd.Function):
        """energies = AdjointExpectation.apply(params, ansatz, hamiltonian):
        params (P) or (S, P) float64; returns a scalar or (S,) energies whose
        backward is the adjoint gradient."""

        @staticmethod
        def forward(ctx, params, ansatz, ham):
            p = params.detach().to("cpu", torch.float64).numpy()
            (e, g), = adjoint_gradient_batch([(ansatz, ham, p.reshape(-1, p.shape[-1]))])
            ctx.save_for_backward(torch.from_numpy(g).to(params.device))
            ctx.one = params.dim() == 1
            out = torch.from_numpy(e).to(params.device)
            return out[0] if ctx.one else out

        @staticmethod
        def backward(ctx, grad_out):
            g, = ctx.saved_tensors
            if ctx.one:
                return grad_out * g[0], None, None
            return grad_out[:, None] * g, None, None

    def expectation(params, ansatz: Ansatz, ham: PauliHamiltonian):
        """Differentiable <psi(params)|H|psi(params)>."""
        return AdjointExpectation.apply(params, ansatz, ham)

except ImportError:   # torch is only needed for the autograd wrapper
    pass

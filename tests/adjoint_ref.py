"""Test infrastructure: energies of parametrised circuits from the oracle (the
C restatement of the reference kernels) and the gradients derived from them
by central finite differences and the parameter-shift rule.  The reference has
no gradient code, so these are the checks the adjoint gradients are held to."""
import numpy as np

from invariantq_b200.gates import gate_matrix

RX, RY, RZ, U3, P, CZ, CX, H, X, SX = range(1, 11)
NAMES = {RX: "rx", RY: "ry", RZ: "rz", U3: "u3", P: "p", CZ: "cz", CX: "cx", H: "h", X: "x"}
SXM = 0.5 * np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]])


def n_params(ops):
    n = 0
    for k, q0, q1, p in ops:
        if k in (RX, RY, RZ, P):
            n = max(n, p + 1)
        elif k == U3:
            n = max(n, p + 3)
    return n


def energy(port, n, ops, theta, coeffs, paulis):
    """<psi(theta)|H|psi(theta)> with every gate applied by the oracle."""
    s = port.zero_state(n)
    for k, q0, q1, p in ops:
        if k in (RX, RY, RZ, P):
            port.apply_1q(s, n, q0, gate_matrix(NAMES[k], [theta[p]]))
        elif k == U3:
            port.apply_1q(s, n, q0, gate_matrix("u3", theta[p:p + 3]))
        elif k in (CZ, CX):
            port.apply_2q(s, n, q0, q1, gate_matrix(NAMES[k]))
        elif k == SX:
            port.apply_1q(s, n, q0, SXM)
        else:
            port.apply_1q(s, n, q0, gate_matrix(NAMES[k]))
    e = 0.0
    for c, ps in zip(coeffs, paulis):
        qs = [q for q, ch in enumerate(ps) if ch != "I"]
        if not qs:
            e += c
            continue
        e += c * port.expval_pauli(s, n, "".join(ps[q] for q in qs), qs).real
    return e


def finite_diff(port, n, ops, theta, coeffs, paulis, h=1e-6):
    g = np.zeros(len(theta))
    for i in range(len(theta)):
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        g[i] = (energy(port, n, ops, tp, coeffs, paulis) - energy(port, n, ops, tm, coeffs, paulis)) / (2 * h)
    return g


def param_shift(port, n, ops, theta, coeffs, paulis):
    """Exact for gates exp(-i theta P / 2): dE = [E(theta + pi/2) - E(theta - pi/2)] / 2."""
    g = np.zeros(len(theta))
    for i in range(len(theta)):
        tp, tm = theta.copy(), theta.copy()
        tp[i] += np.pi / 2
        tm[i] -= np.pi / 2
        g[i] = 0.5 * (energy(port, n, ops, tp, coeffs, paulis) - energy(port, n, ops, tm, coeffs, paulis))
    return g


def random_ansatz(rng, n, ngates):
    ops, p = [], 0
    for _ in range(ngates):
        k = int(rng.choice([RX, RY, RZ, U3, P, CZ, CX, H, SX]))
        q0 = int(rng.integers(n))
        q1 = int((q0 + 1 + rng.integers(n - 1)) % n)
        if k == U3:
            ops.append((k, q0, -1, p))
            p += 3
        elif k in (RX, RY, RZ, P):
            ops.append((k, q0, -1, p))
            p += 1
        elif k in (CZ, CX):
            ops.append((k, q0, q1, -1))
        else:
            ops.append((k, q0, -1, -1))
    return ops


def tfim_ops(n, layers):
    """RY then RZ on every qubit per layer, then a CZ ring (i, i+1 mod n)."""
    ops, p = [], 0
    for _ in range(layers):
        for q in range(n):
            ops.append((RY, q, -1, p))
            p += 1
        for q in range(n):
            ops.append((RZ, q, -1, p))
            p += 1
        for q in range(n if n > 2 else 1):
            ops.append((CZ, q, (q + 1) % n, -1))
    return ops

"""Entanglement entropy across a cut (iq_statevector_entropy) for reduced states
of up to 13 qubits, the half cut range(n // 2) that the reference's driver
computes on every run (invariantq/simulator/statevector.py:87-90,
core/src/statevector.cpp:293-410).  Sides of 7 or more qubits run on the
device (Gram kernel, Householder tridiagonalisation, bisection).

The reference's own Jacobi iteration stops after a fixed number of rotations
and is not converged at these sizes, so the checker is numpy's Hermitian
eigen-solver on the same amplitudes (read back from the library, themselves
pinned to the reference kernels by the other tests): entropies within 1e-9."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _entropy_numpy(amps, n, keep):
    keep = list(keep)
    rest = [q for q in range(n) if q not in keep]
    # axis i of the reshaped tensor is qubit n-1-i
    t = amps.reshape([2] * n)
    axes_keep = [n - 1 - q for q in reversed(keep)]
    axes_rest = [n - 1 - q for q in reversed(rest)]
    m = np.transpose(t, axes_keep + axes_rest).reshape(1 << len(keep), 1 << len(rest))
    rho = m @ m.conj().T if m.shape[0] <= m.shape[1] else m.conj().T @ m
    w = np.linalg.eigvalsh(rho)
    w = w[w > 1e-14]
    return float(-(w * np.log2(w)).sum())


def _brickwall_state(n, depth, seed):
    from invariantq_b200.binding import NativeStateVector
    from invariantq_b200.circuits import brickwall
    from invariantq_b200.simulator import apply_gate_matrix
    c = brickwall(n, depth, seed)
    sv = NativeStateVector(n)
    for op in c.ops:
        apply_gate_matrix(sv, [c.get_qubit_index(q) for q in op.qubits], op.matrix)
    return sv


@pytest.mark.parametrize("n,depth", [(14, 8), (20, 20), (24, 12)])
def test_half_cut_entropy_vs_numpy(n, depth):
    sv = _brickwall_state(n, depth, seed=n)
    got = sv.von_neumann_entropy(list(range(n // 2)))
    want = _entropy_numpy(sv.get_amplitudes(), n, range(n // 2))
    sv.close()
    assert np.isfinite(got)
    assert abs(got - want) < 1e-9, (got, want)


@pytest.mark.parametrize("keep_count", [7, 8, 9, 12])
def test_scattered_subsets_vs_numpy(keep_count):
    """Kept qubits spread over the register; 9 and 12 of 16 leave a smaller
    traced side of 7 and 4 qubits (the spectrum of the smaller side is used)."""
    n = 16
    rng = np.random.default_rng(keep_count)
    sv = _brickwall_state(n, 10, seed=3)
    keep = sorted(int(q) for q in rng.choice(n, keep_count, replace=False))
    got = sv.von_neumann_entropy(keep)
    want = _entropy_numpy(sv.get_amplitudes(), n, keep)
    sv.close()
    assert abs(got - want) < 1e-9, (keep, got, want)


def test_ghz_and_product_states():
    """GHZ across any cut: exactly one bit; a product state: zero."""
    from invariantq_b200.binding import NativeStateVector
    n = 16
    H = np.array([[1, 1], [1, -1]]) / np.sqrt(2)
    CX = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]])
    ghz = NativeStateVector(n)
    ghz.apply_1q(0, H)
    for q in range(n - 1):
        ghz.apply_2q(q, q + 1, CX)
    assert abs(ghz.von_neumann_entropy(list(range(8))) - 1.0) < 1e-12
    assert abs(ghz.von_neumann_entropy([0, 2, 4, 6, 8, 10, 12]) - 1.0) < 1e-12
    ghz.close()
    prod = NativeStateVector(n)
    for q in range(n):
        prod.apply_1q(q, H)
    assert abs(prod.von_neumann_entropy(list(range(8)))) < 1e-12
    prod.close()


def test_sides_above_the_limit_are_rejected():
    from invariantq_b200.binding import NativeStateVector
    sv = NativeStateVector(28)
    with pytest.raises(Exception, match="at most 13"):
        sv.von_neumann_entropy(list(range(14)))
    assert sv.norm_squared() == pytest.approx(1.0)
    sv.close()

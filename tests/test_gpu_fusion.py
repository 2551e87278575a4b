"""Fused circuits (GateFusionPass, k = 2..5) through the CUDA library against
the unfused circuit on the oracle: 1e-12 max-abs."""
import numpy as np
import pytest

from invariantq_b200.circuits import brickwall
from invariantq_b200.fusion import GateFusionPass
from tests.test_fusion import apply_circuit, random_circuit

pytestmark = pytest.mark.gpu
TOL = 1e-12


def run_gpu(c, n):
    from invariantq_b200.binding import NativeStateVector
    from invariantq_b200.simulator import apply_gate_matrix
    sv = NativeStateVector(n)
    for op in c.ops:
        qs = [c.get_qubit_index(q) for q in op.qubits]
        if type(op).__name__ == "FusedGateOp":
            sv.apply_fused(qs, op.fused_matrix)
        else:
            apply_gate_matrix(sv, qs, op.matrix)
    a = sv.get_amplitudes()
    sv.close()
    return a


@pytest.mark.parametrize("k", [2, 3, 4, 5])
def test_fused_brickwall(port, k):
    n = 16
    c = brickwall(n, 10, seed=3)
    f = GateFusionPass(k).run(c)
    assert np.max(np.abs(run_gpu(f, n) - apply_circuit(port, c, n))) < TOL


@pytest.mark.parametrize("k", [3, 5])
def test_fused_random(port, k):
    n = 13
    c = random_circuit(np.random.default_rng(40 + k), n, 200)
    f = GateFusionPass(k).run(c)
    assert np.max(np.abs(run_gpu(f, n) - apply_circuit(port, c, n))) < TOL

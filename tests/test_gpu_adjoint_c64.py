"""The complex64 adjoint variant (states stored as float2, FP64 arithmetic and
sums) against the complex128 adjoint on the same circuits.  The difference is
the float32 rounding of the stored amplitudes, accumulated over the passes: the
tolerance is 2e-5 absolute on energy and gradient (observed <= 2e-7 at these
sizes, 3.4e-8 absolute / 9.3e-8 relative at 30 qubits and 16 layers)."""
import numpy as np
import pytest

from invariantq_b200.circuits import tfim_terms
from tests import adjoint_ref as ar

pytestmark = pytest.mark.gpu
TOL = 2e-5


@pytest.fixture(scope="module")
def G():
    from invariantq_b200 import gradients
    return gradients


@pytest.mark.parametrize("n,layers", [(3, 2), (9, 3), (14, 2), (18, 2)])
def test_tfim_c64_vs_c128(G, n, layers):
    a, h = G.Ansatz.hardware_efficient(n, layers), G.PauliHamiltonian.tfim(n, 0.7)
    th = np.random.default_rng(n).uniform(0, 2 * np.pi, a.num_params)
    e, g = G.adjoint_gradient(a, h, th)
    e32, g32 = G.adjoint_gradient_c64(a, h, th)
    print(f"n={n}: energy {abs(e - e32):.2e} gradient {np.max(np.abs(g - g32)):.2e}")
    assert abs(e - e32) < TOL
    assert np.max(np.abs(g - g32)) < TOL


@pytest.mark.parametrize("n,ngates,seed", [(2, 30, 1), (7, 120, 2)])
def test_mixed_gates_c64_vs_c128(G, n, ngates, seed):
    """Every gate kind (RX/RY/RZ/U3/P, H/X/SX, CZ/CX; runs longer than eight
    gates on one qubit are split) and Y terms in H."""
    rng = np.random.default_rng(seed)
    ops = ar.random_ansatz(rng, n, ngates)
    ops += [(ar.RX, 0, -1, ar.n_params(ops) + i) for i in range(10)]       # a run of ten on qubit 0
    a = G.Ansatz(n, [(k, (q0,) if q1 < 0 else (q0, q1), p) for k, q0, q1, p in ops])
    th = rng.uniform(0, 2 * np.pi, a.num_params)
    paulis = ["".join(rng.choice(list("IXYZ"), n)) for _ in range(5)]
    h = G.PauliHamiltonian(n, rng.normal(size=5), paulis)
    e, g = G.adjoint_gradient(a, h, th)
    e32, g32 = G.adjoint_gradient_c64(a, h, th)
    print(f"mixed n={n}: energy {abs(e - e32):.2e} gradient {np.max(np.abs(g - g32)):.2e}")
    assert abs(e - e32) < TOL
    assert np.max(np.abs(g - g32)) < TOL


def test_tile_path_vs_per_run_passes(G, monkeypatch):
    """From 7 qubits the complex64 gradient runs on the tile-pass executor
    (specialised kernels loading float2 amplitudes, FP64 arithmetic, a float2
    shared tile: one rounding per register stage); the per-run path
    (IQ_C64_TILE=0) rounds after every run of gates.  Both against complex128:
    the tile path is the closer one."""
    n = 16
    a, h = G.Ansatz.hardware_efficient(n, 4), G.PauliHamiltonian.tfim(n, 0.9)
    th = np.random.default_rng(16).uniform(0, 2 * np.pi, a.num_params)
    e, g = G.adjoint_gradient(a, h, th)
    et, gt = G.adjoint_gradient_c64(a, h, th)
    st = G.adjoint_stats()
    assert st["specialised_passes"] > 0 and st["forward_passes"] > 0
    monkeypatch.setenv("IQ_C64_TILE", "0")
    er, gr = G.adjoint_gradient_c64(a, h, th)
    err_tile, err_run = np.max(np.abs(gt - g)), np.max(np.abs(gr - g))
    print(f"c64 tile path {err_tile:.2e}, per-run path {err_run:.2e}")
    assert abs(et - e) < TOL and err_tile < TOL and err_run < TOL
    assert err_tile <= err_run

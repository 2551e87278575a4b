"""The adjoint gradient at 32 qubits, where a third state-sized buffer would not
fit: each parameter set's joint array [psi | lambda] (2^33 complex128
amplitudes, 128 GiB) is the only state memory -- the forward runs on its psi
half in place and lambda = H psi is written to the other half.  Checked
against the parameter-shift rule of the plain energy path on a few angles
(1e-9) and the energy against that path (1e-12)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_adjoint_32_qubits_two_state_buffers():
    import torch
    from invariantq_b200.gradients import Ansatz, PauliHamiltonian, adjoint_gradient, adjoint_release, \
        ansatz_energies, shifted_parameter_sets
    free, _ = torch.cuda.mem_get_info()
    if free < 140 * (1 << 30):
        pytest.skip("needs ~130 GiB of free device memory")
    n, L = 32, 1
    a, h = Ansatz.hardware_efficient(n, L), PauliHamiltonian.tfim(n, 0.9)
    rng = np.random.default_rng(32)
    th = rng.uniform(0, 2 * np.pi, a.num_params)
    e, g = adjoint_gradient(a, h, th)
    adjoint_release()
    idx = np.array([0, 17, n + 5, 2 * n - 1])
    sets = shifted_parameter_sets(th)
    rows = np.concatenate([[2 * j, 2 * j + 1] for j in idx] + [[0]])
    es = ansatz_energies(a, h, np.vstack([sets[rows[:-1]], th[None, :]]))
    ps = 0.5 * (es[0:-1:2] - es[1:-1:2])
    assert abs(e - es[-1]) < 1e-12
    assert np.max(np.abs(g[idx] - ps)) < 1e-9
    adjoint_release()

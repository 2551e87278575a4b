"""GPU adjoint gradients against parameter-shift and central finite differences
of oracle energies, the GPU parameter-shift path, the batch executor and the
autograd wrapper.

Tolerances: energy 1e-12; gradient vs parameter-shift 1e-9 (both exact
methods; they agree to ~1e-15 in practice); gradient vs central differences
with step 1e-6: 1e-9 + 5e-10 * sum|c_t|, because the difference quotient
itself carries a rounding error of about eps * ||H|| / h (||H|| <= sum|c_t|;
5.5e-9 observed at 11 qubits, sum|c_t| = 21)."""
import numpy as np
import pytest

from invariantq_b200.circuits import tfim_terms
from tests import adjoint_ref as ar

pytestmark = pytest.mark.gpu
PS_TOL = 1e-9


def fd_tol(coeffs):
    return 1e-9 + 5e-10 * float(np.sum(np.abs(coeffs)))


@pytest.fixture(scope="module")
def G():
    from invariantq_b200 import gradients
    return gradients


@pytest.fixture(params=["resident", "tile"])
def path(request, monkeypatch):
    """Circuits of <= 12 qubits run on the persistent shared-memory executor by
    default; 'tile' sends them through the tile-pass executor instead."""
    if request.param == "tile":
        monkeypatch.setenv("IQ_RESIDENT_MAX_QUBITS", "0")
    return request.param


def ansatz_of(G, n, ops):
    return G.Ansatz(n, [(k, (a,) if b < 0 else (a, b), p) for k, a, b, p in ops])


@pytest.mark.parametrize("n,layers,seed", [(3, 2, 0), (6, 2, 1), (8, 3, 2), (11, 2, 3)])
def test_tfim_gradient_vs_oracle(G, port, path, n, layers, seed):
    rng = np.random.default_rng(seed)
    ops = ar.tfim_ops(n, layers)
    th = rng.uniform(0, 2 * np.pi, ar.n_params(ops))
    coeffs, paulis = tfim_terms(n, 1.0)
    e, g = G.adjoint_gradient(ansatz_of(G, n, ops), G.PauliHamiltonian(n, coeffs, paulis), th)
    assert abs(e - ar.energy(port, n, ops, th, coeffs, paulis)) < 1e-12
    assert np.max(np.abs(g - ar.param_shift(port, n, ops, th, coeffs, paulis))) < PS_TOL
    assert np.max(np.abs(g - ar.finite_diff(port, n, ops, th, coeffs, paulis))) < fd_tol(coeffs)


@pytest.mark.parametrize("n,ngates,seed", [(2, 20, 4), (5, 50, 5), (7, 80, 6), (9, 120, 7)])
def test_mixed_gates_gradient_vs_oracle(G, port, path, n, ngates, seed):
    """RX/RY/RZ/U3/P rotations among H/SX/CZ/CX, and Y terms in H."""
    rng = np.random.default_rng(seed)
    ops = ar.random_ansatz(rng, n, ngates)
    th = rng.uniform(0, 2 * np.pi, ar.n_params(ops))
    paulis = ["".join(rng.choice(list("IXYZ"), n)) for _ in range(6)]
    coeffs = rng.normal(size=6)
    e, g = G.adjoint_gradient(ansatz_of(G, n, ops), G.PauliHamiltonian(n, coeffs, paulis), th)
    assert abs(e - ar.energy(port, n, ops, th, coeffs, paulis)) < 1e-12
    assert np.max(np.abs(g - ar.param_shift(port, n, ops, th, coeffs, paulis))) < PS_TOL


def test_gpu_parameter_shift_matches_oracle(G, port):
    n, ops = 7, ar.tfim_ops(7, 2)
    th = np.random.default_rng(8).uniform(0, 2 * np.pi, ar.n_params(ops))
    coeffs, paulis = tfim_terms(n, 0.7)
    a, h = ansatz_of(G, n, ops), G.PauliHamiltonian(n, coeffs, paulis)
    assert np.max(np.abs(G.parameter_shift_gradient(a, h, th) - ar.param_shift(port, n, ops, th, coeffs, paulis))) < 1e-12
    assert abs(G.ansatz_energies(a, h, th)[0] - ar.energy(port, n, ops, th, coeffs, paulis)) < 1e-12


@pytest.mark.parametrize("n,layers", [(16, 2), (20, 1)])
def test_large_gradient_vs_gpu_parameter_shift(G, n, layers):
    """Multi-tile circuits: adjoint vs the plain GPU path's parameter shift."""
    a, h = G.Ansatz.hardware_efficient(n, layers), G.PauliHamiltonian.tfim(n, 1.0)
    th = np.random.default_rng(n).uniform(0, 2 * np.pi, a.num_params)
    e, g = G.adjoint_gradient(a, h, th)
    assert abs(e - G.ansatz_energies(a, h, th)[0]) < 1e-12
    assert np.max(np.abs(g - G.parameter_shift_gradient(a, h, th))) < PS_TOL


def test_batch_matches_single_jobs(G, monkeypatch):
    """Uneven circuits, several parameter sets each (run together in one launch
    per pass), on several streams: bit-identical for any number of streams (fixed
    reduction order); equal to one set at a time within 1e-13 through the same
    operation forms (the sets' tiles meet the CTAs in another order) and within
    1e-12 through the single-set forms (rotations and phases, scaled adjoint
    steps: other roundings); to the parameter shift within 1e-9."""
    rng = np.random.default_rng(9)
    jobs = []
    for n, L in [(4, 2), (10, 3), (13, 2), (7, 4), (12, 1)]:
        a, h = G.Ansatz.hardware_efficient(n, L), G.PauliHamiltonian.tfim(n, 1.0)
        jobs.append((a, h, rng.uniform(0, 2 * np.pi, (3, a.num_params))))
    out = G.adjoint_gradient_batch(jobs, num_streams=4)
    st = G.adjoint_stats()
    assert st["resident_sets"] == 12 and st["jobs"] == 3   # the 13-qubit circuit's sets on the tile path
    out1 = G.adjoint_gradient_batch(jobs, num_streams=1)
    for (e, g), (e1, g1) in zip(out, out1):
        assert np.array_equal(e, e1) and np.array_equal(g, g1)
    for (a, h, P), (e, g) in zip(jobs, out):
        for s in range(P.shape[0]):
            e1, g1 = G.adjoint_gradient(a, h, P[s])
            assert abs(e[s] - e1) < 1e-12 and np.max(np.abs(g[s] - g1)) < 1e-12
            assert np.max(np.abs(g1 - G.parameter_shift_gradient(a, h, P[s]))) < PS_TOL
            monkeypatch.setenv("IQ_ADJOINT_SINGLE_FORMS", "0")
            e0, g0 = G.adjoint_gradient(a, h, P[s])
            monkeypatch.delenv("IQ_ADJOINT_SINGLE_FORMS")
            assert e[s] == e0
            assert np.max(np.abs(g[s] - g0)) < 1e-13
            assert np.max(np.abs(g[s] - G.parameter_shift_gradient(a, h, P[s]))) < PS_TOL


def test_batched_sets_at_scale(G):
    """16 parameter sets of a 16-qubit circuit in one batched job against
    each set alone (multi-tile passes, set boundaries inside CTAs' tile runs);
    then the kept workspaces are released and a call after that still works."""
    a, h = G.Ansatz.hardware_efficient(16, 3), G.PauliHamiltonian.tfim(16, 1.0)
    P = np.random.default_rng(13).uniform(0, 2 * np.pi, (16, a.num_params))
    (e, g), = G.adjoint_gradient_batch([(a, h, P)], num_streams=1)
    for s in (0, 7, 15):
        e1, g1 = G.adjoint_gradient(a, h, P[s])
        assert abs(e[s] - e1) < 1e-13
        assert np.max(np.abs(g[s] - g1)) < 1e-12
    assert G.adjoint_release() >= 1
    e2, g2 = G.adjoint_gradient(a, h, P[7])
    assert abs(e2 - e[7]) < 1e-13 and np.max(np.abs(g2 - g[7])) < 1e-12


def test_structure_change_across_sets_is_replanned(G, port, monkeypatch):
    """An angle of 0 turns a fused block monomial: that set gets its own plan
    (tile-pass executor)."""
    monkeypatch.setenv("IQ_RESIDENT_MAX_QUBITS", "0")
    n, ops = 8, ar.tfim_ops(8, 2)
    coeffs, paulis = tfim_terms(n, 1.0)
    a, h = ansatz_of(G, n, ops), G.PauliHamiltonian(n, coeffs, paulis)
    rng = np.random.default_rng(10)
    P = rng.uniform(0, 2 * np.pi, (2, a.num_params))
    P[1, :n] = 0.0
    (e, g), = G.adjoint_gradient_batch([(a, h, P)], num_streams=1)
    for s in range(2):
        assert abs(e[s] - ar.energy(port, n, ops, P[s], coeffs, paulis)) < 1e-12
        assert np.max(np.abs(g[s] - ar.param_shift(port, n, ops, P[s], coeffs, paulis))) < PS_TOL


def test_autograd_function(G):
    import torch
    n = 9
    a, h = G.Ansatz.hardware_efficient(n, 2), G.PauliHamiltonian.tfim(n, 1.0)
    th = torch.tensor(np.random.default_rng(11).uniform(0, 2 * np.pi, a.num_params), requires_grad=True)
    e = G.expectation(th, a, h)
    (2.0 * e).backward()
    e_ref, g_ref = G.adjoint_gradient(a, h, th.detach().numpy())
    assert abs(e.item() - e_ref) < 1e-14
    assert torch.allclose(th.grad, torch.from_numpy(2.0 * g_ref), atol=0, rtol=0)
    P = torch.tensor(np.random.default_rng(12).uniform(0, 2 * np.pi, (3, a.num_params)), requires_grad=True)
    E = G.expectation(P, a, h)
    w = torch.tensor([1.0, -2.0, 0.5], dtype=torch.float64)
    (E * w).sum().backward()
    for s in range(3):
        _, gs = G.adjoint_gradient(a, h, P[s].detach().numpy())
        assert torch.allclose(P.grad[s], w[s] * torch.from_numpy(gs), atol=1e-15, rtol=0)


def test_invalid_inputs_raise(G):
    a = G.Ansatz(3, [("rx", (0,), 0), ("cx", (1, 2), -1)])
    with pytest.raises(ValueError):
        G.adjoint_gradient(G.Ansatz(3, [("cz", (1, 1), -1)]), G.PauliHamiltonian.tfim(3), np.zeros(0))
    with pytest.raises(ValueError):
        G.adjoint_gradient(a, G.PauliHamiltonian(3, [1.0], ["XQZ"]), np.zeros(1))
    with pytest.raises(ValueError):
        G.adjoint_gradient(G.Ansatz(3, [("rx", (5,), 0)]), G.PauliHamiltonian.tfim(3), np.zeros(1))
    e, g = G.adjoint_gradient(a, G.PauliHamiltonian(3, [0.5], ["IIZ"]), np.array([0.3]))
    assert abs(e - 0.5) < 1e-15 and abs(g[0]) < 1e-15


def test_specialised_kernels_equal_interpreting(G, monkeypatch):
    """IQ_ADJOINT_JIT = 1 (kernels generated per pass structure, default) and 0
    (interpreting kernel) run the same plans with the same arithmetic:
    energies and gradients are identical, for one set and for sets batched
    in one launch (adjoint steps, set switches, gradient accumulators)."""
    monkeypatch.setenv("IQ_RESIDENT_MAX_QUBITS", "0")
    rng = np.random.default_rng(31)
    jobs = []
    for n, L in [(12, 3), (9, 2)]:
        a, h = G.Ansatz.hardware_efficient(n, L), G.PauliHamiltonian.tfim(n, 0.8)
        jobs.append((a, h, rng.uniform(0, 2 * np.pi, (4, a.num_params))))
    out = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("IQ_ADJOINT_JIT", flag)
        out[flag] = G.adjoint_gradient_batch(jobs, num_streams=2)
        st = G.adjoint_stats()
        assert (st["specialised_passes"] > 0) == (flag == "1")
        out[flag + "s"] = G.adjoint_gradient(jobs[0][0], jobs[0][1], jobs[0][2][1])
    for (e0, g0), (e1, g1) in zip(out["0"], out["1"]):
        assert np.array_equal(e0, e1) and np.array_equal(g0, g1)
    assert out["0s"][0] == out["1s"][0] and np.array_equal(out["0s"][1], out["1s"][1])


def test_resident_executor_matches_tile_executor(G, monkeypatch):
    """The persistent shared-memory executor (all sets of all circuits of <= 12
    qubits in one launch from a device-side queue, replayed from a captured
    graph) against the tile-pass executor on the same batch: 1e-12; the second
    call of the same structure (graph replay, new parameters staged) equals a
    fresh single-set run exactly, and the results do not depend on the batch."""
    rng = np.random.default_rng(41)
    jobs = []
    for n, L in [(3, 2), (12, 2), (8, 3), (1, 2), (10, 1), (5, 4)]:
        a = G.Ansatz.hardware_efficient(n, L) if n > 1 else G.Ansatz(1, [("ry", (0,), 0), ("rz", (0,), 1)])
        jobs.append((a, G.PauliHamiltonian.tfim(n, 0.9), rng.uniform(0, 2 * np.pi, (5, a.num_params))))
    res = G.adjoint_gradient_batch(jobs)
    assert G.adjoint_stats()["resident_sets"] == 30
    monkeypatch.setenv("IQ_RESIDENT_MAX_QUBITS", "0")
    tile = G.adjoint_gradient_batch(jobs)
    assert G.adjoint_stats()["resident_sets"] == 0
    monkeypatch.delenv("IQ_RESIDENT_MAX_QUBITS")
    for (e0, g0), (e1, g1) in zip(res, tile):
        assert np.max(np.abs(e0 - e1)) < 1e-12 and np.max(np.abs(g0 - g1)) < 1e-12
    jobs2 = [(a, h, P[::-1].copy()) for a, h, P in jobs]        # same structure, other parameters
    res2 = G.adjoint_gradient_batch(jobs2)
    for (e0, g0), (e2, g2) in zip(res, res2):
        assert np.array_equal(e0[::-1], e2) and np.array_equal(g0[::-1], g2)
    a, h, P = jobs[1]
    e1, g1 = G.adjoint_gradient(a, h, P[3])
    assert e1 == res[1][0][3] and np.array_equal(g1, res[1][1][3])

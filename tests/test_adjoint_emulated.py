"""CPU check of the adjoint-gradient pipeline: the op lists built by
iq_sched.cpp (forward, lambda = H psi, backward sweep of adjoint steps on the
joint psi/lambda array) run through the planned passes with the kernel's
semantics (tests/plan_emulator.cpp), against parameter-shift and finite
differences of oracle energies."""
import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

from invariantq_b200.circuits import tfim_terms
from tests import adjoint_ref as ar

REPO = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="session")
def emu(tmp_path_factory):
    out = tmp_path_factory.mktemp("emuadj") / "libplanemu.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(out),
                    str(REPO / "tests" / "plan_emulator.cpp"),
                    str(REPO / "invariantq_b200" / "csrc" / "iq_sched.cpp"),
                    str(REPO / "invariantq_b200" / "csrc" / "iq_jitgen.cpp")], check=True)
    return ctypes.CDLL(str(out))


def emu_grad(emu, n, ops, theta, coeffs, paulis, M=11, c=5, stages=8, budget=80.0, R=4, single_set=False):
    k = np.array([o[0] for o in ops], np.int32)
    q0 = np.array([o[1] for o in ops], np.int32)
    q1 = np.array([o[2] for o in ops], np.int32)
    pi = np.array([o[3] for o in ops], np.int32)
    th = np.ascontiguousarray(theta, np.float64)
    co = np.ascontiguousarray(coeffs, np.float64)
    ps = "".join(paulis).encode()
    e = ctypes.c_double()
    g = np.zeros(len(theta))
    err = ctypes.create_string_buffer(256)
    P = ctypes.c_void_p
    rc = emu.emu_adjoint_forms(n, len(ops), P(k.ctypes.data), P(q0.ctypes.data), P(q1.ctypes.data),
                               P(pi.ctypes.data), P(th.ctypes.data), len(coeffs), P(co.ctypes.data), ps, M, c, R,
                               stages, ctypes.c_double(budget), ctypes.byref(e), P(g.ctypes.data), len(theta),
                               int(single_set), err, 256)
    assert rc == 0, err.value
    return e.value, g


@pytest.mark.parametrize("n,layers,seed", [(6, 2, 0), (8, 3, 1), (9, 2, 2)])
def test_tfim_ansatz_gradient(port, emu, n, layers, seed):
    rng = np.random.default_rng(seed)
    ops = ar.tfim_ops(n, layers)
    theta = rng.uniform(0, 2 * np.pi, ar.n_params(ops))
    coeffs, paulis = tfim_terms(n, 0.7)
    e, g = emu_grad(emu, n, ops, theta, coeffs, paulis)
    assert abs(e - ar.energy(port, n, ops, theta, coeffs, paulis)) < 1e-12
    assert np.max(np.abs(g - ar.param_shift(port, n, ops, theta, coeffs, paulis))) < 1e-10
    assert np.max(np.abs(g - ar.finite_diff(port, n, ops, theta, coeffs, paulis))) < 1e-7


@pytest.mark.parametrize("n,ngates,seed", [(5, 40, 3), (7, 60, 4), (8, 80, 5)])
def test_mixed_gates_gradient(port, emu, n, ngates, seed):
    rng = np.random.default_rng(seed)
    ops = ar.random_ansatz(rng, n, ngates)
    theta = rng.uniform(0, 2 * np.pi, ar.n_params(ops))
    # a random Pauli observable with X, Y and Z terms
    paulis = ["".join(rng.choice(list("IXYZ"), n)) for _ in range(6)]
    coeffs = rng.normal(size=6)
    e, g = emu_grad(emu, n, ops, theta, coeffs, paulis, budget=60.0, stages=4)
    assert abs(e - ar.energy(port, n, ops, theta, coeffs, paulis)) < 1e-12
    assert np.max(np.abs(g - ar.param_shift(port, n, ops, theta, coeffs, paulis))) < 1e-10


@pytest.mark.parametrize("R", [3, 5])
def test_register_slot_variants(port, emu, R):
    """Adjoint steps keep the select bit in slot 0 with 3 and 5 register slots."""
    n, layers = 8, 2
    rng = np.random.default_rng(20 + R)
    ops = ar.tfim_ops(n, layers)
    theta = rng.uniform(0, 2 * np.pi, ar.n_params(ops))
    coeffs, paulis = tfim_terms(n, 0.7)
    e, g = emu_grad(emu, n, ops, theta, coeffs, paulis, R=R)
    assert abs(e - ar.energy(port, n, ops, theta, coeffs, paulis)) < 1e-12
    assert np.max(np.abs(g - ar.param_shift(port, n, ops, theta, coeffs, paulis))) < 1e-10


@pytest.mark.parametrize("n,ngates,seed", [(5, 50, 11), (8, 90, 12), (9, 70, 13)])
def test_single_set_forms(port, emu, n, ngates, seed):
    """A circuit with one parameter set: forward decomposed into rotations and
    phases, adjoint steps in the tan / cot / phase-free forms with their
    scales undone in the order the planned passes run them.  Angles include
    0, pi, +-pi/2 (cot form, exact zeros); against the parameter-shift rule and
    the fused-block lists of a shared plan."""
    rng = np.random.default_rng(seed)
    ops = ar.random_ansatz(rng, n, ngates)
    theta = rng.uniform(0, 2 * np.pi, ar.n_params(ops))
    special = np.array([0.0, np.pi, np.pi / 2, -np.pi / 2, 3 * np.pi])
    theta[::4] = special[np.arange(len(theta[::4])) % len(special)]
    paulis = ["".join(rng.choice(list("IXYZ"), n)) for _ in range(5)]
    coeffs = rng.normal(size=5)
    e1, g1 = emu_grad(emu, n, ops, theta, coeffs, paulis, budget=60.0, stages=4, single_set=True)
    e0, g0 = emu_grad(emu, n, ops, theta, coeffs, paulis, budget=60.0, stages=4)
    assert abs(e1 - ar.energy(port, n, ops, theta, coeffs, paulis)) < 1e-12
    assert np.max(np.abs(g1 - ar.param_shift(port, n, ops, theta, coeffs, paulis))) < 1e-10
    assert np.max(np.abs(g1 - g0)) < 1e-12


def test_scaled_steps_rescale_long_sweep(port, emu):
    """301 RX / RY steps at angles whose divisor is about 1/sqrt(2) take the
    scale of the backward sweep past 2^-64 twice: scalar operations restore it
    and every gradient still matches the parameter-shift rule."""
    n = 7
    ops, p = [], 0
    for layer in range(43):
        for q in range(n):
            ops.append((ar.RY if (layer + q) % 2 else ar.RX, q, -1, p))
            p += 1
        for q in range(n - 1):
            ops.append((ar.CZ, q, q + 1, -1))
    rng = np.random.default_rng(5)
    theta = np.where(rng.random(p) < 0.5, np.pi / 2, -np.pi / 2) + rng.normal(scale=1e-3, size=p)
    coeffs, paulis = tfim_terms(n, 0.6)
    e, g = emu_grad(emu, n, ops, theta, coeffs, paulis, M=9, c=4, single_set=True)
    assert abs(e - ar.energy(port, n, ops, theta, coeffs, paulis)) < 1e-11
    assert np.max(np.abs(g - ar.param_shift(port, n, ops, theta, coeffs, paulis))) < 1e-9

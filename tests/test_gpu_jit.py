"""Specialised pass kernels (option "jit") on the GPU: the same planned passes
(plan_style 2: CX/CZ/SWAP left apart, normalised one-qubit gates) run by the
generated kernels and by the interpreting kernel give identical amplitudes
(same arithmetic expression per operation, same pipeline), and the oracle's
within 1e-12.  Covers register slots R = 3, 4, 5, density matrices,
recorded programs, and flushes that pick up kernels compiled in the background."""
import numpy as np
import pytest

from tests.test_gpu_sv import apply_abi
from tests.test_scheduler_emulated import gen_ops, oracle_apply, rand_unitary

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def B():
    from invariantq_b200 import binding
    return binding


def run_sv(B, n, ops, jit, **opts):
    sv = B.NativeStateVector(n)
    try:
        sv.set_option("jit", jit)
        for k, v in opts.items():
            sv.set_option(k, v)
        apply_abi(sv, ops)
        return sv.get_amplitudes(), sv.stats()
    finally:
        sv.close()


@pytest.mark.parametrize("n,kmax,R,M", [(12, 4, 4, 11), (16, 2, 4, 12), (13, 3, 3, 11), (14, 5, 5, 12)])
def test_specialised_equals_interpreting(B, port, n, kmax, R, M):
    rng = np.random.default_rng(100 + n + R)
    ops = gen_ops(rng, n, 120, kmax=kmax)
    opts = {"tile_bits": M, "reg_slots": R, "budget": 96, "plan_style": 2}
    a0, s0 = run_sv(B, n, ops, 0, **opts)
    a2, s2 = run_sv(B, n, ops, 2, **opts)
    assert s0["jit_passes"] == 0
    assert s2["jit_passes"] == s2["tile_passes"] > 0
    assert np.array_equal(a0, a2)
    ref = oracle_apply(port, port.zero_state(n), n, ops)
    assert np.max(np.abs(a2 - ref)) < TOL


def test_recorded_program_compiles_at_record_end(B):
    """Default jit = 1, 20 qubits: every pass of a recorded program runs specialised."""
    from invariantq_b200.circuits import brickwall
    from invariantq_b200.simulator import apply_gate_matrix
    n = 20
    c = brickwall(n, 12, seed=5)
    out = []
    for jit in (0, 1):
        sv = B.NativeStateVector(n)
        sv.set_option("jit", jit)
        sv.set_option("plan_style", 2)
        with sv.record() as rec:
            for op in c.ops:
                qs = [c.get_qubit_index(q) for q in op.qubits]
                apply_gate_matrix(sv, qs, np.asarray(op.matrix, np.complex128))
        prog = rec.program
        sv.reset()
        prog.run(sv)
        st = sv.stats()
        out.append(sv.get_amplitudes())
        assert st["jit_passes"] == (prog.passes if jit else 0)
        sv.close()
    assert np.array_equal(out[0], out[1])


def test_flushes_use_background_compiled_kernels(B):
    """jit = 1 on 2^18 amplitudes: the first run queues its passes' kernels,
    a run of the same structure after jit_wait uses them."""
    n = 18
    rng = np.random.default_rng(7)
    ops = gen_ops(rng, n, 90, kmax=2)
    a0, _ = run_sv(B, n, ops, 0)
    sv = B.NativeStateVector(n)
    try:
        apply_abi(sv, ops)
        first = sv.get_amplitudes()
        assert B.jit_wait(300.0)
        before = sv.stats()["jit_passes"]
        sv.reset()
        apply_abi(sv, ops)
        again = sv.get_amplitudes()
        assert sv.stats()["jit_passes"] > before
    finally:
        sv.close()
    assert np.array_equal(first, again)            # same plan: interpreting, then specialised
    assert np.max(np.abs(again - a0)) < TOL       # a0: planned for the interpreting kernel
    info = B.jit_info()
    assert info["compiled"] + info["from_disk"] > 0 and info["note"] == ""


def test_density_matrix_specialised(B):
    n = 7
    rng = np.random.default_rng(3)
    mats = []
    for jit in (0, 2):
        dm = B.NativeDensityMatrix(n)
        dm.set_option("jit", jit)
        dm.set_option("plan_style", 2)
        r = np.random.default_rng(3)
        for _ in range(25):
            a, b = (int(x) for x in r.choice(n, 2, replace=False))
            dm.apply_1q_unitary(a, rand_unitary(r, 2))
            dm.apply_2q_unitary(a, b, rand_unitary(r, 4))
            p = 0.05
            dm.apply_1q_kraus(b, [np.sqrt(1 - p) * np.eye(2), np.sqrt(p) * np.array([[0, 1], [1, 0]])])
        mats.append(dm.get_matrix())
        assert (dm.stats()["jit_passes"] > 0) == (jit == 2)
        dm.close()
    assert np.array_equal(mats[0], mats[1])
    assert abs(np.trace(mats[1]).real - 1.0) < 1e-12
    del rng


def test_density_matrix_channel_superoperators(B):
    """Depolarizing, amplitude / phase damping and thermal relaxation channels
    (superoperators of the corner + middle shape, run as X2R operations):
    specialised and interpreting kernels give identical matrices; trace 1."""
    from invariantq_b200.channels import build_kraus_channel
    n = 8
    chans = [build_kraus_channel("depolarizing", [2e-2]), build_kraus_channel("amp_damping", [3e-2]),
             build_kraus_channel("phase_damping", [2e-2]),
             build_kraus_channel("thermal_relaxation", [100e-6, 80e-6, 50e-9])]
    mats = []
    for jit in (0, 2):
        dm = B.NativeDensityMatrix(n)
        dm.set_option("jit", jit)
        dm.set_option("plan_style", 2)
        r = np.random.default_rng(8)
        for _ in range(30):
            a, b = (int(x) for x in r.choice(n, 2, replace=False))
            dm.apply_1q_unitary(a, rand_unitary(r, 2))
            dm.apply_1q_kraus(a, chans[int(r.integers(4))])
            dm.apply_2q_unitary(a, b, np.eye(4)[[0, 1, 3, 2]])
            dm.apply_1q_kraus(b, chans[int(r.integers(4))])
            dm.apply_1q_kraus(b, chans[int(r.integers(4))])
        mats.append(dm.get_matrix())
        assert (dm.stats()["jit_passes"] > 0) == (jit == 2)
        dm.close()
    assert np.array_equal(mats[0], mats[1])
    assert abs(np.trace(mats[1]).real - 1.0) < 1e-12


def test_x_shaped_two_qubit_gates(B, port):
    """Two-qubit gates whose only nonzero entries are the corners
    {00, 11} x {00, 11} and the middle diagonal, with complex entries (a
    unitary on the {00, 11} pair and phases on 01, 10): they run as X2R with
    complex corners and middle; specialised and interpreting kernels agree bit
    for bit, and the oracle within 1e-12."""
    n = 12
    r = np.random.default_rng(21)
    ops = []
    for _ in range(40):
        a, b = (int(x) for x in r.choice(n, 2, replace=False))
        ops.append(("1q", [a], rand_unitary(r, 2)))
        W = rand_unitary(r, 2)
        X = np.zeros((4, 4), np.complex128)
        X[np.ix_([0, 3], [0, 3])] = W
        X[1, 1], X[2, 2] = np.exp(1j * r.uniform(0, 2 * np.pi, 2))
        ops.append(("2q", [a, b], X))
    opts = {"plan_style": 2}
    a0, _ = run_sv(B, n, ops, 0, **opts)
    a2, s2 = run_sv(B, n, ops, 2, **opts)
    assert s2["jit_passes"] == s2["tile_passes"] > 0
    assert np.array_equal(a0, a2)
    ref = oracle_apply(port, port.zero_state(n), n, ops)
    assert np.max(np.abs(a2 - ref)) < TOL


def test_normalised_planning_vs_oracle(B, port):
    """Plan style 2 on the interpreting kernel, more dense one-qubit gates than
    one normalisation run (a CZ after each keeps them from merging)."""
    from tests.test_scheduler_emulated import CZ
    n = 11
    rng = np.random.default_rng(5)
    ops = []
    for _ in range(600):
        q = int(rng.integers(n))
        ops += [("1q", [q], rand_unitary(rng, 2)), ("2q", [q, (q + 1) % n], CZ)]
    ref = oracle_apply(port, port.zero_state(n), n, ops)
    for jit in (0, 2):
        a, st = run_sv(B, n, ops, jit, plan_style=2)
        assert np.max(np.abs(a - ref)) < TOL

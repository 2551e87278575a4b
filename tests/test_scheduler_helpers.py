"""CPU checks of two scheduler helpers (invariantq_b200/csrc/iq_sched.cpp):
the OP_X2R shape classification of channel superoperators, and the scales of a
scaled backward sweep taken in the order the planned passes run its
operations (which differs from the queue order when the planner moves adjoint
steps on different qubits past each other)."""
import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests import adjoint_ref as ar
from tests.test_scheduler_emulated import superop_lsb

REPO = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    out = tmp_path_factory.mktemp("emuhelp") / "libplanemu.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(out),
                    str(REPO / "tests" / "plan_emulator.cpp"),
                    str(REPO / "invariantq_b200" / "csrc" / "iq_sched.cpp"),
                    str(REPO / "invariantq_b200" / "csrc" / "iq_jitgen.cpp")], check=True)
    lib = ctypes.CDLL(str(out))
    lib.emu_classify_xpattern.restype = ctypes.c_int
    return lib


def classify(emu, m):
    flat = np.ascontiguousarray(np.asarray(m, np.complex128).reshape(-1).view(np.float64))
    return emu.emu_classify_xpattern(flat.ctypes.data_as(ctypes.c_void_p))


SHAPE, CORNERS_REAL, MIDDLE_REAL = 1, 2, 4


def test_channel_superoperators_have_the_shape(emu):
    from invariantq_b200.channels import build_kraus_channel
    for name, params in [("depolarizing", [1e-3]), ("amp_damping", [0.3]), ("phase_damping", [0.2]),
                         ("thermal_relaxation", [100e-6, 80e-6, 50e-9])]:
        S = superop_lsb(build_kraus_channel(name, params))
        assert classify(emu, S) == SHAPE | CORNERS_REAL | MIDDLE_REAL, name
    # a bit flip maps |01> to |10>: not the shape
    bit_flip = [np.sqrt(0.9) * np.eye(2), np.sqrt(0.1) * np.array([[0, 1], [1, 0]])]
    assert classify(emu, superop_lsb(bit_flip)) == 0


def test_shape_with_complex_entries(emu):
    S = np.zeros((4, 4), np.complex128)
    S[0, 0], S[0, 3], S[3, 0], S[3, 3] = 0.9, 0.1, 0.2, 0.8
    S[1, 1], S[2, 2] = 0.5 + 0.1j, 0.5 - 0.1j
    assert classify(emu, S) == SHAPE | CORNERS_REAL
    S[0, 3] = 0.1j
    assert classify(emu, S) == SHAPE
    S[1, 2] = 1e-300                       # any other nonzero entry
    assert classify(emu, S) == 0
    assert classify(emu, np.diag([1.0, 2.0, 3.0, 4.0])) == SHAPE | CORNERS_REAL | MIDDLE_REAL


def grad_scales(emu, n, ops, theta, M=9, c=4):
    k = np.array([o[0] for o in ops], np.int32)
    q0 = np.array([o[1] for o in ops], np.int32)
    q1 = np.array([o[2] for o in ops], np.int32)
    pi = np.array([o[3] for o in ops], np.int32)
    th = np.ascontiguousarray(theta, np.float64)
    cap = 4096
    ex, qu = np.zeros(cap), np.zeros(cap)
    P = ctypes.c_void_p
    cnt = emu.emu_grad_scales(n, len(ops), P(k.ctypes.data), P(q0.ctypes.data), P(q1.ctypes.data),
                              P(pi.ctypes.data), P(th.ctypes.data), M, c, P(ex.ctypes.data), P(qu.ctypes.data), cap)
    assert cnt > 0
    return ex[:cnt], qu[:cnt]


def test_scales_follow_the_run_order(emu):
    """Every term's run-order scale is the square of a product of the step
    divisors (each in [1/sqrt 2, 1]); the first term to run has scale 1; the
    planner reorders steps of different qubits, so some run-order scales differ
    from the queue-order ones, which the executor therefore does not use."""
    n, layers = 9, 3
    ops = ar.tfim_ops(n, layers)
    theta = np.random.default_rng(4).uniform(0, 2 * np.pi, ar.n_params(ops))
    ex, qu = grad_scales(emu, n, ops, theta)
    assert np.all(ex > 0) and np.all(ex <= 1.0 + 1e-15)
    assert np.all(ex >= 0.5 ** (len(ex) - 1) - 1e-300)
    assert np.max(ex) == 1.0 and qu[0] == 1.0
    assert np.any(np.abs(ex - qu) > 1e-12 * np.abs(qu))


def test_z_only_sweeps_keep_unit_scales(emu):
    """RZ steps un-apply diag(1, e^{-i theta}): no divisor, every scale 1."""
    n = 8
    ops, p = [], 0
    for _ in range(3):
        for q in range(n):
            ops.append((ar.RZ, q, -1, p))
            p += 1
        for q in range(n - 1):
            ops.append((ar.CZ, q, q + 1, -1))
    theta = np.random.default_rng(5).uniform(0, 2 * np.pi, p)
    ex, qu = grad_scales(emu, n, ops, theta)
    assert np.all(ex == 1.0) and np.all(qu == 1.0)

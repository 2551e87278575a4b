"""Pin the C oracle (oracle/iq_oracle.c) against fixtures produced by the
reference's own core and Python binding (tests/golden/make_golden.py)."""
import numpy as np
import pytest

OP_1Q, OP_2Q, OP_FUSED = 1, 2, 3
TOL = 1e-13


def replay_sv(port, n, kinds, qubits, mats):
    s = port.zero_state(n)
    for kind, qs, m in zip(kinds, qubits, mats):
        qs = [int(q) for q in qs if q >= 0]
        d = 1 << len(qs)
        U = np.ascontiguousarray(m[:d, :d])
        if kind == OP_1Q:
            assert port.apply_1q(s, n, qs[0], U) == 0
        elif kind == OP_2Q:
            assert port.apply_2q(s, n, qs[0], qs[1], U) == 0
        else:
            assert port.apply_fused(s, n, qs, U) == 0
    return s


@pytest.mark.parametrize("n", [3, 5, 8, 10])
def test_sv_op_sequences(port, golden, n):
    g = golden("sv_ops")
    s = replay_sv(port, n, g[f"n{n}_kinds"], g[f"n{n}_qubits"], g[f"n{n}_mats"])
    assert np.max(np.abs(s - g[f"n{n}_amps"])) < TOL


def prep_readout_state(port, g):
    n = 8
    s = port.zero_state(n)
    for kind, qs, m in zip(g["prep_kinds"], g["prep_qubits"], g["prep_mats"]):
        if kind == 1:
            port.apply_1q(s, n, int(qs[0]), np.ascontiguousarray(m[:2, :2]))
        else:
            port.apply_2q(s, n, int(qs[0]), int(qs[1]), np.ascontiguousarray(m))
    return n, s


def test_sv_readout(port, golden):
    g = golden("sv_readout")
    n, s = prep_readout_state(port, g)
    assert np.max(np.abs(s - g["amps"])) < TOL
    assert np.max(np.abs(port.probabilities(s, n) - g["probs"])) < TOL
    mp = np.array([[port.measure_prob(s, n, t, o) for o in (0, 1)] for t in range(n)])
    assert np.max(np.abs(mp - g["measure_prob"])) < TOL
    for ps, pq, pv in zip(g["pauli_strings"], g["pauli_qubits"], g["pauli_values"]):
        qs = [int(q) for q in pq if q >= 0]
        v = port.expval_pauli(s, n, str(ps)[: len(qs)], qs)
        assert abs(v - pv) < TOL
    # sampling: same mt19937_64 stream and lower_bound search -> identical indices
    assert np.array_equal(port.sample(s, n, 4096, 7), g["samples"])
    assert np.array_equal(port.sample(s, n, 1000, 42), g["samples_seed42"])
    for es, ev in zip(g["entropy_sets"], g["entropy"]):
        qs = [int(q) for q in es if q >= 0]
        assert abs(port.entropy(s, n, qs) - ev) < 1e-10
    s2 = s.copy()
    assert port.measure(s2, n, 3, 0.3) == int(g["measure_outcome"])
    assert np.max(np.abs(s2 - g["amps_after_measure"])) < TOL
    assert port.reset_qubit(s2, n, 5, 0.7) == 0
    assert np.max(np.abs(s2 - g["amps_after_reset"])) < TOL


def test_sv_special_cases(port, golden):
    g = golden("sv_readout")
    H = np.array([[1, 1], [1, -1]], np.complex128) / np.sqrt(2)
    CX = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], np.complex128)
    b = port.zero_state(2)
    port.apply_1q(b, 2, 0, H)
    port.apply_2q(b, 2, 0, 1, CX)
    assert np.max(np.abs(b - g["bell_amps"])) < TOL
    assert abs(port.entropy(b, 2, [0]) - float(g["bell_entropy"])) < 1e-12
    # fused k=3 uses an LSB-first local index: CCX lands on basis index 3 (not 7)
    c = port.zero_state(3)
    X = np.array([[0, 1], [1, 0]], np.complex128)
    port.apply_1q(c, 3, 0, X)
    port.apply_1q(c, 3, 1, X)
    ccx = np.eye(8, dtype=np.complex128)
    ccx[6, 6] = ccx[7, 7] = 0
    ccx[6, 7] = ccx[7, 6] = 1
    port.apply_fused(c, 3, [0, 1, 2], ccx)
    assert np.max(np.abs(c - g["ccx_amps"])) < TOL
    assert abs(c[3]) == pytest.approx(1.0)


def test_sv_error_paths(port):
    s = port.zero_state(3)
    U = np.eye(2, dtype=np.complex128)
    assert port.apply_1q(s, 3, 3, U) == -1
    assert port.apply_2q(s, 3, 1, 1, np.eye(4, dtype=np.complex128)) == -1
    assert port.apply_fused(s, 3, [0, 1, 2, 2], np.eye(16, dtype=np.complex128)) == -1
    big = port.zero_state(6)
    assert port.apply_fused(big, 6, [0, 1, 2, 3, 4], np.eye(32, dtype=np.complex128)) == -2
    z = port.zero_state(2)
    assert port.measure_prob(z, 2, 0, 1) == 0.0
    assert port.measure(z, 2, 0, 0.99) == 0  # p0 = 1 > rand


@pytest.mark.parametrize("n", [2, 3, 4])
def test_dm_sequences(port, golden, n):
    g = golden("dm_ops")
    rho = port.zero_rho(n)
    for kind, qs, m, nk in zip(g[f"n{n}_kinds"], g[f"n{n}_qubits"], g[f"n{n}_mats"], g[f"n{n}_nkraus"]):
        if kind == 1:
            assert port.dm_apply_1q(rho, n, int(qs[0]), np.ascontiguousarray(m[0, :2, :2])) == 0
        elif kind == 2:
            assert port.dm_apply_2q(rho, n, int(qs[0]), int(qs[1]), np.ascontiguousarray(m[0])) == 0
        elif kind == 3:
            K = [np.ascontiguousarray(m[j, :2, :2]) for j in range(nk)]
            assert port.dm_apply_kraus_1q(rho, n, int(qs[0]), K) == 0
        else:
            assert port.dm_reset_qubit(rho, n, int(qs[0])) == 0
    assert np.max(np.abs(rho - g[f"n{n}_rho"])) < TOL
    assert abs(port.dm_trace(rho, n) - float(g[f"n{n}_trace"])) < TOL
    assert abs(port.dm_purity(rho, n) - float(g[f"n{n}_purity"])) < TOL
    assert abs(port.dm_entropy(rho, n) - float(g[f"n{n}_entropy"])) < 1e-10
    assert port.dm_measure(rho, n, 0, 0.4) == int(g[f"n{n}_measure_outcome"])
    assert np.max(np.abs(rho - g[f"n{n}_rho_after_measure"])) < TOL

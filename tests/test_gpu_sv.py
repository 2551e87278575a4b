"""GPU parity of the state-vector path (C ABI through the ctypes binding)
against the golden fixtures made by the reference, the C oracle, and the
reference core itself (oracle/_ref).  Amplitude tolerance: 1e-12 max-abs."""
import math

import numpy as np
import pytest

from tests.test_scheduler_emulated import CX, CZ, SWAP, X, S, gen_ops, oracle_apply, rand_unitary

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def SV():
    from invariantq_b200.binding import NativeStateVector
    return NativeStateVector


def apply_abi(sv, ops):
    for kind, qs, U in ops:
        if kind == "1q":
            sv.apply_1q(qs[0], U)
        elif kind == "2q":
            sv.apply_2q(qs[0], qs[1], U)
        else:
            sv.apply_fused(qs, U)


@pytest.mark.parametrize("n", [3, 5, 8, 10])
def test_golden_op_sequences(SV, golden, n):
    g = golden("sv_ops")
    sv = SV(n)
    for kind, qs, m in zip(g[f"n{n}_kinds"], g[f"n{n}_qubits"], g[f"n{n}_mats"]):
        qs = [int(q) for q in qs if q >= 0]
        d = 1 << len(qs)
        U = m[:d, :d]
        if kind == 1:
            sv.apply_1q(qs[0], U)
        elif kind == 2:
            sv.apply_2q(qs[0], qs[1], U)
        else:
            sv.apply_fused(qs, U)
    assert np.max(np.abs(sv.get_amplitudes() - g[f"n{n}_amps"])) < TOL


def readout_state(SV, g):
    n = 8
    sv = SV(n)
    for kind, qs, m in zip(g["prep_kinds"], g["prep_qubits"], g["prep_mats"]):
        if kind == 1:
            sv.apply_1q(int(qs[0]), m[:2, :2])
        else:
            sv.apply_2q(int(qs[0]), int(qs[1]), m)
    return n, sv


def test_golden_readouts(SV, golden):
    g = golden("sv_readout")
    n, sv = readout_state(SV, g)
    assert np.max(np.abs(sv.get_amplitudes() - g["amps"])) < TOL
    assert np.max(np.abs(sv.get_probabilities() - g["probs"])) < TOL
    mp = np.array([[sv.measure_prob(t, o) for o in (0, 1)] for t in range(n)])
    assert np.max(np.abs(mp - g["measure_prob"])) < TOL
    for ps, pq, pv in zip(g["pauli_strings"], g["pauli_qubits"], g["pauli_values"]):
        qs = [int(q) for q in pq if q >= 0]
        assert abs(sv.expectation_value_pauli(str(ps)[: len(qs)], qs) - pv) < TOL
    # same mt19937_64 stream: the shots agree index for index (the CDF is summed
    # in a different order, so a shot landing within ~1e-16 of a boundary could
    # differ; none does for these fixtures)
    assert np.array_equal(sv.sample(4096, 7), g["samples"])
    assert np.array_equal(sv.sample(1000, 42), g["samples_seed42"])
    for es, ev in zip(g["entropy_sets"], g["entropy"]):
        qs = [int(q) for q in es if q >= 0]
        assert abs(sv.von_neumann_entropy(qs) - ev) < 1e-9
    assert sv.measure(3, 0.3) == int(g["measure_outcome"])
    assert np.max(np.abs(sv.get_amplitudes() - g["amps_after_measure"])) < TOL
    sv.reset_qubit(5, 0.7)
    assert np.max(np.abs(sv.get_amplitudes() - g["amps_after_reset"])) < TOL


def test_golden_special_cases(SV, golden):
    g = golden("sv_readout")
    H = np.array([[1, 1], [1, -1]], np.complex128) / math.sqrt(2)
    b = SV(2)
    b.apply_1q(0, H)
    b.apply_2q(0, 1, CX)
    assert np.max(np.abs(b.get_amplitudes() - g["bell_amps"])) < TOL
    assert abs(b.von_neumann_entropy([0]) - float(g["bell_entropy"])) < 1e-12
    c = SV(3)
    c.apply_1q(0, X)
    c.apply_1q(1, X)
    ccx = np.eye(8, dtype=np.complex128)
    ccx[6, 6] = ccx[7, 7] = 0
    ccx[6, 7] = ccx[7, 6] = 1
    c.apply_fused([0, 1, 2], ccx)   # LSB-first local index, as the reference ABI
    assert np.max(np.abs(c.get_amplitudes() - g["ccx_amps"])) < TOL


@pytest.mark.parametrize("n,seed,eager", [(7, 0, 0), (9, 1, 0), (12, 2, 0), (14, 3, 0), (17, 4, 0), (20, 5, 0),
                                          (12, 6, 1), (20, 7, 1)])
def test_random_sequences_vs_oracle(SV, port, n, seed, eager):
    rng = np.random.default_rng(seed)
    ops = gen_ops(rng, n, 120, kmax=4)
    ref = port.zero_state(n)
    ref = oracle_apply(port, ref, n, ops)
    sv = SV(n)
    sv.set_option("eager", eager)
    apply_abi(sv, ops)
    got = sv.get_amplitudes()
    assert np.max(np.abs(got - ref)) < TOL
    assert abs(sv.norm_squared() - 1.0) < 1e-12


@pytest.mark.parametrize("M,c,budget,stages,nbuf", [(12, 5, 80, 8, 3), (11, 6, 40, 4, 2), (13, 5, 200, 8, 1),
                                                    (10, 5, 16, 2, 4), (12, 7, 500, 16, 2), (11, 3, 120, 8, 3),
                                                    (12, 3, 80, 6, 3), (11, 4, 120, 8, 3)])
def test_tile_configurations(SV, port, M, c, budget, stages, nbuf):
    n = 18
    rng = np.random.default_rng(M * 100 + c)
    ops = gen_ops(rng, n, 150, kmax=4)
    ref = oracle_apply(port, port.zero_state(n), n, ops)
    sv = SV(n)
    for k, v in (("tile_bits", M), ("chunk_bits", c), ("budget", budget), ("max_stages", stages), ("nbuf", nbuf)):
        sv.set_option(k, v)
    apply_abi(sv, ops)
    assert np.max(np.abs(sv.get_amplitudes() - ref)) < TOL


@pytest.mark.parametrize("n,M,c,budget,stages,nbuf", [(9, 11, 5, 80, 8, 3), (16, 11, 5, 80, 8, 3),
                                                      (18, 10, 5, 40, 6, 2), (18, 12, 6, 120, 8, 2)])
def test_three_register_slots(SV, port, n, M, c, budget, stages, nbuf):
    """The 256-thread R = 3 tile kernel (operations of width <= 3) against the oracle."""
    rng = np.random.default_rng(n * 7 + M)
    ops = gen_ops(rng, n, 150, kmax=3)
    ref = oracle_apply(port, port.zero_state(n), n, ops)
    sv = SV(n)
    for k, v in (("reg_slots", 3), ("tile_bits", M), ("chunk_bits", c), ("budget", budget), ("max_stages", stages),
                 ("nbuf", nbuf)):
        sv.set_option(k, v)
    assert sv.get_option("reg_slots") == 3
    apply_abi(sv, ops)
    assert np.max(np.abs(sv.get_amplitudes() - ref)) < TOL


def test_five_qubit_blocks(SV):
    """k = 5 fused blocks (the reference stops at 4) against a numpy contraction."""
    from tests.test_scheduler_emulated import apply_lsb_numpy
    n = 14
    rng = np.random.default_rng(11)
    ref = np.zeros(1 << n, np.complex128)
    ref[0] = 1
    sv = SV(n)
    for _ in range(12):
        qs = [int(x) for x in rng.choice(n, 5, replace=False)]
        U = rand_unitary(rng, 32)
        ref = apply_lsb_numpy(ref, n, qs, U)
        sv.apply_fused(qs, U)
        q = int(rng.integers(n))
        V = rand_unitary(rng, 2)
        ref = apply_lsb_numpy(ref, n, [q], V)
        sv.apply_1q(q, V)
    assert np.max(np.abs(sv.get_amplitudes() - ref)) < TOL


def test_reductions_vs_oracle(SV, port):
    n = 16
    rng = np.random.default_rng(3)
    ops = gen_ops(rng, n, 60, kmax=3)
    ref = oracle_apply(port, port.zero_state(n), n, ops)
    sv = SV(n)
    apply_abi(sv, ops)
    p = np.abs(ref) ** 2
    z = np.array([p[((np.arange(1 << n) >> q) & 1) == 0].sum() - p[((np.arange(1 << n) >> q) & 1) == 1].sum()
                  for q in range(n)])
    assert np.max(np.abs(sv.expval_z_all() - z)) < 1e-12
    for t in (0, 5, 15):
        for o in (0, 1):
            assert abs(sv.measure_prob(t, o) - port.measure_prob(ref, n, t, o)) < 1e-12
    for s, qs in (("XYZ", [0, 7, 15]), ("ZZ", [3, 4]), ("YY", [2, 9]), ("XIZY", [1, 2, 3, 11])):
        assert abs(sv.expectation_value_pauli(s, qs) - port.expval_pauli(ref, n, s, qs)) < 1e-12
    # Pauli sums (exact) against numpy
    coeffs = [0.5, -1.25]
    strs = ["Z" + "I" * (n - 2) + "Z", "X" * 3 + "I" * (n - 3)]
    exp = sum(c * port.expval_pauli(ref, n, s.replace("I", ""), [q for q, ch in enumerate(s) if ch != "I"])
              for c, s in zip(coeffs, strs))
    assert abs(sv.expval_pauli_sum(coeffs, strs) - exp) < 1e-11
    # sampling: chi-squared against the exact probabilities (bins with >= 5 expected merged)
    shots = 20000
    smp = sv.sample(shots, 123)
    from tests.stats import chi2_ok
    assert chi2_ok(smp, p, shots)


def test_measure_reset_collapse(SV, port):
    n = 10
    rng = np.random.default_rng(9)
    ops = gen_ops(rng, n, 40, kmax=2)
    ref = oracle_apply(port, port.zero_state(n), n, ops)
    sv = SV(n)
    apply_abi(sv, ops)
    for t, r in ((2, 0.2), (7, 0.9), (4, 0.5)):
        o_ref = port.measure(ref, n, t, r)
        assert sv.measure(t, r) == o_ref
        assert np.max(np.abs(sv.get_amplitudes() - ref)) < TOL
    port.reset_qubit(ref, n, 1, 0.8)
    sv.reset_qubit(1, 0.8)
    assert np.max(np.abs(sv.get_amplitudes() - ref)) < TOL


def test_errors_are_reported_not_fatal(SV):
    sv = SV(4)
    with pytest.raises(ValueError):
        sv.apply_1q(4, np.eye(2))
    with pytest.raises(ValueError):
        sv.apply_2q(1, 1, np.eye(4))
    with pytest.raises(ValueError):
        sv.apply_fused([0, 1, 2, 3, 0, 1], np.eye(64))
    with pytest.raises(ValueError):
        sv.expectation_value_pauli("Z", [9])
    # the state is untouched by the rejected calls
    a = sv.get_amplitudes()
    assert a[0] == 1 and np.count_nonzero(a) == 1
    # a zero-probability collapse raises instead of aborting the process
    # (the reference throws through extern "C" here): |0>, rand >= p0 = 1
    z = SV(1)
    with pytest.raises(RuntimeError):
        z.measure(0, 1.5)
    assert z.get_amplitudes()[0] == 1


def test_brickwall_20q_vs_reference_core(SV, port):
    """The 20-qubit depth-20 brick-wall (590 gates): amplitudes, probabilities,
    <Z_i> for every qubit and 8192 shots against the reference."""
    from invariantq_b200.circuits import brickwall
    from invariantq_b200.simulator import apply_gate_matrix
    from tests.stats import chi2_ok
    n, depth = 20, 20
    c = brickwall(n, depth, seed=0)
    try:
        from oracle.oracle import RefCore
        ref_sv = RefCore().sv(n)
    except FileNotFoundError:
        ref_sv = None
    sv = SV(n)
    ref = port.zero_state(n)
    for op in c.ops:
        qs = [c.get_qubit_index(q) for q in op.qubits]
        apply_gate_matrix(sv, qs, op.matrix)
        if ref_sv is not None:
            (ref_sv.apply_1q(qs[0], op.matrix) if len(qs) == 1 else ref_sv.apply_2q(qs[0], qs[1], op.matrix))
        else:
            (port.apply_1q(ref, n, qs[0], op.matrix) if len(qs) == 1 else port.apply_2q(ref, n, qs[0], qs[1],
                                                                                       op.matrix))
    if ref_sv is not None:
        ref = ref_sv.amplitudes()
    got = sv.get_amplitudes()
    assert np.max(np.abs(got - ref)) < TOL
    p = np.abs(ref) ** 2
    assert np.max(np.abs(sv.get_probabilities() - p)) < TOL
    bits = (np.arange(1 << n)[:, None] >> np.arange(n)[None, :]) & 1
    z = (p[:, None] * (1 - 2 * bits)).sum(0)
    assert np.max(np.abs(sv.expval_z_all() - z)) < 1e-12
    shots = sv.sample(8192, 11)
    assert chi2_ok(shots, p, 8192)
    if ref_sv is not None:
        same = np.mean(shots == ref_sv.sample(8192, 11))
        assert same > 0.999


def test_brickwall_24q_depth40_vs_reference_core(SV):
    """The 30-qubit workload's parity instance: 24 qubits, depth 40 (1420 gates)."""
    from oracle.oracle import RefCore
    from invariantq_b200.circuits import brickwall
    from invariantq_b200.simulator import apply_gate_matrix
    try:
        core = RefCore()
    except FileNotFoundError:
        pytest.skip("reference core not built (make -C oracle ref)")
    n, depth = 24, 40
    c = brickwall(n, depth, seed=0)
    ref_sv = core.sv(n)
    sv = SV(n)
    for op in c.ops:
        qs = [c.get_qubit_index(q) for q in op.qubits]
        apply_gate_matrix(sv, qs, op.matrix)
        (ref_sv.apply_1q(qs[0], op.matrix) if len(qs) == 1 else ref_sv.apply_2q(qs[0], qs[1], op.matrix))
    err = np.max(np.abs(sv.get_amplitudes() - ref_sv.amplitudes()))
    assert err < TOL, err


def test_30q_properties():
    """Full size (16 GiB state): the depth-40 brick-wall keeps the norm, and the
    circuit followed by its inverse returns |0...0> (size-independent checks)."""
    from invariantq_b200.binding import NativeStateVector
    from invariantq_b200.circuits import brickwall
    from invariantq_b200.simulator import apply_gate_matrix
    n = 30
    c = brickwall(n, 40, seed=0)
    sv = NativeStateVector(n)
    gates = [([c.get_qubit_index(q) for q in op.qubits], op.matrix) for op in c.ops]
    for qs, m in gates:
        apply_gate_matrix(sv, qs, m)
    assert abs(sv.norm_squared() - 1.0) < 1e-10
    for qs, m in reversed(gates):
        apply_gate_matrix(sv, qs, np.conj(m).T)
    assert abs(sv.measure_prob(0, 0) - 1.0) < 1e-10
    z = sv.expval_z_all()
    assert np.max(np.abs(z - 1.0)) < 1e-9
    sv.close()

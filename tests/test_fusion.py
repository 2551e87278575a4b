"""CPU checks of the k-qubit fusion pass (invariantq_b200/fusion.py): for
k = 1..5 the fused circuit applied by the oracle equals the unfused circuit
(1e-12 max-abs), blocks never exceed k wires, and non-unitary operations keep
their place relative to the gates on their wires."""
import numpy as np
import pytest

from invariantq_b200.circuits import brickwall
from invariantq_b200.fusion import GateFusionPass, embed_lsb, msb_to_lsb
from invariantq_b200.ir import BarrierOp, CircuitIR, GateOp, MeasureOp, QWire
from tests.test_scheduler_emulated import apply_lsb_numpy

TOL = 1e-12


def apply_circuit(port, c, n):
    """Every op through the oracle in the C ABI's convention of its width."""
    s = port.zero_state(n)
    for op in c.ops:
        kind = type(op).__name__
        if kind not in ("GateOp", "FusedGateOp"):
            continue
        qs = [c.get_qubit_index(q) for q in op.qubits]
        m = np.asarray(op.matrix if kind == "GateOp" else op.fused_matrix, np.complex128)
        if kind == "GateOp" and len(qs) >= 3:   # gate matrices are MSB-first over the listed wires
            qs, m = list(reversed(qs)), m
        if len(qs) == 1:
            assert port.apply_1q(s, n, qs[0], m) == 0
        elif len(qs) == 2:
            assert port.apply_2q(s, n, qs[0], qs[1], m) == 0
        elif len(qs) <= 4:
            assert port.apply_fused(s, n, qs, m) == 0
        else:
            s[:] = apply_lsb_numpy(s, n, qs, m)
    return s


def random_circuit(rng, n, ngates):
    c = CircuitIR("rand")
    c.add_qubit_register("q", n)
    for _ in range(ngates):
        g = rng.choice(["u3", "cx", "cz", "swap", "ccx", "h", "rz", "ry"])
        if g in ("u3", "h", "rz", "ry"):
            q = [int(rng.integers(n))]
        elif g == "ccx":
            q = [int(x) for x in rng.choice(n, 3, replace=False)]
        else:
            q = [int(x) for x in rng.choice(n, 2, replace=False)]
        params = {"u3": 3, "rz": 1, "ry": 1}.get(g, 0)
        c.add_op(GateOp(name=g, qubits=[QWire("q", x) for x in q], params=list(rng.uniform(0, 2 * np.pi, params))))
    return c


def test_embed_and_reorder():
    rng = np.random.default_rng(0)
    u = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))[0]
    # embedding on the same wires is the identity map; a wire permutation is a basis permutation
    assert np.allclose(embed_lsb(u, [3, 5], [3, 5]), u)
    v = embed_lsb(u, [3, 5], [5, 3])
    assert np.allclose(v, msb_to_lsb(u))
    big = embed_lsb(u, [1, 0], [0, 1, 2])      # u on wires 0, 1 (swapped), identity on wire 2
    assert np.allclose(big, np.kron(np.eye(2), msb_to_lsb(u)))


@pytest.mark.parametrize("n,seed", [(5, 1), (7, 2), (9, 3)])
@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_random_circuits(port, n, seed, k):
    rng = np.random.default_rng(seed * 10 + k)
    c = random_circuit(rng, n, 120)
    f = GateFusionPass(k).run(c)
    assert len(f.ops) <= len(c.ops)
    for op in f.ops:
        if type(op).__name__ == "FusedGateOp":
            assert len(op.qubits) <= k
            m = op.fused_matrix
            assert np.allclose(m @ m.conj().T, np.eye(m.shape[0]), atol=1e-12)
    ref = apply_circuit(port, c, n)
    got = apply_circuit(port, f, n)
    assert np.max(np.abs(got - ref)) < TOL


@pytest.mark.parametrize("k,max_blocks", [(2, 400), (3, 330), (4, 250), (5, 230)])
def test_brickwall_blocks(port, k, max_blocks):
    """20-qubit depth-20 brick-wall (590 gates): fewer blocks as k grows, same state."""
    n = 12
    c = brickwall(n, 20, seed=0)
    f = GateFusionPass(k).run(c)
    nblocks = len(f.ops)
    assert nblocks < len(c.ops)
    widths = [len(op.qubits) for op in f.ops]
    assert max(widths) <= k
    assert np.max(np.abs(apply_circuit(port, f, n) - apply_circuit(port, c, n))) < TOL


def test_measure_and_barrier_keep_order():
    n = 3
    c = CircuitIR("m")
    c.add_qubit_register("q", n)
    c.add_clbit_register("c", n)
    w = [QWire("q", i) for i in range(n)]
    c.add_op(GateOp(name="h", qubits=[w[0]]))
    c.add_op(GateOp(name="cx", qubits=[w[0], w[1]]))
    c.add_op(MeasureOp(qubits=[w[1]]))
    c.add_op(GateOp(name="x", qubits=[w[1]]))
    c.add_op(GateOp(name="h", qubits=[w[2]]))
    c.add_op(BarrierOp(qubits=list(w)))
    c.add_op(GateOp(name="cz", qubits=[w[1], w[2]]))
    f = GateFusionPass(3).run(c)
    kinds = [type(op).__name__ for op in f.ops]
    im = kinds.index("MeasureOp")
    ib = kinds.index("BarrierOp")
    # the h+cx block on wires 0,1 precedes the measurement; x on wire 1 follows it
    before = f.ops[:im]
    assert any(set(c.get_qubit_index(q) for q in op.qubits) >= {0, 1} for op in before)
    assert ib > im
    after_barrier = f.ops[ib + 1:]
    assert len(after_barrier) == 1 and [c.get_qubit_index(q) for q in after_barrier[0].qubits] == [1, 2]
    # original ops are not modified
    assert [op.id for op in c.ops] == list(range(7))


def test_rejects_bad_width():
    with pytest.raises(ValueError):
        GateFusionPass(6)

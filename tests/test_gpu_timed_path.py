"""Parity of the exact configurations the benchmark times.

The 30-qubit benchmark records the depth-40 brick-wall as a device-resident
program whose passes all run as specialised (run-time compiled) pass kernels.
These tests record the 24-qubit instance of the same generator the same way and
compare the final amplitudes with the reference core (oracle/_ref, the
reference's own C++ kernels, one gate at a time: statevector.cpp:26-87) at
1e-12 max-abs, asserting that every pass of every run went through a
specialised kernel:

* the library's default plan and the fewer-passes plan (3 chunk qubits,
  budget 160);
* the circuit fused by GateFusionPass at k = 2..5 (fused k-qubit blocks through
  iq_statevector_apply_fused, the k-sweep the benchmark reports);
* a 10-qubit noisy density-matrix program (20 index bits) with jit = 2 against
  the reference core's density-matrix kernels (density_matrix.cpp:18-163).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def ref24():
    from invariantq_b200.circuits import brickwall
    from oracle.oracle import RefCore
    try:
        core = RefCore()
    except FileNotFoundError:
        pytest.skip("reference core not built (make -C oracle ref)")
    n, depth = 24, 40
    c = brickwall(n, depth, seed=0)
    sv = core.sv(n)
    for op in c.ops:
        qs = [c.get_qubit_index(q) for q in op.qubits]
        (sv.apply_1q(qs[0], op.matrix) if len(qs) == 1 else sv.apply_2q(qs[0], qs[1], op.matrix))
    return c, sv.amplitudes()


def _run_recorded(c_ops, n, opts, fused=None):
    """Record the operations as a program on a fresh handle with `opts`, run it
    from |0...0> and return (amplitudes, program passes, specialised passes of
    the run, tile passes of the run)."""
    from invariantq_b200.binding import NativeStateVector
    from invariantq_b200.simulator import apply_gate_matrix
    sv = NativeStateVector(n)
    try:
        for k, v in opts.items():
            sv.set_option(k, v)
        with sv.record() as rec:
            for qs, m, is_fused in c_ops:
                if is_fused:
                    sv.apply_fused(qs, m)
                else:
                    apply_gate_matrix(sv, qs, m)
        prog = rec.program
        sv.reset()
        s0 = sv.stats()
        prog.run(sv)
        amps = sv.get_amplitudes()
        s1 = sv.stats()
        return amps, prog.passes, s1["jit_passes"] - s0["jit_passes"], s1["tile_passes"] - s0["tile_passes"]
    finally:
        sv.close()


def _plain_ops(c):
    return [([c.get_qubit_index(q) for q in op.qubits], np.asarray(op.matrix, np.complex128), False) for op in c.ops]


@pytest.mark.parametrize("opts", [{}, {"chunk_bits": 3, "budget": 160}, {"chunk_bits": 5, "budget": 120},
                                  {"jit": 2}],
                         ids=["library-default", "chunk3-budget160", "chunk5-budget120", "jit2"])
def test_brickwall_24q_recorded_program_vs_reference(ref24, opts):
    c, ref = ref24
    amps, passes, jit_passes, tile_passes = _run_recorded(_plain_ops(c), 24, opts)
    assert passes > 0 and jit_passes == passes == tile_passes
    err = float(np.max(np.abs(amps - ref)))
    assert err < TOL, err


@pytest.mark.parametrize("policy", ["dense", "cost"])
@pytest.mark.parametrize("k", [2, 3, 4, 5])
def test_fusion_pass_blocks_24q_vs_reference(ref24, k, policy):
    """GateFusionPass(k) output recorded and run with specialised kernels, its
    blocks applied as dense k-qubit matrices in the ABI's convention ('dense')
    or as the driver chooses per block ('cost': dense matrix or original gates)."""
    from invariantq_b200.fusion import GateFusionPass
    from invariantq_b200.simulator import fused_block_choice
    c, ref = ref24
    f = GateFusionPass(k).run(c)
    ops = []
    nfused = 0
    for op in f.ops:
        qs = [f.get_qubit_index(q) for q in op.qubits]
        if type(op).__name__ == "FusedGateOp":
            if policy == "cost" and fused_block_choice(op) == "originals":
                for o in op.original_ops:
                    ops.append(([f.get_qubit_index(q) for q in o.qubits], np.asarray(o.matrix, np.complex128), False))
            else:
                ops.append((qs, np.asarray(op.fused_matrix, np.complex128), True))
                nfused += 1
        else:
            ops.append((qs, np.asarray(op.matrix, np.complex128), False))
    assert nfused > 0
    amps, passes, jit_passes, tile_passes = _run_recorded(ops, 24, {"jit": 2})
    assert passes > 0 and jit_passes == passes == tile_passes
    err = float(np.max(np.abs(amps - ref)))
    assert err < TOL, (k, err)


def test_noisy_density_matrix_program_jit2_vs_reference():
    """10-qubit noisy brick-wall (the 14-qubit workload's channel mix) recorded
    as a density-matrix program with jit = 2: elements, trace and purity against
    the reference core."""
    from invariantq_b200.binding import NativeDensityMatrix
    from invariantq_b200.channels import build_kraus_channel
    from invariantq_b200.circuits import noisy_brickwall
    from oracle.oracle import RefCore
    try:
        core = RefCore()
    except FileNotFoundError:
        pytest.skip("reference core not built (make -C oracle ref)")
    n, depth = 10, 4
    c = noisy_brickwall(n, depth, seed=3)
    dep = build_kraus_channel("depolarizing", [1e-3])
    ref = core.dm(n)
    dm = NativeDensityMatrix(n)
    dm.set_option("jit", 2)
    with dm.record() as rec:
        for op in c.ops:
            qs = [c.get_qubit_index(q) for q in op.qubits]
            if type(op).__name__ == "GateOp":
                if len(qs) == 1:
                    ref.apply_1q(qs[0], op.matrix)
                    dm.apply_1q_unitary(qs[0], op.matrix)
                    ref.apply_kraus_1q(qs[0], dep)
                    dm.apply_1q_kraus(qs[0], dep)
                else:
                    ref.apply_2q(qs[0], qs[1], op.matrix)
                    dm.apply_2q_unitary(qs[0], qs[1], op.matrix)
            else:
                K = build_kraus_channel(op.channel_name, op.params)
                for q in qs:
                    ref.apply_kraus_1q(q, K)
                    dm.apply_1q_kraus(q, K)
    prog = rec.program
    dm.reset()
    s0 = dm.stats()
    prog.run(dm)
    rho = dm.get_matrix()
    s1 = dm.stats()
    assert s1["jit_passes"] - s0["jit_passes"] == prog.passes == s1["tile_passes"] - s0["tile_passes"]
    rho_ref = ref.matrix()
    assert np.max(np.abs(rho - rho_ref)) < TOL
    assert abs(dm.trace() - ref.trace()) < TOL
    assert abs(dm.purity() - ref.purity()) < TOL
    dm.close()

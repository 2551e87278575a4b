"""CPU check of the gate scheduler and the tile-pass descriptor semantics.

tests/plan_emulator.cpp runs the passes planned by invariantq_b200/csrc/
iq_sched.cpp with the kernel's semantics (tensor-map boxes from the shared
addressing helpers, octet lanes, register slots).  Random gate sequences are
applied both ways and compared with the C oracle, which applies the reference
kernels one call at a time."""
import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="session")
def emu(tmp_path_factory):
    out = tmp_path_factory.mktemp("emu") / "libplanemu.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(out),
                    str(REPO / "tests" / "plan_emulator.cpp"),
                    str(REPO / "invariantq_b200" / "csrc" / "iq_sched.cpp"),
                    str(REPO / "invariantq_b200" / "csrc" / "iq_jitgen.cpp")], check=True)
    L = ctypes.CDLL(str(out))
    L.emu_apply.restype = ctypes.c_int
    return L


def rand_unitary(rng, d):
    z = (rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


CX = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], np.complex128)
CZ = np.diag([1, 1, 1, -1]).astype(np.complex128)
SWAP = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], np.complex128)
X = np.array([[0, 1], [1, 0]], np.complex128)
S = np.diag([1, 1j])


def gen_ops(rng, n, nops, kmax=4, mono_frac=0.3):
    """ABI-level ops: (kind, qubits, U) with kind in {1q, 2q, fused}."""
    ops = []
    for _ in range(nops):
        k = int(rng.integers(1, kmax + 1))
        k = min(k, n)
        qs = [int(x) for x in rng.choice(n, size=k, replace=False)]
        if k == 1:
            U = [X, S, np.diag([np.exp(1j * 0.3), np.exp(-0.7j)])][int(rng.integers(3))] \
                if rng.random() < mono_frac else rand_unitary(rng, 2)
            ops.append(("1q", qs, U))
        elif k == 2:
            U = [CX, CZ, SWAP][int(rng.integers(3))] if rng.random() < mono_frac else rand_unitary(rng, 4)
            ops.append(("2q" if rng.random() < 0.7 else "fused", qs, U))
        else:
            ops.append(("fused", qs, rand_unitary(rng, 1 << k)))
    return ops


def to_lsb(kind, qs, U):
    """The runtime's conversion to the internal LSB-first convention."""
    if len(qs) == 2:             # apply_2q and fused k=2: qs[0] is the MSB
        return [qs[1], qs[0]], U
    return list(qs), U


def apply_lsb_numpy(state, n, qs, U):
    k = len(qs)
    t = state.reshape([2] * n, order="F")
    rest = [q for q in range(n) if q not in qs]
    # local index bit i <-> qs[i]: in Fortran order axis qs[0] varies fastest
    moved = np.transpose(t, list(qs) + rest).reshape(1 << k, -1, order="F")
    out = (U @ moved).reshape([2] * n, order="F")
    return np.transpose(out, np.argsort(list(qs) + rest)).reshape(-1, order="F")


def run_emu(emu, n, lsb_ops, state, M=12, c=5, R=4, max_stages=8, budget=80.0, fuse=1):
    nops = len(lsb_ops)
    ks = np.array([len(q) for q, _ in lsb_ops], dtype=np.int32)
    qs = np.full((nops, 5), -1, dtype=np.int32)
    offs = np.zeros(nops, dtype=np.int64)
    pool = []
    off = 0
    for i, (q, U) in enumerate(lsb_ops):
        qs[i, : len(q)] = q
        offs[i] = off
        flat = np.asarray(U, np.complex128).reshape(-1)
        pool.append(flat)
        off += flat.size
    pool = np.concatenate(pool) if pool else np.zeros(1, np.complex128)
    st = np.ascontiguousarray(state.copy())
    npasses = ctypes.c_int(0)
    per = np.zeros(max(nops, 1), dtype=np.int32)
    err = ctypes.create_string_buffer(512)
    rc = emu.emu_apply(n, M, c, R, max_stages, ctypes.c_double(budget), fuse, nops,
                       ks.ctypes.data_as(ctypes.c_void_p), qs.ctypes.data_as(ctypes.c_void_p),
                       pool.ctypes.data_as(ctypes.c_void_p), offs.ctypes.data_as(ctypes.c_void_p),
                       st.ctypes.data_as(ctypes.c_void_p), ctypes.byref(npasses),
                       per.ctypes.data_as(ctypes.c_void_p), err, 512)
    assert rc == 0, err.value.decode()
    return st, npasses.value, per[: npasses.value]


def oracle_apply(port, state, n, ops):
    for kind, qs, U in ops:
        if kind == "1q":
            assert port.apply_1q(state, n, qs[0], U) == 0
        elif kind == "2q":
            assert port.apply_2q(state, n, qs[0], qs[1], U) == 0
        elif len(qs) <= 4:
            assert port.apply_fused(state, n, qs, U) == 0
        else:
            state[:] = apply_lsb_numpy(state, n, qs, U)
    return state


@pytest.mark.parametrize("n,M,c,R,stages,budget,seed", [
    (7, 12, 5, 4, 8, 80.0, 0),      # whole array is one tile
    (8, 12, 5, 4, 8, 80.0, 1),
    (10, 10, 5, 4, 8, 80.0, 2),     # exactly one tile of 2^10
    (12, 10, 5, 4, 4, 40.0, 3),     # several tiles
    (13, 11, 6, 4, 6, 60.0, 4),
    (14, 12, 5, 4, 8, 80.0, 5),
    (15, 12, 7, 4, 3, 30.0, 6),
    (16, 13, 5, 4, 8, 200.0, 7),
    (14, 12, 5, 5, 8, 500.0, 8),    # five register slots
    (10, 10, 5, 3, 8, 80.0, 9),     # three register slots (256-thread variant)
    (13, 11, 5, 3, 6, 60.0, 10),
    (14, 11, 6, 3, 8, 120.0, 11),
    (14, 11, 3, 4, 8, 120.0, 12),   # three chunk bits: more high tile bits per pass
    (15, 12, 3, 4, 6, 80.0, 13),
    (13, 11, 4, 4, 8, 96.0, 14),
])
def test_emulated_passes_match_oracle(port, emu, n, M, c, R, stages, budget, seed):
    rng = np.random.default_rng(seed)
    ops = gen_ops(rng, n, 80, kmax=R)
    ref = np.zeros(1 << n, np.complex128)
    ref[0] = 1
    # start from a random state so every amplitude matters
    ref = rand_unitary(rng, 1 << min(n, 6))[:, 0].repeat(1 << (n - min(n, 6)))
    ref = ref / np.linalg.norm(ref)
    start = ref.copy()
    ref = oracle_apply(port, ref, n, ops)
    lsb = [to_lsb(*o) for o in ops]
    # fuse 2: the specialised kernels' planning (CX/CZ/SWAP apart, normalised one-qubit gates)
    for fuse in (0, 1, 2):
        got, npasses, per = run_emu(emu, n, lsb, start, M=M, c=c, R=R, max_stages=stages, budget=budget, fuse=fuse)
        assert fuse == 2 or per.sum() <= len(ops)    # style 2 splits one-qubit gates into rotations and phases
        assert fuse or per.sum() == len(ops)
        assert np.max(np.abs(got - ref)) < 1e-12


def brickwall_ops(n, depth, seed):
    from invariantq_b200.gates import gate_matrix
    rng = np.random.default_rng(seed)
    ang = rng.uniform(0, 2 * np.pi, size=(depth, n, 3))
    ops = []
    for l in range(depth):
        for q in range(n):
            ops.append(("1q", [q], gate_matrix("u3", ang[l, q])))
        for q in range(l % 2, n - 1, 2):
            ops.append(("2q", [q, q + 1], CX))
    return ops


def test_brickwall_pass_count_and_parity(port, emu):
    n, depth = 16, 8
    ops = brickwall_ops(n, depth, 0)
    ref = np.zeros(1 << n, np.complex128)
    ref[0] = 1
    start = ref.copy()
    ref = oracle_apply(port, ref, n, ops)
    for fuse in (1, 2):
        got, npasses, per = run_emu(emu, n, [to_lsb(*o) for o in ops], start, M=12, c=5, fuse=fuse)
        assert np.max(np.abs(got - ref)) < 1e-12
        # far fewer passes than gates
        assert npasses < len(ops) / 4


def test_normalisation_segments_keep_scale(port, emu):
    """More dense one-qubit gates than one normalisation run (kNormSegment =
    256): every run's carrier restores the scale before the state is read."""
    n = 9
    rng = np.random.default_rng(21)
    ops = []
    for _ in range(700):   # a CZ after every gate keeps the one-qubit gates from merging
        q = int(rng.integers(n))
        ops += [("1q", [q], rand_unitary(rng, 2)), ("2q", [q, (q + 1) % n], CZ)]
    ops += [("2q", [0, 5], CX), ("1q", [3], rand_unitary(rng, 2))]
    ref = np.zeros(1 << n, np.complex128)
    ref[0] = 1
    start = ref.copy()
    ref = oracle_apply(port, ref, n, ops)
    got, npasses, per = run_emu(emu, n, [to_lsb(*o) for o in ops], start, M=9, c=5, budget=1e9, fuse=2)
    assert np.max(np.abs(got - ref)) < 1e-12
    assert abs(np.linalg.norm(got) - 1.0) < 1e-12


@pytest.mark.parametrize("R", [3, 4])
def test_brickwall_register_slots(port, emu, R):
    """The brick-wall planned with 3 and 4 register slots gives the oracle's state."""
    n, depth = 15, 6
    ops = brickwall_ops(n, depth, 1)
    ref = np.zeros(1 << n, np.complex128)
    ref[0] = 1
    start = ref.copy()
    ref = oracle_apply(port, ref, n, ops)
    got, npasses, per = run_emu(emu, n, [to_lsb(*o) for o in ops], start, M=11, c=5, R=R)
    assert np.max(np.abs(got - ref)) < 1e-12


def superop_lsb(kraus):
    """sum_k K (x) conj(K) on the local bits (column bit, row bit): local index
    bit 0 = the column qubit, bit 1 = the row qubit (the runtime's dm_kraus)."""
    S = np.zeros((4, 4), np.complex128)
    for K in kraus:
        for ro in range(2):
            for co in range(2):
                for ri in range(2):
                    for ci in range(2):
                        S[ro * 2 + co, ri * 2 + ci] += K[ro, ri] * np.conj(K[co, ci])
    return S


def plan_kinds(emu, nbits, lsb_ops, M, c, fuse=2):
    nops = len(lsb_ops)
    ks = np.array([len(q) for q, _ in lsb_ops], dtype=np.int32)
    qs = np.full((nops, 5), -1, dtype=np.int32)
    offs = np.zeros(nops, dtype=np.int64)
    pool, off = [], 0
    for i, (q, U) in enumerate(lsb_ops):
        qs[i, : len(q)] = q
        offs[i] = off
        pool.append(np.asarray(U, np.complex128).reshape(-1))
        off += pool[-1].size
    pool = np.concatenate(pool)
    buf = ctypes.create_string_buffer(16 << 20)
    rc = emu.emu_plan_dump(nbits, M, c, 4, 8, ctypes.c_double(160.0), fuse, nops,
                           ks.ctypes.data_as(ctypes.c_void_p), qs.ctypes.data_as(ctypes.c_void_p),
                           pool.ctypes.data_as(ctypes.c_void_p), offs.ctypes.data_as(ctypes.c_void_p),
                           buf, ctypes.c_longlong(len(buf)))
    assert rc > 0
    return buf.value.decode()


@pytest.mark.parametrize("nq,M,c,seed", [(6, 10, 4, 0), (7, 12, 4, 1), (8, 11, 5, 2)])
def test_channel_superoperators_x_pattern(emu, nq, M, c, seed):
    """A noisy density-matrix circuit as the runtime queues it (unitary U on the
    row bit and conj(U) on the column bit, Kraus channels as superoperators on
    the (column, row) bit pair, CX on row and column pairs), planned in the
    specialised-kernel style: the channels' superoperators run as X2R
    operations (only their corners and middle read), and the result equals the
    dense matrices applied one by one (1e-12)."""
    from invariantq_b200.channels import build_kraus_channel
    from invariantq_b200.gates import gate_matrix
    rng = np.random.default_rng(seed)
    nb = 2 * nq
    chans = [build_kraus_channel("depolarizing", [1e-3]), build_kraus_channel("amp_damping", [2e-3]),
             build_kraus_channel("phase_damping", [1e-3]),
             build_kraus_channel("thermal_relaxation", [100e-6, 80e-6, 50e-9])]
    cx = gate_matrix("cx")
    cx_lsb = cx[np.ix_([0, 2, 1, 3], [0, 2, 1, 3])]   # control on local bit 1
    ops = []
    for layer in range(4):
        for q in range(nq):
            U = gate_matrix("u3", list(rng.uniform(0, 2 * np.pi, 3)))
            ops += [([nq + q], U), ([q], np.conj(U)), ([q, nq + q], superop_lsb(chans[0]))]
        for q in range(layer % 2, nq - 1, 2):
            ops += [([nq + q + 1, nq + q], cx_lsb), ([q + 1, q], cx_lsb)]
            for qq in (q, q + 1):
                ops += [([qq, nq + qq], superop_lsb(chans[1])), ([qq, nq + qq], superop_lsb(chans[2]))]
        for q in range(nq):
            ops.append(([q, nq + q], superop_lsb(chans[3])))
    rho = rng.normal(size=1 << nb) + 1j * rng.normal(size=1 << nb)
    want = rho.copy()
    for qs, U in ops:
        want = apply_lsb_numpy(want, nb, qs, U)
    got, npasses, per = run_emu(emu, nb, ops, rho, M=M, c=c, budget=160.0, fuse=2)
    assert np.max(np.abs(got - want)) < 1e-12 * max(1.0, np.max(np.abs(want)))
    dump = plan_kinds(emu, nb, ops, M, c)
    assert "X2R" in dump and "D2R" not in dump

"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run where the reference sources exist (they do not travel to the GPU machine):

    make -C oracle ref            # builds oracle/_ref/libinvariantq.so from the reference sources
    python tests/golden/make_golden.py --reference <reference checkout>
                                        # or IQ_REFERENCE_DIR=<reference checkout>

The script copies the reference's Python package into a temporary directory,
drops the reference core built by ``oracle/Makefile`` next to its ctypes
binding (``invariantq/core/binding.py:15-40`` looks there first), imports it,
and records what the reference's own code returns:

* ``sv_ops.npz``       -- random 1q / 2q / fused-k (k = 3, 4) sequences through
                          ``NativeStateVector`` (binding.py:302-395), final amplitudes.
* ``sv_readout.npz``   -- probabilities, measure_prob, Pauli expectations,
                          sampled shots, entropy, measure / reset collapses.
* ``dm_ops.npz``       -- density-matrix unitaries, every Kraus channel of
                          ``invariantq/noise/channels.py``, reset, measure, trace,
                          purity, entropy (``NativeDensityMatrix`` binding.py:398-476).
* ``gates.npz``        -- the gate-matrix table of ``invariantq/ir/qir.py:67-208``
                          and the Kraus sets of ``channels.py:11-103``.
* ``simulators.npz``   -- ``StateVectorSimulator.run`` / ``DensityMatrixSimulator.run``
                          on seeded circuits (including the brick-wall U3+CX workload).
* ``binding_argtypes.json`` -- the ctypes signature the reference's binding sets on
                          each of the 49 C-ABI functions (binding.py:54-299).
* ``abi_traces.json``  -- every C-ABI call the reference's own tests make
                          (tests/test_core_math.py:10-69,
                          tests/test_independent_reference.py:15-61) when run on
                          the reference core through its unmodified binding and
                          drivers: arguments, and the values the core returned,
                          for a replay against another library.

Every input is seeded; the fixtures are small (kilobytes).
"""
from __future__ import annotations

import argparse
import importlib
import math
import os
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent


def rand_unitary(rng, d):
    z = (rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))) / math.sqrt(2)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def load_reference(ref_dir: Path, tmp: Path):
    lib = REPO / "oracle" / "_ref" / "libinvariantq.so"
    if not lib.exists():
        raise SystemExit("oracle/_ref/libinvariantq.so missing: run `make -C oracle ref` first")
    shutil.copytree(ref_dir / "invariantq", tmp / "invariantq")
    shutil.copy(lib, tmp / "invariantq" / "core" / "libinvariantq.so")
    sys.path.insert(0, str(tmp))
    iq = importlib.import_module("invariantq")
    binding = importlib.import_module("invariantq.core.binding")
    assert binding.HAS_NATIVE_CORE, binding.native_core_status()
    return iq, binding


OP_1Q, OP_2Q, OP_FUSED = 1, 2, 3


def gen_sv_ops(binding, out):
    rng = np.random.default_rng(1234)
    data = {}
    for n in (3, 5, 8, 10):
        nops = 60
        kinds = np.zeros(nops, np.int64)
        qubits = np.full((nops, 4), -1, np.int64)
        mats = np.zeros((nops, 16, 16), np.complex128)
        sv = binding.NativeStateVector(n)
        for i in range(nops):
            kmax = min(n, 4)
            k = int(rng.integers(1, kmax + 1))
            qs = [int(x) for x in rng.choice(n, size=k, replace=False)]
            U = rand_unitary(rng, 1 << k)
            if k == 1:
                kinds[i] = OP_1Q
                sv.apply_1q(qs[0], U)
            elif k == 2 and rng.random() < 0.5:
                kinds[i] = OP_2Q
                sv.apply_2q(qs[0], qs[1], U)
            else:
                kinds[i] = OP_FUSED
                sv.apply_fused(qs, U)
            qubits[i, :k] = qs
            mats[i, : 1 << k, : 1 << k] = U
        data[f"n{n}_kinds"] = kinds
        data[f"n{n}_qubits"] = qubits
        data[f"n{n}_mats"] = mats
        data[f"n{n}_amps"] = sv.get_amplitudes()
    np.savez_compressed(out / "sv_ops.npz", **data)


def gen_sv_readout(binding, out):
    rng = np.random.default_rng(99)
    n = 8
    sv = binding.NativeStateVector(n)
    # a fixed entangling preparation: random 1q layer, CX ladder, random 2q gates
    prep = []
    for q in range(n):
        U = rand_unitary(rng, 2)
        sv.apply_1q(q, U)
        prep.append((1, [q], U))
    CX = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], np.complex128)
    for q in range(n - 1):
        sv.apply_2q(q, q + 1, CX)
        prep.append((2, [q, q + 1], CX))
    for _ in range(6):
        q0, q1 = [int(x) for x in rng.choice(n, 2, replace=False)]
        U = rand_unitary(rng, 4)
        sv.apply_2q(q0, q1, U)
        prep.append((2, [q0, q1], U))
    d = {}
    d["prep_kinds"] = np.array([p[0] for p in prep])
    d["prep_qubits"] = np.array([p[1] + [-1] * (2 - len(p[1])) for p in prep])
    mats = np.zeros((len(prep), 4, 4), np.complex128)
    for i, p in enumerate(prep):
        m = p[2]
        mats[i, : m.shape[0], : m.shape[1]] = m
    d["prep_mats"] = mats
    d["amps"] = sv.get_amplitudes()
    d["probs"] = sv.get_probabilities()
    d["measure_prob"] = np.array([[sv.measure_prob(t, o) for o in (0, 1)] for t in range(n)])
    paulis, pqubits, pvals = [], [], []
    for _ in range(24):
        L = int(rng.integers(1, n + 1))
        qs = [int(x) for x in rng.choice(n, L, replace=False)]
        s = "".join(rng.choice(list("IXYZ"), L))
        paulis.append(s.ljust(n, "-"))
        pqubits.append(qs + [-1] * (n - L))
        pvals.append(sv.expectation_value_pauli(s, qs))
    d["pauli_strings"] = np.array(paulis)
    d["pauli_qubits"] = np.array(pqubits)
    d["pauli_values"] = np.array(pvals)
    d["sample_seed"] = np.array(7)
    d["samples"] = sv.sample(4096, 7)
    d["samples_seed42"] = sv.sample(1000, 42)
    ent_sets = [[0], [1, 2], [0, 3, 5], [7]]
    d["entropy_sets"] = np.array([s + [-1] * (3 - len(s)) for s in ent_sets])
    d["entropy"] = np.array([sv.von_neumann_entropy(s) for s in ent_sets])
    # collapses: measure qubit 3 with rand 0.3, then reset qubit 5 with rand 0.7
    d["measure_outcome"] = np.array(sv.measure(3, 0.3))
    d["amps_after_measure"] = sv.get_amplitudes()
    sv.reset_qubit(5, 0.7)
    d["amps_after_reset"] = sv.get_amplitudes()
    # Bell-state entropy and the fused-3q (LSB-first) convention on a CCX matrix
    b = binding.NativeStateVector(2)
    H = np.array([[1, 1], [1, -1]], np.complex128) / math.sqrt(2)
    b.apply_1q(0, H)
    b.apply_2q(0, 1, CX)
    d["bell_entropy"] = np.array(b.von_neumann_entropy([0]))
    d["bell_amps"] = b.get_amplitudes()
    c = binding.NativeStateVector(3)
    X = np.array([[0, 1], [1, 0]], np.complex128)
    c.apply_1q(0, X)
    c.apply_1q(1, X)
    ccx = np.eye(8, dtype=np.complex128)
    ccx[6, 6] = ccx[7, 7] = 0
    ccx[6, 7] = ccx[7, 6] = 1
    c.apply_fused([0, 1, 2], ccx)
    d["ccx_amps"] = c.get_amplitudes()
    np.savez_compressed(out / "sv_readout.npz", **d)


def gen_dm_ops(iq, binding, out):
    from invariantq.noise.channels import build_kraus_channel  # noqa: E402
    rng = np.random.default_rng(2024)
    channels = [("depolarizing", [0.05]), ("amplitude_damping", [0.1]), ("phase_damping", [0.2]),
                ("bit_flip", [0.07]), ("phase_flip", [0.03]), ("thermal_relaxation", [100e-6, 80e-6, 50e-9]),
                ("thermal_relaxation", [20e-6, 90e-6, 400e-9])]
    d = {}
    for n in (2, 3, 4):
        dm = binding.NativeDensityMatrix(n)
        rec_kind, rec_q, rec_m, rec_nk = [], [], [], []
        for step in range(30):
            r = rng.random()
            if r < 0.35:
                t = int(rng.integers(n))
                U = rand_unitary(rng, 2)
                dm.apply_1q_unitary(t, U)
                rec_kind.append(1); rec_q.append([t, -1]); m = np.zeros((4, 4, 4), np.complex128)
                m[0, :2, :2] = U; rec_m.append(m); rec_nk.append(1)
            elif r < 0.6:
                q0, q1 = [int(x) for x in rng.choice(n, 2, replace=False)]
                U = rand_unitary(rng, 4)
                dm.apply_2q_unitary(q0, q1, U)
                rec_kind.append(2); rec_q.append([q0, q1]); m = np.zeros((4, 4, 4), np.complex128)
                m[0] = U; rec_m.append(m); rec_nk.append(1)
            elif r < 0.95:
                t = int(rng.integers(n))
                name, params = channels[int(rng.integers(len(channels)))]
                K = build_kraus_channel(name, params)
                dm.apply_1q_kraus(t, K)
                rec_kind.append(3); rec_q.append([t, -1]); m = np.zeros((4, 4, 4), np.complex128)
                for j, k in enumerate(K):
                    m[j, :2, :2] = k
                rec_m.append(m); rec_nk.append(len(K))
            else:
                t = int(rng.integers(n))
                dm.reset_qubit(t)
                rec_kind.append(4); rec_q.append([t, -1]); rec_m.append(np.zeros((4, 4, 4), np.complex128))
                rec_nk.append(0)
        d[f"n{n}_kinds"] = np.array(rec_kind)
        d[f"n{n}_qubits"] = np.array(rec_q)
        d[f"n{n}_mats"] = np.array(rec_m)
        d[f"n{n}_nkraus"] = np.array(rec_nk)
        d[f"n{n}_rho"] = dm.get_matrix()
        d[f"n{n}_trace"] = np.array(dm.trace())
        d[f"n{n}_purity"] = np.array(dm.purity())
        d[f"n{n}_entropy"] = np.array(dm.von_neumann_entropy())
        o = dm.measure(0, 0.4)
        d[f"n{n}_measure_outcome"] = np.array(o)
        d[f"n{n}_rho_after_measure"] = dm.get_matrix()
    np.savez_compressed(out / "dm_ops.npz", **d)


def gen_gates(iq, out):
    from invariantq.ir.qir import GateOp, QWire  # noqa: E402
    from invariantq.noise.channels import build_kraus_channel  # noqa: E402
    d = {}
    q = [QWire("q", 0), QWire("q", 1), QWire("q", 2)]
    fixed = ["i", "id", "x", "y", "z", "h", "s", "sdg", "t", "tdg", "cx", "cnot", "cy", "cz", "ch", "iswap",
             "swap", "ccx", "toffoli", "cswap", "fredkin"]
    arity = {"cx": 2, "cnot": 2, "cy": 2, "cz": 2, "ch": 2, "iswap": 2, "swap": 2, "ccx": 3, "toffoli": 3,
             "cswap": 3, "fredkin": 3}
    for name in fixed:
        d[f"gate_{name}"] = GateOp(name=name, qubits=q[: arity.get(name, 1)]).matrix
    rng = np.random.default_rng(5)
    for name, npar, ar in [("rx", 1, 1), ("ry", 1, 1), ("rz", 1, 1), ("p", 1, 1), ("phase", 1, 1), ("u3", 3, 1),
                           ("crx", 1, 2), ("cry", 1, 2), ("crz", 1, 2), ("cp", 1, 2), ("cphase", 1, 2)]:
        params = [float(x) for x in rng.uniform(0, 2 * np.pi, npar)]
        d[f"param_{name}"] = np.array(params)
        d[f"gate_{name}"] = GateOp(name=name, qubits=q[:ar], params=params).matrix
    for name, params in [("depolarizing", [0.1]), ("amplitude_damping", [0.2]), ("phase_damping", [0.3]),
                         ("bit_flip", [0.15]), ("phase_flip", [0.25]),
                         ("thermal_relaxation", [100e-6, 80e-6, 50e-9]),
                         ("thermal_relaxation", [50e-6, 120e-6, 1e-6]), ("depolarizing_2q", [0.2])]:
        key = f"kraus_{name}_" + "_".join(f"{p:g}" for p in params)
        d[key] = np.array(build_kraus_channel(name, params))
    np.savez_compressed(out / "gates.npz", **d)


def brickwall_reference_circuit(iq, n, depth, seed):
    """The U3 + CX brick-wall workload, built from the reference's own IR ops."""
    from invariantq.ir.qir import CircuitIR, GateOp, QWire  # noqa: E402
    rng = np.random.default_rng(seed)
    angles = rng.uniform(0.0, 2.0 * np.pi, size=(depth, n, 3))
    c = CircuitIR(name=f"brickwall_{n}q_d{depth}")
    c.add_qubit_register("q", n)
    c.add_clbit_register("c", n)
    for layer in range(depth):
        for q in range(n):
            c.add_op(GateOp(name="u3", qubits=[QWire("q", q)], params=[float(a) for a in angles[layer, q]]))
        for q in range(layer % 2, n - 1, 2):
            c.add_op(GateOp(name="cx", qubits=[QWire("q", q), QWire("q", q + 1)]))
    return c, angles


def gen_simulators(iq, out):
    from invariantq.benchmarks.suite import create_random_circuit, create_ghz_circuit  # noqa: E402
    from invariantq.ir.qir import CircuitIR, GateOp, NoiseOp, QWire  # noqa: E402
    d = {}
    sim = iq.StateVectorSimulator()
    for seed in range(3):
        c = create_random_circuit(num_qubits=4, depth=6, seed=seed)
        r = sim.run(c, shots=100, seed=seed)
        d[f"random4_s{seed}_amps"] = r.statevector
        d[f"random4_s{seed}_ops"] = np.array([f"{op.name}:" + ",".join(str(q.index) for q in op.qubits) + ":"
                                              + ",".join(repr(float(p)) for p in op.params) for op in c.ops])
    g = create_ghz_circuit(5)
    r = sim.run(g, shots=256, seed=3)
    d["ghz5_amps"] = r.statevector
    d["ghz5_counts_keys"] = np.array(sorted(r.counts))
    d["ghz5_counts_vals"] = np.array([r.counts[k] for k in sorted(r.counts)])
    c, angles = brickwall_reference_circuit(iq, 8, 6, seed=0)
    r = sim.run(c, shots=8192, seed=11)
    d["brick8_angles"] = angles
    d["brick8_amps"] = r.statevector
    keys = sorted(r.counts)
    d["brick8_counts_keys"] = np.array(keys)
    d["brick8_counts_vals"] = np.array([r.counts[k] for k in keys])
    d["brick8_entropy"] = np.array(r.entanglement_entropy)
    # density matrix: noisy brick-wall at 4 qubits (the channel mix of the 14q DM workload)
    from invariantq.noise.channels import build_kraus_channel  # noqa: E402
    n, depth = 4, 3
    rng = np.random.default_rng(17)
    ang = rng.uniform(0.0, 2.0 * np.pi, size=(depth, n, 3))
    dc = CircuitIR(name="noisy4")
    dc.add_qubit_register("q", n)
    for layer in range(depth):
        for q in range(n):
            dc.add_op(GateOp(name="u3", qubits=[QWire("q", q)], params=[float(a) for a in ang[layer, q]]))
        for q in range(layer % 2, n - 1, 2):
            dc.add_op(GateOp(name="cx", qubits=[QWire("q", q), QWire("q", q + 1)]))
            dc.add_op(NoiseOp(qubits=[QWire("q", q), QWire("q", q + 1)], channel_name="amp_damping", params=[2e-3]))
            dc.add_op(NoiseOp(qubits=[QWire("q", q), QWire("q", q + 1)], channel_name="phase_damping", params=[1e-3]))
        dc.add_op(NoiseOp(qubits=[QWire("q", q) for q in range(n)], channel_name="thermal_relaxation",
                          params=[100e-6, 80e-6, 50e-9]))
    noise_model = {"u3": build_kraus_channel("depolarizing", [1e-3])}
    dres = iq.DensityMatrixSimulator(noise_model=noise_model).run(dc, shots=64, seed=5)
    d["noisy4_angles"] = ang
    d["noisy4_rho"] = dres.density_matrix
    d["noisy4_trace"] = np.array(dres.metadata["trace"])
    d["noisy4_purity"] = np.array(dres.metadata["purity"])
    np.savez_compressed(out / "simulators.npz", **d)


# ---------------------------------------------------------------- C-ABI traces

def _ctype_name(t):
    if t is None:
        return None
    return t.__name__


def gen_binding_argtypes(binding, out):
    """argtypes / restype the reference binding sets on every exported function."""
    import json
    names = (out / "c_api_symbols.txt").read_text().split()
    table = {}
    for name in names:
        fn = getattr(binding._NATIVE_LIB, name)
        table[name] = {"argtypes": [_ctype_name(t) for t in (fn.argtypes or [])], "restype": _ctype_name(fn.restype)}
    (out / "binding_argtypes.json").write_text(json.dumps(table, indent=1, sort_keys=True) + "\n")


class _Tracer:
    """Stands in for the binding's ``_NATIVE_LIB``: forwards every call to the
    reference core and records the state-vector and density-matrix calls with
    their input arrays and the values the core returned."""

    # pointer arguments: (index, kind, length rule); kinds: din (double input),
    # zin (size_t input), dout / uout (double / uint64 output), ref (double by reference)
    SPEC = {
        "iq_statevector_apply_1q": [(2, "din", lambda a, n: 4), (3, "din", lambda a, n: 4)],
        "iq_statevector_apply_2q": [(3, "din", lambda a, n: 16), (4, "din", lambda a, n: 16)],
        "iq_statevector_apply_fused": [(1, "zin", lambda a, n: a[2]), (3, "din", lambda a, n: 4 ** a[2]),
                                       (4, "din", lambda a, n: 4 ** a[2])],
        "iq_statevector_get_amplitudes": [(1, "dout", lambda a, n: 1 << n), (2, "dout", lambda a, n: 1 << n)],
        "iq_statevector_get_probabilities": [(1, "dout", lambda a, n: 1 << n)],
        "iq_statevector_sample": [(3, "uout", lambda a, n: a[1])],
        "iq_statevector_entropy": [(1, "zin", lambda a, n: a[2])],
        "iq_statevector_expval_pauli": [(2, "zin", lambda a, n: a[3]), (4, "ref", None), (5, "ref", None)],
        "iq_density_matrix_apply_1q_unitary": [(2, "din", lambda a, n: 4), (3, "din", lambda a, n: 4)],
        "iq_density_matrix_apply_2q_unitary": [(3, "din", lambda a, n: 16), (4, "din", lambda a, n: 16)],
        "iq_density_matrix_apply_kraus_1q": [(3, "din", lambda a, n: 4 * a[2]), (4, "din", lambda a, n: 4 * a[2])],
        "iq_density_matrix_get_elements": [(1, "dout", lambda a, n: 1 << (2 * n)),
                                           (2, "dout", lambda a, n: 1 << (2 * n))],
    }

    def __init__(self, lib):
        self._lib = lib
        self.calls = []
        self.handles = {}      # core pointer -> (id, qubits)

    def __getattr__(self, name):
        fn = getattr(self._lib, name)
        if not (name.startswith("iq_statevector_") or name.startswith("iq_density_matrix_")):
            return fn
        tracer = self

        def call(*args):
            return tracer._call(name, fn, args)
        return call

    def _call(self, name, fn, args):
        import ctypes
        args = list(args)
        spec = {i: (kind, rule) for i, kind, rule in self.SPEC.get(name, [])}
        rec_args = []
        if name.endswith("_create"):
            n = int(args[0])
        else:
            hid, n = self.handles[int(args[0])]
        plain = [a if not isinstance(a, (int, float)) else a for a in args]
        for i, a in enumerate(args):
            if i == 0 and not name.endswith("_create"):
                rec_args.append({"h": hid})
            elif i in spec:
                kind, rule = spec[i]
                if kind in ("din", "zin"):
                    L = int(rule(plain, n))
                    ct = ctypes.c_double if kind == "din" else ctypes.c_size_t
                    arr = np.ctypeslib.as_array(ctypes.cast(a, ctypes.POINTER(ct)), shape=(L,)).copy()
                    rec_args.append({kind: arr.tolist()})
                elif kind in ("dout", "uout"):
                    rec_args.append({kind: int(rule(plain, n))})
                else:
                    rec_args.append({"ref": 1})
            elif isinstance(a, bytes):
                rec_args.append({"s": a.decode("ascii")})
            elif isinstance(a, float):
                rec_args.append(a)
            else:
                rec_args.append(int(a))
        ret = fn(*args)
        rec = {"fn": name, "args": rec_args}
        outs = {}
        for i, (kind, rule) in spec.items():
            if kind in ("dout", "uout"):
                L = int(rule(plain, n))
                ct = ctypes.c_double if kind == "dout" else ctypes.c_uint64
                arr = np.ctypeslib.as_array(ctypes.cast(args[i], ctypes.POINTER(ct)), shape=(L,)).copy()
                outs[str(i)] = arr.tolist() if kind == "dout" else [int(x) for x in arr]
            elif kind == "ref":
                outs[str(i)] = float(args[i]._obj.value)
        if outs:
            rec["out"] = outs
        if name.endswith("_create"):
            hid = len(self.handles)
            self.handles[int(ret)] = (hid, n)
            rec["ret"] = {"h": hid}
        elif ret is not None:
            rec["ret"] = ret if isinstance(ret, float) else int(ret)
        self.calls.append(rec)
        return ret


def gen_abi_traces(binding, ref_dir: Path, out: Path):
    """Run the reference's own tests that pin this path (their functions called
    as written, on the reference core, through the unmodified binding and
    drivers) with the binding's library replaced by a tracer, and store each
    test's C-ABI call sequence with the core's results.  The independent
    einsum reference's state vectors (independent_reference.py:13-73) are kept
    beside the traces of the tests that compare against them."""
    import json
    tests_dir = ref_dir / "tests"
    sys.path.insert(0, str(tests_dir))
    scenarios = []
    real = binding._NATIVE_LIB
    try:
        for mod_name, funcs in (("test_core_math", ["test_single_qubit_gates", "test_bell_state_entanglement",
                                                     "test_product_state_zero_entropy",
                                                     "test_pauli_expectation_values", "test_measurement_collapse"]),
                                ("test_independent_reference", ["test_independent_reference_ghz",
                                                                "test_independent_reference_random_circuits",
                                                                "test_independent_reference_against_density_matrix"])):
            mod = importlib.import_module(mod_name)
            for f in funcs:
                tracer = _Tracer(real)
                binding._NATIVE_LIB = tracer
                try:
                    getattr(mod, f)()
                finally:
                    binding._NATIVE_LIB = real
                scenarios.append({"test": f"{mod_name}.py::{f}", "calls": tracer.calls})
    finally:
        sys.path.remove(str(tests_dir))
    # the independent reference's states for the circuits those tests build
    from invariantq.benchmarks.suite import create_random_circuit, create_ghz_circuit  # noqa: E402
    from invariantq.verification.independent_reference import run_independent_reference  # noqa: E402
    indep = {"ghz4": run_independent_reference(create_ghz_circuit(4))}
    for seed in range(5):
        indep[f"random4_s{seed}"] = run_independent_reference(create_random_circuit(num_qubits=4, depth=6, seed=seed))
    doc = {"scenarios": scenarios,
           "independent": {k: {"re": np.real(v).tolist(), "im": np.imag(v).tolist()} for k, v in indep.items()}}
    (out / "abi_traces.json").write_text(json.dumps(doc) + "\n")


def gen_symbols(ref_dir: Path, out: Path):
    """The exported function names of the reference C ABI (core/include/c_api.h)."""
    import re
    text = (ref_dir / "core" / "include" / "c_api.h").read_text()
    names = re.findall(r"\b(iq_[a-z0-9_]+)\s*\(", text)
    (out / "c_api_symbols.txt").write_text("\n".join(names) + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("IQ_REFERENCE_DIR"),
                    help="the reference checkout (default: $IQ_REFERENCE_DIR)")
    ap.add_argument("--out", default=str(HERE))
    a = ap.parse_args()
    if not a.reference:
        raise SystemExit("give the reference checkout with --reference or IQ_REFERENCE_DIR")
    out = Path(a.out)
    with tempfile.TemporaryDirectory() as td:
        iq, binding = load_reference(Path(a.reference), Path(td))
        gen_sv_ops(binding, out)
        gen_sv_readout(binding, out)
        gen_dm_ops(iq, binding, out)
        gen_gates(iq, out)
        gen_simulators(iq, out)
        gen_symbols(Path(a.reference), out)
        gen_binding_argtypes(binding, out)
        gen_abi_traces(binding, Path(a.reference), out)
    for f in sorted(out.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()

"""The library as a drop-in for the reference's ctypes binding.

* CPU: every function of the reference ABI binds on this library with exactly
  the ctypes signature the reference's binding sets (binding.py:54-299, kept in
  tests/golden/binding_argtypes.json by make_golden.py).
* CPU, where a reference checkout is named by IQ_REFERENCE_DIR: the
  reference's unmodified ``invariantq`` package, with this library placed where
  its loader looks first (binding.py:15-40), imports with the native core
  active and every signature set.
* GPU: the C-ABI call sequences the reference's own tests make
  (tests/test_core_math.py:10-69, tests/test_independent_reference.py:15-61,
  recorded on the reference core through its unmodified binding and drivers,
  tests/golden/abi_traces.json) replayed on this library through those
  signatures; every value the reference core returned is matched (amplitudes,
  probabilities, density-matrix elements, trace, purity, Pauli expectations
  1e-12; entropies 1e-9; measurement outcomes and sampled shots exactly), and
  the tests' own checks against the independent einsum reference hold.
"""
import ctypes
import json
import os
import shutil
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = 1e-12

_CT = {"c_void_p": ctypes.c_void_p, "c_ulong": ctypes.c_ulong, "c_int": ctypes.c_int, "c_double": ctypes.c_double,
       "c_char_p": ctypes.c_char_p, "c_uint": ctypes.c_uint, "c_long": ctypes.c_long,
       "LP_c_double": ctypes.POINTER(ctypes.c_double), "LP_c_ulong": ctypes.POINTER(ctypes.c_ulong),
       "LP_c_int": ctypes.POINTER(ctypes.c_int), "LP_c_ubyte": ctypes.POINTER(ctypes.c_ubyte),
       "LP_c_uint": ctypes.POINTER(ctypes.c_uint)}


def _table():
    return json.loads((GOLDEN / "binding_argtypes.json").read_text())


def _bind_as_reference():
    """A separate CDLL object for this library with the reference binding's
    signatures (the package's own binding keeps its own function objects)."""
    from invariantq_b200 import _lib
    path = _lib.LIB_PATH
    if not Path(path).exists():
        pytest.skip("libinvariantq.so not built")
    lib = ctypes.CDLL(str(path))
    for name, sig in _table().items():
        fn = getattr(lib, name)
        fn.argtypes = [_CT[t] for t in sig["argtypes"]]
        fn.restype = None if sig["restype"] is None else _CT[sig["restype"]]
    return lib


def test_reference_signatures_bind_on_this_library():
    table = _table()
    assert len(table) == 49
    lib = _bind_as_reference()
    for name in table:
        assert getattr(lib, name).argtypes is not None or table[name]["argtypes"] == []


@pytest.mark.skipif(not os.environ.get("IQ_REFERENCE_DIR"), reason="IQ_REFERENCE_DIR names no reference checkout")
def test_unmodified_reference_binding_loads_this_library(tmp_path):
    ref = Path(os.environ["IQ_REFERENCE_DIR"])
    if not (ref / "invariantq" / "core" / "binding.py").exists():
        pytest.skip("IQ_REFERENCE_DIR has no invariantq/core/binding.py")
    from invariantq_b200 import _lib
    shutil.copytree(ref / "invariantq", tmp_path / "invariantq")
    shutil.copy(_lib.LIB_PATH, tmp_path / "invariantq" / "core" / "libinvariantq.so")
    code = (
        "import json, sys\n"
        "import invariantq.core.binding as b\n"
        "assert b.HAS_NATIVE_CORE, b.native_core_status()\n"
        "names = [l for l in open(sys.argv[1]).read().split()]\n"
        "sig = {n: [t.__name__ for t in getattr(b._NATIVE_LIB, n).argtypes or []] for n in names}\n"
        "print(json.dumps({'lib': b._NATIVE_LIB._name, 'sig': sig}))\n")
    r = subprocess.run([sys.executable, "-c", code, str(GOLDEN / "c_api_symbols.txt")], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300,
                       env={**os.environ, "PYTHONPATH": str(tmp_path)})
    assert r.returncode == 0, r.stderr[-2000:]
    doc = json.loads(r.stdout.strip().splitlines()[-1])
    assert doc["lib"] == str(tmp_path / "invariantq" / "core" / "libinvariantq.so")
    table = _table()
    for name, args in doc["sig"].items():
        assert args == table[name]["argtypes"], name


def _traces():
    return json.loads((GOLDEN / "abi_traces.json").read_text())


def _replay(lib, calls):
    """Replays one recorded call sequence; returns the list of
    (function, recorded result, our result) pairs to compare."""
    handles = {}
    pairs = []
    keep = []
    for c in calls:
        name = c["fn"]
        args, outs = [], {}
        for i, a in enumerate(c["args"]):
            if isinstance(a, dict):
                if "h" in a:
                    args.append(handles[a["h"]])
                elif "din" in a:
                    arr = np.ascontiguousarray(a["din"], dtype=np.float64)
                    keep.append(arr)
                    args.append(arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
                elif "zin" in a:
                    arr = np.ascontiguousarray(a["zin"], dtype=np.uint64)
                    keep.append(arr)
                    args.append(arr.ctypes.data_as(ctypes.POINTER(ctypes.c_ulong)))
                elif "dout" in a:
                    arr = np.full(a["dout"], np.nan)
                    outs[str(i)] = arr
                    args.append(arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
                elif "uout" in a:
                    arr = np.zeros(a["uout"], dtype=np.uint64)
                    outs[str(i)] = arr
                    args.append(arr.ctypes.data_as(ctypes.POINTER(ctypes.c_ulong)))
                elif "ref" in a:
                    v = ctypes.c_double(np.nan)
                    outs[str(i)] = v
                    args.append(ctypes.byref(v))
                elif "s" in a:
                    args.append(a["s"].encode("ascii"))
                else:
                    raise AssertionError(f"unknown argument {a}")
            else:
                args.append(a)
        ret = getattr(lib, name)(*args)
        if name.endswith("_create"):
            assert ret, f"{name} returned NULL"
            handles[c["ret"]["h"]] = ret
            continue
        if "ret" in c:
            pairs.append((name, c["ret"], ret))
        for i, want in c.get("out", {}).items():
            got = outs[i]
            pairs.append((name, want, got.value if isinstance(got, ctypes.c_double) else got))
    return pairs


def _check(name, want, got):
    if name in ("iq_statevector_entropy", "iq_density_matrix_entropy"):
        assert abs(got - want) < 1e-9, (name, want, got)
    elif name in ("iq_statevector_measure", "iq_density_matrix_measure"):
        assert got == want, (name, want, got)
    elif name == "iq_statevector_sample":
        assert np.array_equal(np.asarray(got, dtype=np.uint64), np.asarray(want, dtype=np.uint64)), name
    else:
        assert np.max(np.abs(np.asarray(got, dtype=np.float64) - np.asarray(want, dtype=np.float64))) < TOL, name


@pytest.mark.gpu
@pytest.mark.parametrize("scenario", [s["test"] for s in _traces()["scenarios"]])
def test_replay_reference_test_calls(scenario):
    doc = _traces()
    calls = next(s["calls"] for s in doc["scenarios"] if s["test"] == scenario)
    lib = _bind_as_reference()
    pairs = _replay(lib, calls)
    assert pairs
    for name, want, got in pairs:
        _check(name, want, got)
    # the test's own comparison with the independent einsum reference
    # (test_independent_reference.py:15-45): fidelity of the returned states
    amps = [(w, g) for (n, w, g) in pairs if n == "iq_statevector_get_amplitudes"]
    states = [np.asarray(amps[i][1]) + 1j * np.asarray(amps[i + 1][1]) for i in range(0, len(amps), 2)]
    indep = doc["independent"]
    if scenario.endswith("::test_independent_reference_ghz"):
        ref = np.asarray(indep["ghz4"]["re"]) + 1j * np.asarray(indep["ghz4"]["im"])
        assert abs(abs(np.vdot(ref, states[0])) ** 2 - 1.0) < 1e-12
    if scenario.endswith("::test_independent_reference_random_circuits"):
        assert len(states) == 5
        for seed, st in enumerate(states):
            v = indep[f"random4_s{seed}"]
            ref = np.asarray(v["re"]) + 1j * np.asarray(v["im"])
            assert abs(abs(np.vdot(ref, st)) ** 2 - 1.0) < 1e-10

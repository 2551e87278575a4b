"""TEST INFRASTRUCTURE ONLY -- the oracle's Python face.

Two CPU checkers, never part of the shipped path:

* ``Port``    -- ctypes wrapper of ``oracle/liboracle.so``, the plain-C
  restatement of the reference kernels (``oracle/iq_oracle.c``).  It operates
  on numpy ``complex128`` arrays in place.
* ``RefCore`` -- ctypes wrapper of ``oracle/_ref/libinvariantq.so``, the
  reference's own C++/OpenMP core compiled from its sources by
  ``oracle/Makefile`` (``make -C oracle ref``).  Its handle API mirrors the
  reference binding (``invariantq/core/binding.py:302-476``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path
from typing import List, Optional, Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libinvariantq.so"

_dp = ctypes.POINTER(ctypes.c_double)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_szp = ctypes.POINTER(ctypes.c_size_t)
_vp = ctypes.c_void_p
_sz = ctypes.c_size_t


def build(ref: bool = False, ref_dir: Optional[str] = None) -> None:
    """Compile the C restatement and, if asked and a reference checkout is named
    (``ref_dir`` or the environment variable IQ_REFERENCE_DIR) and holds the
    core sources, the reference core into oracle/_ref."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    src = ref_dir or os.environ.get("IQ_REFERENCE_DIR")
    if ref and src and Path(src, "core").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={src}"], check=True)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _split(m) -> tuple:
    m = np.asarray(m, dtype=np.complex128).reshape(-1)
    return (np.ascontiguousarray(m.real, dtype=np.float64),
            np.ascontiguousarray(m.imag, dtype=np.float64))


class Port:
    """The C restatement; every method mirrors one reference function."""

    def __init__(self, path: Path = PORT_LIB):
        if not Path(path).exists():
            build()
        L = ctypes.CDLL(str(path))
        self.L = L
        cp = ctypes.c_void_p
        sig = {
            "or_sv_init": ([cp, ctypes.c_int], None),
            "or_sv_apply_1q": ([cp, ctypes.c_int, _sz, _dp, _dp], ctypes.c_int),
            "or_sv_apply_2q": ([cp, ctypes.c_int, _sz, _sz, _dp, _dp], ctypes.c_int),
            "or_sv_apply_fused": ([cp, ctypes.c_int, _szp, _sz, _dp, _dp], ctypes.c_int),
            "or_sv_measure_prob": ([cp, ctypes.c_int, _sz, ctypes.c_int], ctypes.c_double),
            "or_sv_collapse": ([cp, ctypes.c_int, _sz, ctypes.c_int], ctypes.c_int),
            "or_sv_measure": ([cp, ctypes.c_int, _sz, ctypes.c_double], ctypes.c_int),
            "or_sv_reset_qubit": ([cp, ctypes.c_int, _sz, ctypes.c_double], ctypes.c_int),
            "or_sv_norm2": ([cp, ctypes.c_int], ctypes.c_double),
            "or_sv_probabilities": ([cp, ctypes.c_int, _dp], None),
            "or_mt64_uniform": ([ctypes.c_uint64, _sz, _dp], None),
            "or_sv_sample": ([cp, ctypes.c_int, _sz, ctypes.c_uint64, _u64p], None),
            "or_sv_expval_pauli": ([cp, ctypes.c_int, ctypes.c_char_p, _szp, _sz, _dp, _dp], ctypes.c_int),
            "or_sv_entropy": ([cp, ctypes.c_int, _szp, _sz], ctypes.c_double),
            "or_dm_init": ([cp, ctypes.c_int], None),
            "or_dm_apply_1q_unitary": ([cp, ctypes.c_int, _sz, _dp, _dp], ctypes.c_int),
            "or_dm_apply_2q_unitary": ([cp, ctypes.c_int, _sz, _sz, _dp, _dp], ctypes.c_int),
            "or_dm_apply_kraus_1q": ([cp, ctypes.c_int, _sz, _sz, _dp, _dp], ctypes.c_int),
            "or_dm_trace": ([cp, ctypes.c_int], ctypes.c_double),
            "or_dm_purity": ([cp, ctypes.c_int], ctypes.c_double),
            "or_dm_measure_prob": ([cp, ctypes.c_int, _sz, ctypes.c_int], ctypes.c_double),
            "or_dm_measure": ([cp, ctypes.c_int, _sz, ctypes.c_double], ctypes.c_int),
            "or_dm_reset_qubit": ([cp, ctypes.c_int, _sz], ctypes.c_int),
            "or_dm_entropy": ([cp, ctypes.c_int], ctypes.c_double),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res

    # -- state vector -------------------------------------------------------
    @staticmethod
    def zero_state(n: int) -> np.ndarray:
        s = np.zeros(1 << n, dtype=np.complex128)
        s[0] = 1.0
        return s

    def apply_1q(self, s, n, t, U):
        r, i = _split(U)
        return self.L.or_sv_apply_1q(s.ctypes.data, n, t, _dptr(r), _dptr(i))

    def apply_2q(self, s, n, q0, q1, U):
        r, i = _split(U)
        return self.L.or_sv_apply_2q(s.ctypes.data, n, q0, q1, _dptr(r), _dptr(i))

    def apply_fused(self, s, n, qubits: Sequence[int], U):
        r, i = _split(U)
        q = np.ascontiguousarray(qubits, dtype=np.uint64)
        return self.L.or_sv_apply_fused(s.ctypes.data, n, q.ctypes.data_as(_szp), len(qubits),
                                        _dptr(r), _dptr(i))

    def measure_prob(self, s, n, t, outcome):
        return self.L.or_sv_measure_prob(s.ctypes.data, n, t, outcome)

    def measure(self, s, n, t, rand_val):
        return self.L.or_sv_measure(s.ctypes.data, n, t, rand_val)

    def reset_qubit(self, s, n, t, rand_val=0.0):
        return self.L.or_sv_reset_qubit(s.ctypes.data, n, t, rand_val)

    def norm2(self, s, n):
        return self.L.or_sv_norm2(s.ctypes.data, n)

    def probabilities(self, s, n):
        out = np.empty(1 << n, dtype=np.float64)
        self.L.or_sv_probabilities(s.ctypes.data, n, _dptr(out))
        return out

    def uniforms(self, seed: int, count: int) -> np.ndarray:
        out = np.empty(count, dtype=np.float64)
        self.L.or_mt64_uniform(seed, count, _dptr(out))
        return out

    def sample(self, s, n, shots, seed):
        out = np.empty(shots, dtype=np.uint64)
        self.L.or_sv_sample(s.ctypes.data, n, shots, seed, out.ctypes.data_as(_u64p))
        return out

    def expval_pauli(self, s, n, pauli: str, qubits: Sequence[int]) -> complex:
        q = np.ascontiguousarray(qubits, dtype=np.uint64)
        re, im = ctypes.c_double(), ctypes.c_double()
        self.L.or_sv_expval_pauli(s.ctypes.data, n, pauli.encode("ascii"), q.ctypes.data_as(_szp),
                                  len(qubits), ctypes.byref(re), ctypes.byref(im))
        return complex(re.value, im.value)

    def entropy(self, s, n, qubits: Sequence[int]) -> float:
        q = np.ascontiguousarray(qubits, dtype=np.uint64)
        return self.L.or_sv_entropy(s.ctypes.data, n, q.ctypes.data_as(_szp), len(qubits))

    # -- density matrix -----------------------------------------------------
    @staticmethod
    def zero_rho(n: int) -> np.ndarray:
        r = np.zeros((1 << n, 1 << n), dtype=np.complex128)
        r[0, 0] = 1.0
        return r

    def dm_apply_1q(self, rho, n, t, U):
        r, i = _split(U)
        return self.L.or_dm_apply_1q_unitary(rho.ctypes.data, n, t, _dptr(r), _dptr(i))

    def dm_apply_2q(self, rho, n, q0, q1, U):
        r, i = _split(U)
        return self.L.or_dm_apply_2q_unitary(rho.ctypes.data, n, q0, q1, _dptr(r), _dptr(i))

    def dm_apply_kraus_1q(self, rho, n, t, kraus: List[np.ndarray]):
        st = np.stack([np.asarray(k, dtype=np.complex128).reshape(-1) for k in kraus])
        r, i = _split(st)
        return self.L.or_dm_apply_kraus_1q(rho.ctypes.data, n, t, len(kraus), _dptr(r), _dptr(i))

    def dm_trace(self, rho, n):
        return self.L.or_dm_trace(rho.ctypes.data, n)

    def dm_purity(self, rho, n):
        return self.L.or_dm_purity(rho.ctypes.data, n)

    def dm_measure(self, rho, n, t, rand_val):
        return self.L.or_dm_measure(rho.ctypes.data, n, t, rand_val)

    def dm_reset_qubit(self, rho, n, t):
        return self.L.or_dm_reset_qubit(rho.ctypes.data, n, t)

    def dm_entropy(self, rho, n):
        return self.L.or_dm_entropy(rho.ctypes.data, n)


class RefCore:
    """ctypes access to the reference's own compiled core (SV and DM handles)."""

    def __init__(self, path: Path = REF_LIB):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference sources exist")
        L = ctypes.CDLL(str(path))
        self.L = L
        sig = {
            "iq_statevector_create": ([_sz], _vp),
            "iq_statevector_free": ([_vp], None),
            "iq_statevector_reset": ([_vp], None),
            "iq_statevector_apply_1q": ([_vp, _sz, _dp, _dp], None),
            "iq_statevector_apply_2q": ([_vp, _sz, _sz, _dp, _dp], None),
            "iq_statevector_apply_fused": ([_vp, _szp, _sz, _dp, _dp], None),
            "iq_statevector_measure": ([_vp, _sz, ctypes.c_double], ctypes.c_int),
            "iq_statevector_reset_qubit": ([_vp, _sz, ctypes.c_double], None),
            "iq_statevector_measure_prob": ([_vp, _sz, ctypes.c_int], ctypes.c_double),
            "iq_statevector_get_amplitudes": ([_vp, _dp, _dp], None),
            "iq_statevector_get_probabilities": ([_vp, _dp], None),
            "iq_statevector_sample": ([_vp, _sz, ctypes.c_uint64, _u64p], None),
            "iq_statevector_entropy": ([_vp, _szp, _sz], ctypes.c_double),
            "iq_statevector_expval_pauli": ([_vp, ctypes.c_char_p, _szp, _sz, _dp, _dp], None),
            "iq_density_matrix_create": ([_sz], _vp),
            "iq_density_matrix_free": ([_vp], None),
            "iq_density_matrix_reset": ([_vp], None),
            "iq_density_matrix_apply_1q_unitary": ([_vp, _sz, _dp, _dp], None),
            "iq_density_matrix_apply_2q_unitary": ([_vp, _sz, _sz, _dp, _dp], None),
            "iq_density_matrix_apply_kraus_1q": ([_vp, _sz, _sz, _dp, _dp], None),
            "iq_density_matrix_get_elements": ([_vp, _dp, _dp], None),
            "iq_density_matrix_trace": ([_vp], ctypes.c_double),
            "iq_density_matrix_purity": ([_vp], ctypes.c_double),
            "iq_density_matrix_entropy": ([_vp], ctypes.c_double),
            "iq_density_matrix_measure": ([_vp, _sz, ctypes.c_double], ctypes.c_int),
            "iq_density_matrix_reset_qubit": ([_vp, _sz], None),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res

    def sv(self, n: int) -> "RefSV":
        return RefSV(self, n)

    def dm(self, n: int) -> "RefDM":
        return RefDM(self, n)


class RefSV:
    def __init__(self, core: RefCore, n: int):
        self.L, self.n, self.dim = core.L, n, 1 << n
        self.h = self.L.iq_statevector_create(n)
        if not self.h:
            raise MemoryError("reference create failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.iq_statevector_free(self.h)
            self.h = None

    def reset(self):
        self.L.iq_statevector_reset(self.h)

    def apply_1q(self, t, U):
        r, i = _split(U)
        self.L.iq_statevector_apply_1q(self.h, t, _dptr(r), _dptr(i))

    def apply_2q(self, q0, q1, U):
        r, i = _split(U)
        self.L.iq_statevector_apply_2q(self.h, q0, q1, _dptr(r), _dptr(i))

    def apply_fused(self, qubits, U):
        r, i = _split(U)
        q = np.ascontiguousarray(qubits, dtype=np.uint64)
        self.L.iq_statevector_apply_fused(self.h, q.ctypes.data_as(_szp), len(qubits), _dptr(r), _dptr(i))

    def amplitudes(self) -> np.ndarray:
        re = np.empty(self.dim)
        im = np.empty(self.dim)
        self.L.iq_statevector_get_amplitudes(self.h, _dptr(re), _dptr(im))
        return re + 1j * im

    def probabilities(self) -> np.ndarray:
        p = np.empty(self.dim)
        self.L.iq_statevector_get_probabilities(self.h, _dptr(p))
        return p

    def measure_prob(self, t, o):
        return self.L.iq_statevector_measure_prob(self.h, t, o)

    def measure(self, t, r):
        return self.L.iq_statevector_measure(self.h, t, r)

    def reset_qubit(self, t, r=0.0):
        self.L.iq_statevector_reset_qubit(self.h, t, r)

    def sample(self, shots, seed):
        out = np.empty(shots, dtype=np.uint64)
        self.L.iq_statevector_sample(self.h, shots, seed, out.ctypes.data_as(_u64p))
        return out

    def expval_pauli(self, pauli, qubits):
        q = np.ascontiguousarray(qubits, dtype=np.uint64)
        re, im = ctypes.c_double(), ctypes.c_double()
        self.L.iq_statevector_expval_pauli(self.h, pauli.encode("ascii"), q.ctypes.data_as(_szp),
                                           len(qubits), ctypes.byref(re), ctypes.byref(im))
        return complex(re.value, im.value)

    def entropy(self, qubits):
        q = np.ascontiguousarray(qubits, dtype=np.uint64)
        return self.L.iq_statevector_entropy(self.h, q.ctypes.data_as(_szp), len(qubits))


class RefDM:
    def __init__(self, core: RefCore, n: int):
        self.L, self.n, self.dim = core.L, n, 1 << n
        self.h = self.L.iq_density_matrix_create(n)
        if not self.h:
            raise MemoryError("reference create failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.iq_density_matrix_free(self.h)
            self.h = None

    def apply_1q(self, t, U):
        r, i = _split(U)
        self.L.iq_density_matrix_apply_1q_unitary(self.h, t, _dptr(r), _dptr(i))

    def apply_2q(self, q0, q1, U):
        r, i = _split(U)
        self.L.iq_density_matrix_apply_2q_unitary(self.h, q0, q1, _dptr(r), _dptr(i))

    def apply_kraus_1q(self, t, kraus):
        st = np.stack([np.asarray(k, dtype=np.complex128).reshape(-1) for k in kraus])
        r, i = _split(st)
        self.L.iq_density_matrix_apply_kraus_1q(self.h, t, len(kraus), _dptr(r), _dptr(i))

    def matrix(self) -> np.ndarray:
        tot = self.dim * self.dim
        re = np.empty(tot)
        im = np.empty(tot)
        self.L.iq_density_matrix_get_elements(self.h, _dptr(re), _dptr(im))
        return (re + 1j * im).reshape(self.dim, self.dim)

    def trace(self):
        return self.L.iq_density_matrix_trace(self.h)

    def purity(self):
        return self.L.iq_density_matrix_purity(self.h)

    def entropy(self):
        return self.L.iq_density_matrix_entropy(self.h)

    def measure(self, t, r):
        return self.L.iq_density_matrix_measure(self.h, t, r)

    def reset_qubit(self, t):
        self.L.iq_density_matrix_reset_qubit(self.h, t)

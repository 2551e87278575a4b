"""Handle wrappers with the method surface of the reference's ctypes binding
(``NativeStateVector`` invariantq/core/binding.py:302-395, ``NativeDensityMatrix``
binding.py:398-476), backed by the CUDA library.  Extra methods expose the
additions of include/invariantq_b200.h.

Unlike the reference (whose C++ aborts the process on a bad argument, and whose
fallback raises ValueError), errors recorded by the library are raised here as
ValueError (bad argument), MemoryError (allocation) or IQError.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Sequence

import numpy as np

from . import _lib
from ._lib import c_dp, c_szp, c_u64p, check


def _split(matrix) -> tuple:
    m = np.asarray(matrix, dtype=np.complex128).reshape(-1)
    return (np.ascontiguousarray(m.real, dtype=np.float64), np.ascontiguousarray(m.imag, dtype=np.float64))


def _p(a: np.ndarray):
    return a.ctypes.data_as(c_dp)


def native_core_status() -> dict:
    lib = _lib.load()
    return {"active": True, "implementation": "cuda-sm_100a", "version": lib.iq_version().decode(),
            "library": str(_lib.LIB_PATH)}


class _Handle:
    _kind = "statevector"

    def set_option(self, key: str, value: float) -> None:
        if self._lib.iq_handle_set_option(self._ptr, key.encode(), float(value)) != 0:
            check(self._lib)
            raise ValueError(f"invalid option {key}={value}")

    def get_option(self, key: str) -> float:
        return self._lib.iq_handle_get_option(self._ptr, key.encode())

    def stats(self) -> Dict[str, float]:
        out = np.zeros(8)
        self._lib.iq_handle_stats(self._ptr, _p(out), 8)
        keys = ("passes", "ops", "bytes", "launches", "flushes", "tile_passes", "h2d_bytes", "jit_passes")
        return dict(zip(keys, out.tolist()))

    def record(self):
        """Context manager: operations issued inside become a device-resident
        ``Program`` (planned once, replayed with ``run``)."""
        return _Recorder(self)

    def profile_read(self, max_items: int = 1 << 16) -> np.ndarray:
        out = np.zeros(max_items)
        n = self._lib.iq_handle_profile_read(self._ptr, _p(out), max_items)
        return out[:n].copy()


class Program:
    """Planned tile passes + matrices resident on the device (iq_handle_record_end)."""

    def __init__(self, handle: "_Handle", ptr: int):
        self._lib = handle._lib
        self._ptr = ptr
        out = np.zeros(4)
        self._lib.iq_program_info(ptr, _p(out), 4)
        self.passes, self.ops, self.matrix_bytes, self.planned_cost = int(out[0]), int(out[1]), out[2], out[3]

    def pass_info(self) -> List[Dict[str, float]]:
        """Per pass: operations, planned cost (real FMAs per amplitude),
        register stages, tile bits, chunk bits, tiles."""
        out, rows = np.zeros(6), []
        keys = ("ops", "cost", "stages", "tile_bits", "chunk_bits", "tiles")
        for i in range(self.passes):
            if self._lib.iq_program_pass_info(self._ptr, i, _p(out), 6) != 6:
                break
            rows.append(dict(zip(keys, out.tolist())))
        return rows

    def run(self, handle: "_Handle") -> None:
        if self._lib.iq_handle_program_run(handle._ptr, self._ptr) != 0:
            check(self._lib)

    def __del__(self):
        if getattr(self, "_ptr", None):
            self._lib.iq_program_free(self._ptr)
            self._ptr = None


class _Recorder:
    def __init__(self, h: "_Handle"):
        self.h = h
        self.program = None

    def __enter__(self):
        if self.h._lib.iq_handle_record_begin(self.h._ptr) != 0:
            check(self.h._lib)
        return self

    def __exit__(self, et, ev, tb):
        p = self.h._lib.iq_handle_record_end(self.h._ptr)
        if not p:
            check(self.h._lib)
            raise RuntimeError("recording failed")
        self.program = Program(self.h, p)
        return False


class NativeStateVector(_Handle):
    """Dense complex128 state vector in GPU memory (binding.py:302-395)."""

    def __init__(self, num_qubits: int):
        self._lib = _lib.load()
        self.num_qubits = int(num_qubits)
        self.dim = 1 << self.num_qubits
        self._ptr = self._lib.iq_statevector_create(self.num_qubits)
        if not self._ptr:
            check(self._lib)
            raise MemoryError("Failed to allocate StateVector on the GPU")

    def __del__(self):
        if getattr(self, "_ptr", None):
            self._lib.iq_statevector_free(self._ptr)
            self._ptr = None

    def close(self):
        self.__del__()

    def reset(self):
        self._lib.iq_statevector_reset(self._ptr)
        check(self._lib)

    def apply_1q(self, target: int, matrix):
        r, i = _split(matrix)
        self._lib.iq_statevector_apply_1q(self._ptr, target, _p(r), _p(i))
        check(self._lib)

    def apply_2q(self, q0: int, q1: int, matrix):
        r, i = _split(matrix)
        self._lib.iq_statevector_apply_2q(self._ptr, q0, q1, _p(r), _p(i))
        check(self._lib)

    def apply_fused(self, qubits: Sequence[int], matrix):
        r, i = _split(matrix)
        q = np.ascontiguousarray(qubits, dtype=np.uint64)
        self._lib.iq_statevector_apply_fused(self._ptr, q.ctypes.data_as(c_szp), len(qubits), _p(r), _p(i))
        check(self._lib)

    def measure(self, target: int, rand_val: float) -> int:
        o = self._lib.iq_statevector_measure(self._ptr, target, rand_val)
        check(self._lib)
        return o

    def reset_qubit(self, target: int, rand_val: float = 0.0):
        self._lib.iq_statevector_reset_qubit(self._ptr, target, rand_val)
        check(self._lib)

    def measure_prob(self, target: int, outcome: int) -> float:
        p = self._lib.iq_statevector_measure_prob(self._ptr, target, outcome)
        check(self._lib)
        return p

    def get_amplitudes(self) -> np.ndarray:
        re = np.empty(self.dim)
        im = np.empty(self.dim)
        self._lib.iq_statevector_get_amplitudes(self._ptr, _p(re), _p(im))
        check(self._lib)
        return re + 1j * im

    def get_probabilities(self) -> np.ndarray:
        p = np.empty(self.dim)
        self._lib.iq_statevector_get_probabilities(self._ptr, _p(p))
        check(self._lib)
        return p

    def sample(self, num_shots: int, seed: int = 42) -> np.ndarray:
        out = np.empty(num_shots, dtype=np.uint64)
        self._lib.iq_statevector_sample(self._ptr, num_shots, seed, out.ctypes.data_as(c_u64p))
        check(self._lib)
        return out

    def sample_counts(self, num_shots: int, seed: int = 42):
        """(outcomes ascending, their counts) of the shots sample() draws with
        this seed, sampled and counted on the device."""
        vals = np.empty(max(num_shots, 1), dtype=np.uint64)
        cnts = np.empty(max(num_shots, 1), dtype=np.uint64)
        nu = ctypes.c_size_t()
        if self._lib.iq_statevector_sample_counts(self._ptr, num_shots, seed, vals.ctypes.data_as(c_u64p),
                                                  cnts.ctypes.data_as(c_u64p), ctypes.byref(nu)) != 0:
            check(self._lib)
            raise RuntimeError("sample_counts failed")
        return vals[:nu.value].copy(), cnts[:nu.value].copy()

    def von_neumann_entropy(self, subsystem_qubits: List[int]) -> float:
        q = np.ascontiguousarray(subsystem_qubits, dtype=np.uint64)
        v = self._lib.iq_statevector_entropy(self._ptr, q.ctypes.data_as(c_szp), len(subsystem_qubits))
        check(self._lib)
        return v

    def expectation_value_pauli(self, pauli_str: str, qubits: List[int]) -> complex:
        q = np.ascontiguousarray(qubits, dtype=np.uint64)
        re, im = ctypes.c_double(), ctypes.c_double()
        self._lib.iq_statevector_expval_pauli(self._ptr, pauli_str.encode("ascii"), q.ctypes.data_as(c_szp),
                                              len(qubits), ctypes.byref(re), ctypes.byref(im))
        check(self._lib)
        return complex(re.value, im.value)

    # ---- additions
    def flush(self):
        if self._lib.iq_statevector_flush(self._ptr) != 0:
            check(self._lib)

    def sync(self):
        if self._lib.iq_statevector_sync(self._ptr) != 0:
            check(self._lib)

    def norm_squared(self) -> float:
        v = self._lib.iq_statevector_norm(self._ptr)
        check(self._lib)
        return v

    def expval_z_all(self) -> np.ndarray:
        out = np.empty(self.num_qubits)
        if self._lib.iq_statevector_expval_z_all(self._ptr, _p(out)) != 0:
            check(self._lib)
        return out

    def expval_pauli_sum(self, coeffs: Sequence[float], paulis: Sequence[str]) -> complex:
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        s = "".join(paulis).encode("ascii")
        if any(len(p) != self.num_qubits for p in paulis):
            raise ValueError("every Pauli string needs one character per qubit")
        re, im = ctypes.c_double(), ctypes.c_double()
        if self._lib.iq_statevector_expval_pauli_sum(self._ptr, len(paulis), _p(c), s, ctypes.byref(re),
                                                     ctypes.byref(im)) != 0:
            check(self._lib)
        return complex(re.value, im.value)

    def set_amplitudes(self, amps) -> None:
        a = np.asarray(amps, dtype=np.complex128).reshape(-1)
        if a.size != self.dim:
            raise ValueError("amplitude count does not match 2^n")
        re = np.ascontiguousarray(a.real)
        im = np.ascontiguousarray(a.imag)
        if self._lib.iq_statevector_set_amplitudes(self._ptr, _p(re), _p(im)) != 0:
            check(self._lib)

    def pack_half(self, bit: int, value: int, d_dst: int) -> None:
        """Copy the amplitudes with index bit `bit` == value (increasing index
        order) to the device buffer at address d_dst (2^(n-1) complex128)."""
        if self._lib.iq_statevector_pack_half(self._ptr, bit, value, ctypes.c_void_p(d_dst)) != 0:
            check(self._lib)
            raise RuntimeError("pack_half failed")

    def unpack_half(self, bit: int, value: int, d_src: int) -> None:
        """The reverse of pack_half: overwrite that half from the device buffer."""
        if self._lib.iq_statevector_unpack_half(self._ptr, bit, value, ctypes.c_void_p(d_src)) != 0:
            check(self._lib)
            raise RuntimeError("unpack_half failed")

    def device_ptr(self) -> int:
        p = self._lib.iq_statevector_device_ptr(self._ptr)
        check(self._lib)
        return p

    def stream(self) -> int:
        return self._lib.iq_statevector_stream(self._ptr)


class NativeDensityMatrix(_Handle):
    """Dense complex128 density matrix in GPU memory (binding.py:398-476)."""

    _kind = "density_matrix"

    def __init__(self, num_qubits: int):
        self._lib = _lib.load()
        self.num_qubits = int(num_qubits)
        self.dim = 1 << self.num_qubits
        self._ptr = self._lib.iq_density_matrix_create(self.num_qubits)
        if not self._ptr:
            check(self._lib)
            raise MemoryError("Failed to allocate DensityMatrix on the GPU")

    def __del__(self):
        if getattr(self, "_ptr", None):
            self._lib.iq_density_matrix_free(self._ptr)
            self._ptr = None

    def close(self):
        self.__del__()

    def reset(self):
        self._lib.iq_density_matrix_reset(self._ptr)
        check(self._lib)

    def apply_1q_unitary(self, target: int, matrix):
        r, i = _split(matrix)
        self._lib.iq_density_matrix_apply_1q_unitary(self._ptr, target, _p(r), _p(i))
        check(self._lib)

    def apply_2q_unitary(self, q0: int, q1: int, matrix):
        r, i = _split(matrix)
        self._lib.iq_density_matrix_apply_2q_unitary(self._ptr, q0, q1, _p(r), _p(i))
        check(self._lib)

    def apply_1q_kraus(self, target: int, kraus_ops: List[np.ndarray]):
        st = np.stack([np.asarray(k, dtype=np.complex128).reshape(-1) for k in kraus_ops])
        r, i = _split(st)
        self._lib.iq_density_matrix_apply_kraus_1q(self._ptr, target, len(kraus_ops), _p(r), _p(i))
        check(self._lib)

    def apply_2q_kraus(self, q0: int, q1: int, kraus_ops: List[np.ndarray]):
        """Two-qubit Kraus channel (the method the reference driver calls at
        invariantq/simulator/density_matrix.py:47 but never defines)."""
        st = np.stack([np.asarray(k, dtype=np.complex128).reshape(-1) for k in kraus_ops])
        if st.shape[1] != 16:
            raise ValueError("two-qubit Kraus operators must be 4x4")
        r, i = _split(st)
        self._lib.iq_density_matrix_apply_kraus_2q(self._ptr, q0, q1, len(kraus_ops), _p(r), _p(i))
        check(self._lib)

    def get_matrix(self) -> np.ndarray:
        tot = self.dim * self.dim
        re = np.empty(tot)
        im = np.empty(tot)
        self._lib.iq_density_matrix_get_elements(self._ptr, _p(re), _p(im))
        check(self._lib)
        return (re + 1j * im).reshape(self.dim, self.dim)

    def get_diagonal(self) -> np.ndarray:
        out = np.empty(self.dim)
        self._lib.iq_density_matrix_get_diagonal(self._ptr, _p(out))
        check(self._lib)
        return out

    def trace(self) -> float:
        v = self._lib.iq_density_matrix_trace(self._ptr)
        check(self._lib)
        return v

    def purity(self) -> float:
        v = self._lib.iq_density_matrix_purity(self._ptr)
        check(self._lib)
        return v

    def von_neumann_entropy(self) -> float:
        v = self._lib.iq_density_matrix_entropy(self._ptr)
        check(self._lib)
        return v

    def measure_prob(self, target: int, outcome: int) -> float:
        v = self._lib.iq_density_matrix_measure_prob(self._ptr, target, outcome)
        check(self._lib)
        return v

    def measure(self, target: int, rand_val: float) -> int:
        o = self._lib.iq_density_matrix_measure(self._ptr, target, rand_val)
        check(self._lib)
        return o

    def reset_qubit(self, target: int):
        self._lib.iq_density_matrix_reset_qubit(self._ptr, target)
        check(self._lib)

    def flush(self):
        if self._lib.iq_density_matrix_flush(self._ptr) != 0:
            check(self._lib)

    def device_ptr(self) -> int:
        p = self._lib.iq_density_matrix_device_ptr(self._ptr)
        check(self._lib)
        return p


def selftest_bounded_wait(limit_ms: float = 20.0) -> tuple:
    """Runs the tile kernel's bounded wait on an mbarrier that never completes
    (iq_selftest_bounded_wait): returns (status, waited_ms).  Status 1 means the
    wait gave up and reported a timed-out tile load, as it should."""
    lib = _lib.load()
    waited = ctypes.c_double()
    st = lib.iq_selftest_bounded_wait(float(limit_ms), ctypes.byref(waited))
    if st < 0:
        check(lib)
        raise RuntimeError("iq_selftest_bounded_wait failed")
    return st, waited.value


def mt64_uniform(seed: int, count: int) -> np.ndarray:
    """`count` draws of uniform_real_distribution(0, 1) over mt19937_64(seed),
    generated on the GPU (the numbers iq_statevector_sample uses)."""
    lib = _lib.load()
    out = np.empty(max(count, 1))
    if lib.iq_mt64_uniform(int(seed), count, _p(out)) != 0:
        check(lib)
        raise RuntimeError("iq_mt64_uniform failed")
    return out[:count].copy()


def jit_info() -> dict:
    """Specialised pass kernels of this process (iq_jit_info)."""
    lib = _lib.load()
    out = np.zeros(2)
    note = ctypes.create_string_buffer(512)
    lib.iq_jit_info(_p(out), 2, note, 512)
    return {"compiled": int(out[0]), "from_disk": int(out[1]), "note": note.value.decode(errors="replace")}


def jit_wait(timeout_s: float = 120.0) -> bool:
    """Wait for background kernel compilations (iq_jit_wait); True when idle."""
    return _lib.load().iq_jit_wait(float(timeout_s)) == 0

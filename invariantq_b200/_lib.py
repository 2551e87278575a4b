"""ctypes loader for the in-tree CUDA library ``libinvariantq.so``.

There is no CPU fallback: if the library is missing, cannot be loaded, or no
sm_100 GPU is visible, the calls that need it raise.  The symbol table matches
include/invariantq_b200.h (the reference ABI of core/include/c_api.h:10-65
plus the additions)."""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("IQ_LIBRARY") or _PKG / "libinvariantq.so")

c_dp = ctypes.POINTER(ctypes.c_double)
c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_szp = ctypes.POINTER(ctypes.c_size_t)
_v = ctypes.c_void_p
_sz = ctypes.c_size_t
_d = ctypes.c_double
_i = ctypes.c_int
c_ip = ctypes.POINTER(ctypes.c_int)


class AdjointCircuit(ctypes.Structure):
    """iq_adjoint_circuit (include/invariantq_b200.h)."""
    _fields_ = [("num_qubits", _sz), ("num_ops", _sz), ("kinds", c_ip), ("q0", c_ip), ("q1", c_ip),
                ("param_index", c_ip), ("num_params", _sz), ("num_sets", _sz), ("params", c_dp),
                ("num_terms", _sz), ("coeffs", c_dp), ("paulis", ctypes.c_char_p), ("energy_out", c_dp),
                ("grad_out", c_dp)]


SIGNATURES = {
    # reference ABI: state vector
    "iq_statevector_create": ([_sz], _v),
    "iq_statevector_free": ([_v], None),
    "iq_statevector_reset": ([_v], None),
    "iq_statevector_apply_1q": ([_v, _sz, c_dp, c_dp], None),
    "iq_statevector_apply_2q": ([_v, _sz, _sz, c_dp, c_dp], None),
    "iq_statevector_apply_fused": ([_v, c_szp, _sz, c_dp, c_dp], None),
    "iq_statevector_measure": ([_v, _sz, _d], _i),
    "iq_statevector_reset_qubit": ([_v, _sz, _d], None),
    "iq_statevector_measure_prob": ([_v, _sz, _i], _d),
    "iq_statevector_get_amplitudes": ([_v, c_dp, c_dp], None),
    "iq_statevector_get_probabilities": ([_v, c_dp], None),
    "iq_statevector_sample": ([_v, _sz, ctypes.c_uint64, c_u64p], None),
    "iq_statevector_entropy": ([_v, c_szp, _sz], _d),
    "iq_statevector_expval_pauli": ([_v, ctypes.c_char_p, c_szp, _sz, c_dp, c_dp], None),
    # reference ABI: density matrix
    "iq_density_matrix_create": ([_sz], _v),
    "iq_density_matrix_free": ([_v], None),
    "iq_density_matrix_reset": ([_v], None),
    "iq_density_matrix_apply_1q_unitary": ([_v, _sz, c_dp, c_dp], None),
    "iq_density_matrix_apply_2q_unitary": ([_v, _sz, _sz, c_dp, c_dp], None),
    "iq_density_matrix_apply_kraus_1q": ([_v, _sz, _sz, c_dp, c_dp], None),
    "iq_density_matrix_get_elements": ([_v, c_dp, c_dp], None),
    "iq_density_matrix_trace": ([_v], _d),
    "iq_density_matrix_purity": ([_v], _d),
    "iq_density_matrix_entropy": ([_v], _d),
    "iq_density_matrix_measure": ([_v, _sz, _d], _i),
    "iq_density_matrix_reset_qubit": ([_v, _sz], None),
    # reference ABI: stabilizer / MPS (forwarded to a CPU core when one is configured)
    "iq_stabilizer_create": ([_sz], _v),
    "iq_stabilizer_free": ([_v], None),
    "iq_stabilizer_reset": ([_v], None),
    "iq_stabilizer_reset_qubit": ([_v, _sz, _d], None),
    "iq_stabilizer_apply_h": ([_v, _sz], None),
    "iq_stabilizer_apply_s": ([_v, _sz], None),
    "iq_stabilizer_apply_sdg": ([_v, _sz], None),
    "iq_stabilizer_apply_cnot": ([_v, _sz, _sz], None),
    "iq_stabilizer_apply_cz": ([_v, _sz, _sz], None),
    "iq_stabilizer_apply_swap": ([_v, _sz, _sz], None),
    "iq_stabilizer_apply_x": ([_v, _sz], None),
    "iq_stabilizer_apply_y": ([_v, _sz], None),
    "iq_stabilizer_apply_z": ([_v, _sz], None),
    "iq_stabilizer_measure": ([_v, _sz, _d], _i),
    "iq_stabilizer_to_string": ([_v, ctypes.c_char_p, _sz], None),
    "iq_mps_create": ([_sz, _sz, _d], _v),
    "iq_mps_free": ([_v], None),
    "iq_mps_reset": ([_v], None),
    "iq_mps_apply_1q": ([_v, _sz, c_dp, c_dp], None),
    "iq_mps_apply_2q": ([_v, _sz, _sz, c_dp, c_dp], None),
    "iq_mps_entropy": ([_v, _sz], _d),
    "iq_mps_to_statevector": ([_v, c_dp, c_dp], None),
    "iq_mps_measure": ([_v, _sz, _d], _i),
    # additions
    "iq_last_error": ([ctypes.c_char_p, _sz], _i),
    "iq_clear_error": ([], None),
    "iq_version": ([], ctypes.c_char_p),
    "iq_kernel_launches": ([], ctypes.c_uint64),
    "iq_statevector_flush": ([_v], _i),
    "iq_statevector_sync": ([_v], _i),
    "iq_statevector_norm": ([_v], _d),
    "iq_statevector_expval_z_all": ([_v, c_dp], _i),
    "iq_statevector_expval_pauli_sum": ([_v, _sz, c_dp, ctypes.c_char_p, c_dp, c_dp], _i),
    "iq_statevector_set_amplitudes": ([_v, c_dp, c_dp], _i),
    "iq_statevector_device_ptr": ([_v], _v),
    "iq_statevector_pack_half": ([_v, _sz, _i, _v], _i),
    "iq_statevector_sample_counts": ([_v, _sz, ctypes.c_uint64, c_u64p, c_u64p, c_szp], _i),
    "iq_mt64_uniform": ([ctypes.c_uint64, _sz, c_dp], _i),
    "iq_statevector_unpack_half": ([_v, _sz, _i, _v], _i),
    "iq_statevector_stream": ([_v], _v),
    "iq_statevector_num_qubits": ([_v], _sz),
    "iq_handle_set_option": ([_v, ctypes.c_char_p, _d], _i),
    "iq_handle_get_option": ([_v, ctypes.c_char_p], _d),
    "iq_handle_stats": ([_v, c_dp, _sz], _i),
    "iq_handle_profile_read": ([_v, c_dp, _sz], _i),
    "iq_handle_record_begin": ([_v], _i),
    "iq_handle_record_end": ([_v], _v),
    "iq_handle_program_run": ([_v, _v], _i),
    "iq_program_info": ([_v, c_dp, _sz], _i),
    "iq_program_pass_info": ([_v, _sz, c_dp, _sz], _i),
    "iq_program_free": ([_v], None),
    "iq_statevector_expval_z_all_noalloc": ([_v, _sz, _v, _v], _i),
    "iq_adjoint_gradient": ([_sz, _sz, c_ip, c_ip, c_ip, c_ip, _sz, c_dp, _sz, c_dp, ctypes.c_char_p, c_dp, c_dp],
                            _i),
    "iq_adjoint_gradient_batch": ([ctypes.POINTER(AdjointCircuit), _sz, _i], _i),
    "iq_adjoint_gradient_c64": ([_sz, _sz, c_ip, c_ip, c_ip, c_ip, _sz, c_dp, _sz, c_dp, ctypes.c_char_p, c_dp, c_dp],
                                _i),
    "iq_ansatz_energy": ([ctypes.POINTER(AdjointCircuit)], _i),
    "iq_adjoint_stats": ([c_dp, _sz], _i),
    "iq_selftest_bounded_wait": ([_d, c_dp], _i),
    "iq_jit_info": ([c_dp, _sz, ctypes.c_char_p, _sz], _i),
    "iq_jit_wait": ([_d], _i),
    "iq_adjoint_release": ([], _i),
    "iq_density_matrix_flush": ([_v], _i),
    "iq_density_matrix_apply_kraus_2q": ([_v, _sz, _sz, _sz, c_dp, c_dp], None),
    "iq_density_matrix_get_diagonal": ([_v, c_dp], None),
    "iq_density_matrix_measure_prob": ([_v, _sz, _i], _d),
    "iq_density_matrix_device_ptr": ([_v], _v),
}

_LIB = None
_LOAD_ERROR = None


def load(path: Path | None = None) -> ctypes.CDLL:
    """Load the library (once) and declare every signature; raises on failure."""
    global _LIB, _LOAD_ERROR
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} not found: build it with `python -m invariantq_b200.build` "
                           "(there is no CPU fallback for this path)")
    lib = ctypes.CDLL(str(p))
    for name, (args, res) in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    if path is None:
        _LIB = lib
    return lib


class IQError(RuntimeError):
    """An error the CUDA library recorded (iq_last_error)."""


def check(lib: ctypes.CDLL) -> None:
    code = lib.iq_last_error(None, 0)
    if code:
        buf = ctypes.create_string_buffer(512)
        lib.iq_last_error(buf, 512)
        lib.iq_clear_error()
        msg = buf.value.decode(errors="replace")
        if code == 1:
            raise ValueError(msg)
        if code == 3:
            raise MemoryError(msg)
        raise IQError(msg)

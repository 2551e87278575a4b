"""The allocation-free <Z_q> entry point (iq_statevector_expval_z_all_noalloc).

It serves callers that cannot call cudaMalloc where they need the result (a
host whose GPU memory is already committed to the state, or code inside another
framework that owns the free device memory): they pass their own device buffers
and the library works in a fixed scratch array that is part of its device code.
This file is collected last so a failure here cannot hide other failures."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _state(n, seed):
    from invariantq_b200.binding import NativeStateVector
    from tests.test_scheduler_emulated import gen_ops
    from tests.test_gpu_sv import apply_abi
    sv = NativeStateVector(n)
    apply_abi(sv, gen_ops(np.random.default_rng(seed), n, 40, kmax=min(3, n)))
    return sv


def _call(lib, sv, n, out):
    return lib.iq_statevector_expval_z_all_noalloc(ctypes.c_void_p(sv.device_ptr()), n,
                                                   ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(sv.stream()))


def test_noalloc_matches_existing_entry_point_twice():
    """Two calls in a row (sharing the fixed scratch) agree with
    iq_statevector_expval_z_all at 1e-12, for sizes whose reduction uses a
    partial first chunk (1, 3, 8 qubits) and several chunks (11, 18)."""
    import torch
    from invariantq_b200 import _lib
    lib = _lib.load()
    for n, seed in ((18, 1), (11, 2), (8, 4), (3, 5), (1, 6)):
        sv = _state(n, seed) if n > 1 else None
        if sv is None:
            from invariantq_b200.binding import NativeStateVector
            sv = NativeStateVector(1)
            sv.apply_1q(0, np.array([[np.cos(0.3), -np.sin(0.3)], [np.sin(0.3), np.cos(0.3)]]))
        expected = sv.expval_z_all()            # the existing entry point (per-handle scratch)
        out = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        dev_before = torch.cuda.current_device()
        for _ in range(2):
            assert _call(lib, sv, n, out) == 0
            sv.sync()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.max(np.abs(got - expected)) < 1e-12, (n, got, expected)
            out.fill_(float("nan"))
        assert torch.cuda.current_device() == dev_before   # the caller's device is left as it was
        sv.close()


def test_noalloc_unnormalised_amplitudes():
    """Amplitudes that are not normalised: <Z_q> is sum|a|^2 - 2 sum_{bit q = 1} |a|^2."""
    import torch
    from invariantq_b200 import _lib
    from invariantq_b200.binding import NativeStateVector
    lib = _lib.load()
    n = 9
    rng = np.random.default_rng(9)
    a = 3.0 * (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n))
    sv = NativeStateVector(n)
    sv.set_amplitudes(a)
    p = np.abs(a) ** 2
    bits = (np.arange(1 << n)[:, None] >> np.arange(n)[None, :]) & 1
    want = p.sum() - 2.0 * (p[:, None] * bits).sum(0)
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        assert _call(lib, sv, n, out) == 0
        sv.sync()
        got = out.cpu().numpy()
        assert np.max(np.abs(got - want)) < 1e-12 * max(1.0, p.sum())
    assert np.max(np.abs(sv.expval_z_all() - want)) < 1e-12 * max(1.0, p.sum())
    sv.close()


def test_noalloc_leaves_free_device_memory_unchanged():
    """After its first call on the device (the one-time set-up), a call takes no
    device memory: the free memory the driver reports is the same afterwards."""
    import torch
    from invariantq_b200 import _lib
    from invariantq_b200.binding import jit_wait
    lib = _lib.load()
    n = 16
    sv = _state(n, 7)
    out = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert _call(lib, sv, n, out) == 0          # set-up call
    sv.sync()
    out.fill_(0.0)                              # torch's own kernel loaded before the measurement
    torch.cuda.synchronize()
    jit_wait(120.0)                             # no background kernel compilation in flight
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _call(lib, sv, n, out) == 0
    sv.sync()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.max(np.abs(out.cpu().numpy() - sv.expval_z_all())) < 1e-12
    sv.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from invariantq_b200 import _lib
    lib = _lib.load()
    sv = _state(8, 3)
    rc = lib.iq_statevector_expval_z_all_noalloc(ctypes.c_void_p(sv.device_ptr()), 35, ctypes.c_void_p(sv.device_ptr()),
                                                 ctypes.c_void_p(sv.stream()))
    assert rc == -1
    buf = ctypes.create_string_buffer(256)
    assert lib.iq_last_error(buf, 256) != 0
    assert b"scratch" in buf.value
    lib.iq_clear_error()
    # 34 qubits (the largest size) passes the size check: with host buffers the
    # call is then rejected for the memory kind, before anything is launched
    host = np.zeros(4)
    rc = lib.iq_statevector_expval_z_all_noalloc(host.ctypes.data_as(ctypes.c_void_p), 34,
                                                 host.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(sv.stream()))
    assert rc == -1
    assert lib.iq_last_error(buf, 256) != 0
    assert b"scratch" not in buf.value and b"device or managed memory" in buf.value
    lib.iq_clear_error()
    sv.close()

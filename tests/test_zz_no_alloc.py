"""The allocation-free <Z_q> entry point (iq_statevector_expval_z_all_noalloc).

It serves callers that cannot call cudaMalloc where they need the result (a
host whose GPU memory is already committed to the state, or code inside another
framework that owns the free device memory): they pass their own device buffers
and the library uses only a fixed scratch array it has held since loading.
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
    apply_abi(sv, gen_ops(np.random.default_rng(seed), n, 40, kmax=3))
    return sv


def test_noalloc_matches_existing_entry_point_twice():
    import torch
    from invariantq_b200 import _lib
    lib = _lib.load()
    for n, seed in ((18, 1), (11, 2)):
        sv = _state(n, seed)
        expected = sv.expval_z_all()            # the existing entry point (per-handle scratch)
        out = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        for _ in range(2):                      # two calls in a row share the fixed scratch
            rc = lib.iq_statevector_expval_z_all_noalloc(ctypes.c_void_p(sv.device_ptr()), n,
                                                          ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(sv.stream()))
            assert rc == 0
            sv.sync()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.max(np.abs(got - expected)) < 1e-12
            out.fill_(float("nan"))
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

"""Per-pass kernel generator (iq_jitgen.cpp) on the CPU: plans random and
brick-wall circuits with the scheduler, generates each pass's specialised
kernel source, and compiles it with NVRTC for sm_100a (NVRTC needs no GPU).
The GPU tests check the compiled kernels' amplitudes."""
import ctypes
import os
import re
from pathlib import Path

import numpy as np
import pytest

from tests.test_scheduler_emulated import brickwall_ops, emu, gen_ops, to_lsb   # noqa: F401  (fixture)

REPO = Path(__file__).resolve().parent.parent
CSRC = REPO / "invariantq_b200" / "csrc"


def nvrtc_lib():
    for name in ("/usr/local/cuda/lib64/libnvrtc.so.12", "libnvrtc.so.12"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    return None


def sources(emu, n, lsb_ops, M=12, c=5, R=4, budget=80.0, fuse=1):
    nops = len(lsb_ops)
    ks = np.array([len(q) for q, _ in lsb_ops], dtype=np.int32)
    qs = np.full((nops, 5), -1, dtype=np.int32)
    offs = np.zeros(nops, dtype=np.int64)
    pool, off = [], 0
    for i, (q, U) in enumerate(lsb_ops):
        qs[i, : len(q)] = q
        offs[i] = off
        flat = np.asarray(U, np.complex128).reshape(-1)
        pool.append(flat)
        off += flat.size
    pool = np.concatenate(pool)
    buf = ctypes.create_string_buffer(64 << 20)
    emu.emu_jit_sources.restype = ctypes.c_int
    rc = emu.emu_jit_sources(n, M, c, R, 8, ctypes.c_double(budget), fuse, nops,
                             ks.ctypes.data_as(ctypes.c_void_p), qs.ctypes.data_as(ctypes.c_void_p),
                             pool.ctypes.data_as(ctypes.c_void_p), offs.ctypes.data_as(ctypes.c_void_p),
                             buf, ctypes.c_longlong(len(buf)))
    text = buf.value.decode()
    assert rc > 0, text
    out = text.split("\n//@@PASS@@\n")
    assert len(out) == rc
    return out


def compile_nvrtc(lib, src):
    names = [b"iq_plan.h", b"iq_pipe.cuh"]
    texts = [(CSRC / n.decode()).read_bytes() for n in names]
    prog = ctypes.c_void_p()
    arr_n = (ctypes.c_char_p * 2)(*names)
    arr_t = (ctypes.c_char_p * 2)(*texts)
    assert lib.nvrtcCreateProgram(ctypes.byref(prog), src.encode(), b"pass.cu", 2, arr_t, arr_n) == 0
    opts = [b"-arch=sm_100a", b"-std=c++17", b"-default-device"]
    rc = lib.nvrtcCompileProgram(prog, len(opts), (ctypes.c_char_p * len(opts))(*opts))
    n = ctypes.c_size_t()
    lib.nvrtcGetProgramLogSize(prog, ctypes.byref(n))
    log = ctypes.create_string_buffer(n.value + 1)
    lib.nvrtcGetProgramLog(prog, log)
    size = ctypes.c_size_t()
    if rc == 0:
        lib.nvrtcGetCUBINSize(prog, ctypes.byref(size))
    lib.nvrtcDestroyProgram(ctypes.byref(prog))
    return rc, log.value.decode(), size.value


def test_generated_sources_are_straight_line(emu):
    rng = np.random.default_rng(3)
    n = 14
    ops = [to_lsb(*o) for o in gen_ops(rng, n, 60, kmax=4)]
    srcs = sources(emu, n, ops, R=4)
    for s in srcs:
        assert "iq_jit_pass" in s and "tile_pipeline<128>" in s
        assert "switch" not in s                       # no run-time dispatch
        # every matrix entry is read from the kernel parameters
        for m in re.findall(r"Mt\.m\[(\d+)\]", s):
            size = int(re.search(r"double2 m\[(\d+)\]", s).group(1))
            assert int(m) < size


@pytest.mark.parametrize("R,kmax", [(4, 4), (3, 3), (5, 5)])
def test_generated_kernels_compile(emu, R, kmax):
    lib = nvrtc_lib()
    if lib is None:
        pytest.skip("libnvrtc not available")
    rng = np.random.default_rng(10 + R)
    n = 13
    ops = [to_lsb(*o) for o in gen_ops(rng, n, 40, kmax=kmax)]
    srcs = sources(emu, n, ops, R=R)
    for s in srcs[:3]:
        rc, log, size = compile_nvrtc(lib, s)
        assert rc == 0, log[:3000]
        assert size > 0


def test_brickwall_kernel_compiles(emu):
    lib = nvrtc_lib()
    if lib is None:
        pytest.skip("libnvrtc not available")
    n = 20
    ops = [to_lsb(*o) for o in brickwall_ops(n, 8, 1)]
    srcs = sources(emu, n, ops, M=11, budget=120.0)
    rc, log, size = compile_nvrtc(lib, max(srcs, key=len))
    assert rc == 0, log[:3000]


@pytest.mark.parametrize("narrow", [0, 1])
def test_adjoint_kernels_compile(emu, narrow):
    """The shared-memory form the adjoint executor runs (parameter sets,
    adjoint steps with gradient accumulators), for complex128 arrays through
    the TMA pipeline and for complex64 arrays with direct loads and stores."""
    from tests import adjoint_ref as ar
    lib = nvrtc_lib()
    if lib is None:
        pytest.skip("libnvrtc not available")
    n = 12
    ops = ar.tfim_ops(n, 2)
    th = np.random.default_rng(4).uniform(0, 2 * np.pi, ar.n_params(ops))
    k = np.array([o[0] for o in ops], np.int32)
    q0 = np.array([o[1] for o in ops], np.int32)
    q1 = np.array([o[2] for o in ops], np.int32)
    pi = np.array([o[3] for o in ops], np.int32)
    buf = ctypes.create_string_buffer(64 << 20)
    P = ctypes.c_void_p
    rc = emu.emu_adjoint_sources(n, len(ops), P(k.ctypes.data), P(q0.ctypes.data), P(q1.ctypes.data),
                                 P(pi.ctypes.data), P(th.ctypes.data), 12, 4, 4, 8, ctypes.c_double(160.0), narrow,
                                 buf, ctypes.c_longlong(len(buf)))
    text = buf.value.decode()
    assert rc > 0, text
    srcs = text.split("\n//@@PASS@@\n")
    assert all(("narrow=1" in s) == bool(narrow) for s in srcs)
    # every adjoint-step form: phase-free Z steps, and the single-set plans'
    # tan / cot Y steps
    forms = ["unrotate<2, 1>", "unrotate<1, 1>", "unrotate<1, 2>"]
    picked = [next(s for s in srcs if f in s) for f in forms]
    for s in [srcs[0], max(srcs, key=len)] + picked:
        rc, log, size = compile_nvrtc(lib, s)
        assert rc == 0, log[:3000]
        assert size > 0


def test_channel_kernels_compile(emu):
    """Passes of a noisy density-matrix circuit in the specialised style hold
    X2R operations (xpat4 on real / complex corners and middle) that compile."""
    from tests.test_scheduler_emulated import superop_lsb
    from invariantq_b200.channels import build_kraus_channel
    from invariantq_b200.gates import gate_matrix
    lib = nvrtc_lib()
    if lib is None:
        pytest.skip("libnvrtc not available")
    nq, rng = 8, np.random.default_rng(2)
    dep = superop_lsb(build_kraus_channel("depolarizing", [1e-3]))
    amp = superop_lsb(build_kraus_channel("amp_damping", [2e-3]))
    ops = []
    for q in range(nq):
        U = gate_matrix("u3", list(rng.uniform(0, 2 * np.pi, 3)))
        ops += [([nq + q], U), ([q], np.conj(U)), ([q, nq + q], dep), ([q, nq + q], amp)]
    srcs = sources(emu, 2 * nq, ops, M=12, c=4, budget=160.0, fuse=2)
    picked = [s for s in srcs if "xpat4<" in s]
    assert picked
    rc, log, size = compile_nvrtc(lib, max(picked, key=len))
    assert rc == 0, log[:3000]

"""CPU checks of the shared library: it loads without a GPU, exports every
function include/invariantq_b200.h declares (which covers the reference's 49
c_api.h symbols), and creating a handle without a GPU fails cleanly."""
import ctypes
import re
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def lib():
    from invariantq_b200 import _lib
    if not _lib.LIB_PATH.exists():
        from invariantq_b200.build import build
        build()
    return _lib.load()


def header_symbols():
    text = (REPO / "include" / "invariantq_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(iq_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol(lib):
    names = header_symbols()
    assert len(names) >= 49
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_abi_is_covered(lib):
    ref = (REPO / "tests" / "golden" / "c_api_symbols.txt").read_text().split()
    assert len(ref) == 49
    assert set(ref) <= set(header_symbols())
    for n in ref:
        assert hasattr(lib, n)


def test_binding_signatures_cover_header():
    from invariantq_b200._lib import SIGNATURES
    assert set(header_symbols()) <= set(SIGNATURES)


def test_create_without_gpu_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    assert not lib.iq_statevector_create(4)
    buf = ctypes.create_string_buffer(256)
    assert lib.iq_last_error(buf, 256) != 0
    assert buf.value
    lib.iq_clear_error()
    from invariantq_b200.binding import NativeStateVector
    with pytest.raises(Exception):
        NativeStateVector(3)


def test_stabilizer_mps_forwarding_without_cpu_core(lib):
    import os
    if os.environ.get("IQ_CPU_CORE_LIB"):
        pytest.skip("a CPU core is configured")
    assert not lib.iq_stabilizer_create(3)
    assert lib.iq_last_error(None, 0) == 6
    lib.iq_clear_error()

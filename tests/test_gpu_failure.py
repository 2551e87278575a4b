"""Failure detection on the GPU without a GPU fault: the tile kernel's bounded
wait gives up on an mbarrier phase that nothing completes, and reports it in
the status word; a handle whose status word reports a timed-out pass raises
on its next synchronising call, clears it, and keeps working."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
H = np.array([[1, 1], [1, -1]]) / np.sqrt(2)
X = np.array([[0, 1], [1, 0]])


def test_bounded_wait_gives_up_and_reports():
    from invariantq_b200.binding import selftest_bounded_wait
    for limit in (5.0, 50.0):
        st, waited = selftest_bounded_wait(limit)
        assert st == 1                              # a tile load that did not complete
        assert 0.9 * limit <= waited < limit + 250.0   # warps start their clocks a few ns apart
    with pytest.raises(ValueError):
        selftest_bounded_wait(0.0)


def test_context_usable_after_bounded_wait():
    from invariantq_b200.binding import NativeStateVector, selftest_bounded_wait
    assert selftest_bounded_wait(10.0)[0] == 1
    sv = NativeStateVector(14)
    try:
        for q in range(14):
            sv.apply_1q(q, H)
        sv.sync()
        assert abs(sv.norm_squared() - 1.0) < 1e-12
        assert np.max(np.abs(sv.expval_z_all())) < 1e-12
    finally:
        sv.close()


def test_status_word_raises_then_recovers():
    from invariantq_b200._lib import IQError
    from invariantq_b200.binding import NativeStateVector
    sv = NativeStateVector(12)
    try:
        sv.apply_1q(3, H)
        sv.set_option("inject_status", 1)
        with pytest.raises(IQError, match="timed out waiting for a tile load"):
            sv.sync()
        sv.set_option("inject_status", 2)
        with pytest.raises(IQError, match="its consumers"):
            sv.expval_z_all()
        with pytest.raises(ValueError):
            sv.set_option("inject_status", 7)
        sv.reset()                                   # the status word was cleared by the report
        sv.apply_1q(5, X)
        sv.sync()
        z = sv.expval_z_all()
        assert z[5] == -1.0 and z[3] == 1.0
    finally:
        sv.close()

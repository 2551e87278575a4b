"""Measurement shots on the device: the mt19937_64 stream generated by the GPU
equals the oracle's restatement of std::mt19937_64 with
uniform_real_distribution(0, 1) bit for bit; shots equal the oracle's
(statevector.cpp:235-256: serial CDF, lower_bound) on random states; the counts
computed on the device equal the counts of the shots."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [0, 7, 42, 2 ** 63 + 12345])
def test_device_mt19937_64_stream(port, seed):
    import ctypes
    from invariantq_b200.binding import mt64_uniform
    n = 5000
    want = np.empty(n)
    port.L.or_mt64_uniform(ctypes.c_uint64(seed), n, want.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    got = mt64_uniform(seed, n)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n,shots,seed", [(5, 1000, 3), (13, 8192, 11), (17, 20000, 5)])
def test_shots_and_counts_vs_oracle(port, n, shots, seed):
    from invariantq_b200.binding import NativeStateVector
    rng = np.random.default_rng(n)
    a = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    a /= np.linalg.norm(a)
    sv = NativeStateVector(n)
    sv.set_amplitudes(a)
    got = sv.sample(shots, seed)
    want = port.sample(a.copy(), n, shots, seed)
    assert np.mean(got == want) > 0.999           # identical but for a shot on a block boundary
    vals, cnts = sv.sample_counts(shots, seed)
    u, c = np.unique(got, return_counts=True)
    assert np.array_equal(vals, u) and np.array_equal(cnts, c)
    assert int(cnts.sum()) == shots and np.all(np.diff(vals.astype(np.int64)) > 0)
    sv.close()

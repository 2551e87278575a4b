"""The sharded state vector (invariantq_b200/sharded.py) on CPU ranks (gloo):
the qubit-remap logic and the pairwise half-slice exchanges, with a NumPy
stand-in for each rank's GPU slice.  2 and 4 ranks run random circuits of
one-, two- and three-qubit gates (on global qubits too); rank 0 compares the
gathered state, <Z_q> and the norm with an unsharded NumPy run: 1e-12."""
import datetime
import os
import pickle
import socket

import numpy as np
import pytest


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def apply_ir(state, n, qubits, U):
    """Gate in the IR convention (first listed qubit = most significant bit of
    the matrix index) on a state whose index bit q is qubit q."""
    k = len(qubits)
    t = state.reshape([2] * n)                   # axis n-1-q <-> qubit q
    axes = [n - 1 - q for q in qubits]
    t = np.moveaxis(t, axes, list(range(k)))
    shp = t.shape
    t = (np.asarray(U, np.complex128) @ t.reshape(1 << k, -1)).reshape(shp)
    return np.moveaxis(t, list(range(k)), axes).reshape(-1)


class NumpySlice:
    """A rank's slice held as a NumPy vector (test stand-in for NativeSlice)."""

    def __init__(self, local_bits):
        self.n = local_bits
        self.s = np.zeros(1 << local_bits, np.complex128)

    def apply(self, phys, matrix):
        self.s = apply_ir(self.s, self.n, list(phys), matrix)

    def set_zero(self, is_origin):
        self.s[:] = 0
        if is_origin:
            self.s[0] = 1

    def _half(self, bit, value):
        idx = np.arange(1 << self.n)
        return idx[((idx >> bit) & 1) == value]

    def pack(self, bit, value):
        import torch
        h = self.s[self._half(bit, value)]
        return torch.from_numpy(np.stack([h.real, h.imag], 1).copy())

    def unpack(self, bit, value, buf):
        a = buf.numpy()
        self.s[self._half(bit, value)] = a[:, 0] + 1j * a[:, 1]

    def norm_and_z(self):
        p = np.abs(self.s) ** 2
        bits = (np.arange(1 << self.n)[:, None] >> np.arange(self.n)[None, :]) & 1
        return float(p.sum()), (p[:, None] * (1 - 2 * bits)).sum(0)

    def amplitudes(self):
        return self.s.copy()

    def close(self):
        pass


def random_gates(n, count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        k = int(rng.choice([1, 2, 2, 3]))
        qs = [int(q) for q in rng.choice(n, k, replace=False)]
        z = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
        q, r = np.linalg.qr(z)
        out.append((qs, q * (np.diag(r) / np.abs(np.diag(r)))))
    return out


def _rank(rank, world, port, n, seed, out_dir):
    import torch.distributed as dist
    from invariantq_b200.sharded import ShardedStateVector, TorchComm
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sv = ShardedStateVector(n, TorchComm(), backend=NumpySlice)
        for qs, U in random_gates(n, 60, seed):
            sv.apply(qs, U)
        amps = sv.get_amplitudes()
        z = sv.expval_z_all()
        nrm = sv.norm_squared()
        if rank == 0:
            with open(os.path.join(out_dir, "sharded.pkl"), "wb") as f:
                pickle.dump((amps, z, nrm, sv.exchanges), f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n", [(2, 6), (4, 7)])
def test_sharded_state_vector_gloo(tmp_path, world, n):
    import torch.multiprocessing as mp
    seed = 10 + world
    mp.start_processes(_rank, args=(world, free_port(), n, seed, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    amps, z, nrm, exchanges = pickle.load(open(tmp_path / "sharded.pkl", "rb"))
    ref = np.zeros(1 << n, np.complex128)
    ref[0] = 1
    for qs, U in random_gates(n, 60, seed):
        ref = apply_ir(ref, n, qs, U)
    assert exchanges > 0
    assert np.max(np.abs(amps - ref)) < 1e-12
    p = np.abs(ref) ** 2
    bits = (np.arange(1 << n)[:, None] >> np.arange(n)[None, :]) & 1
    assert np.max(np.abs(z - (p[:, None] * (1 - 2 * bits)).sum(0))) < 1e-12
    assert abs(nrm - 1.0) < 1e-12


def test_apply_ir_convention():
    """The stand-in's gate convention is the library's: CX with control listed
    first flips the second qubit when the first is 1."""
    CX = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]])
    s = np.zeros(8, np.complex128)
    s[0b001] = 1                       # qubit 0 = 1
    out = apply_ir(s, 3, [0, 2], CX)   # control 0, target 2
    assert out[0b101] == 1

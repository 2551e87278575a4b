"""The sharded state vector's GPU pieces: the half-slice pack / unpack kernels
(iq_statevector_pack_half / unpack_half) against NumPy, and a 20-qubit
brick-wall sharded over 2 ranks -- two processes on this one GPU, each holding
a 19-qubit slice through the library, exchanging halves through gloo (host
memory; no kernel waits on another rank) -- against the unsharded library run
(1e-12).  Several GPUs exchange through NCCL with the same code."""
import datetime
import os
import pickle

import numpy as np
import pytest

from tests.test_sharded import free_port

pytestmark = pytest.mark.gpu


def test_pack_unpack_half():
    import torch
    from invariantq_b200.binding import NativeStateVector
    n = 12
    rng = np.random.default_rng(3)
    a = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    sv = NativeStateVector(n)
    sv.set_amplitudes(a)
    idx = np.arange(1 << n)
    for bit in (0, 4, 5, 11):
        for val in (0, 1):
            buf = torch.empty((1 << (n - 1), 2), dtype=torch.float64, device="cuda")
            sv.pack_half(bit, val, buf.data_ptr())
            got = buf.cpu().numpy()
            want = a[((idx >> bit) & 1) == val]
            assert np.array_equal(got[:, 0] + 1j * got[:, 1], want)
    new = rng.normal(size=(1 << (n - 1), 2))
    sv.unpack_half(7, 1, torch.from_numpy(new).cuda().data_ptr())
    b = a.copy()
    b[((idx >> 7) & 1) == 1] = new[:, 0] + 1j * new[:, 1]
    assert np.array_equal(sv.get_amplitudes(), b)
    with pytest.raises(ValueError):
        sv.pack_half(n, 0, buf.data_ptr())
    sv.close()


def _rank(rank, world, port, n, depth, out_dir):
    import torch
    import torch.distributed as dist
    from invariantq_b200.circuits import brickwall
    from invariantq_b200.sharded import ShardedStateVector, TorchComm
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        c = brickwall(n, depth, seed=9)
        sv = ShardedStateVector(n, TorchComm())
        for op in c.ops:
            sv.apply([c.get_qubit_index(q) for q in op.qubits], op.matrix)
        amps = sv.get_amplitudes()
        z = sv.expval_z_all()
        nrm = sv.norm_squared()
        if rank == 0:
            with open(os.path.join(out_dir, "gpu_sharded.pkl"), "wb") as f:
                pickle.dump((amps, z, nrm, sv.exchanges), f)
        dist.barrier()
        sv.close()
    finally:
        dist.destroy_process_group()


def test_sharded_brickwall_two_ranks_one_gpu(tmp_path):
    import torch.multiprocessing as mp
    from invariantq_b200.binding import NativeStateVector
    from invariantq_b200.circuits import brickwall
    from invariantq_b200.simulator import apply_gate_matrix
    n, depth, world = 20, 6, 2
    mp.start_processes(_rank, args=(world, free_port(), n, depth, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    amps, z, nrm, exchanges = pickle.load(open(tmp_path / "gpu_sharded.pkl", "rb"))
    c = brickwall(n, depth, seed=9)
    sv = NativeStateVector(n)
    for op in c.ops:
        apply_gate_matrix(sv, [c.get_qubit_index(q) for q in op.qubits], op.matrix)
    ref = sv.get_amplitudes()
    assert exchanges > 0
    assert np.max(np.abs(amps - ref)) < 1e-12
    assert np.max(np.abs(z - sv.expval_z_all())) < 1e-12
    assert abs(nrm - 1.0) < 1e-12
    sv.close()

"""Two ranks on the CPU (gloo) running the replica logic bench.py uses with one
process per GPU: disjoint, covering shares of the 256-circuit gradient batch,
the max-over-ranks timing reduction, and sharded gradients equal to the
unsharded ones.  Each rank computes its share through the CPU emulator of the
planned passes (no collective on the data path); rank 0 compares."""
import datetime
import os
import pickle
import socket
import subprocess
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
SMALL = [(5, 2, 1), (6, 2, 2), (7, 1, 3), (8, 2, 4), (6, 3, 5)]   # (qubits, layers, seed)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def emulated(emu_path, items):
    import ctypes
    from invariantq_b200.circuits import tfim_terms
    from tests import adjoint_ref as ar
    from tests.test_adjoint_emulated import emu_grad
    emu = ctypes.CDLL(emu_path)
    out = {}
    for n, layers, seed in items:
        ops = ar.tfim_ops(n, layers)
        th = np.random.default_rng(seed).uniform(0, 2 * np.pi, ar.n_params(ops))
        c, p = tfim_terms(n, 1.0)
        out[(n, layers, seed)] = emu_grad(emu, n, ops, th, c, p)
    return out


def _rank(rank, world, port, emu_path, out_dir):
    import torch.distributed as dist
    from bench import gradient_jobs
    from invariantq_b200.replicas import max_over_ranks, shard
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        jobs = gradient_jobs(256, 16)
        mine = shard(list(range(len(jobs))), rank, world)
        qubits = [jobs[i][0].num_qubits for i in mine]
        t = max_over_ranks(0.25 * (rank + 1))
        res = emulated(emu_path, shard(SMALL, rank, world))
        gathered = [None] * world
        dist.all_gather_object(gathered, (mine, qubits, t, res))
        if rank == 0:
            with open(os.path.join(out_dir, "ranks.pkl"), "wb") as f:
                pickle.dump(gathered, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def emu_path(tmp_path_factory):
    out = tmp_path_factory.mktemp("emu_mp") / "libplanemu.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(out),
                    str(REPO / "tests" / "plan_emulator.cpp"),
                    str(REPO / "invariantq_b200" / "csrc" / "iq_sched.cpp"),
                    str(REPO / "invariantq_b200" / "csrc" / "iq_jitgen.cpp")], check=True)
    return str(out)


def test_two_ranks_gloo(emu_path, tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank, args=(world, free_port(), emu_path, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    gathered = pickle.loads((tmp_path / "ranks.pkl").read_bytes())
    shares = [g[0] for g in gathered]
    assert sorted(shares[0] + shares[1]) == list(range(256))           # every circuit exactly once
    assert not set(shares[0]) & set(shares[1])
    assert abs(len(shares[0]) - len(shares[1])) <= 1
    q0, q1 = np.mean(gathered[0][1]), np.mean(gathered[1][1])           # interleaved: similar sizes
    assert abs(q0 - q1) < 1.5
    assert all(g[2] == 0.5 for g in gathered)                           # MAX over ranks
    merged = {}
    for g in gathered:
        merged.update(g[3])
    alone = emulated(emu_path, SMALL)
    assert set(merged) == set(alone)
    for k, (e, g) in alone.items():
        e2, g2 = merged[k]
        assert e2 == e and np.array_equal(g2, g)


def test_shard_rejects_bad_rank():
    from invariantq_b200.replicas import max_over_ranks, shard
    with pytest.raises(ValueError):
        shard([1, 2, 3], 2, 2)
    assert shard(list(range(7)), 1, 3) == [1, 4]
    assert max_over_ranks(1.5) == 1.5    # no process group: the value itself


def _leaving_rank(rank, world, port, out_dir):
    """Rank 1 leaves after the first step (between steps: nothing of its own in
    flight); rank 0 goes on to the next step's timing reduction, which must end
    with an error, not wait for good."""
    import time
    import torch.distributed as dist
    from invariantq_b200.replicas import max_over_ranks
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    first = max_over_ranks(1.0 + rank)
    if rank == 1:
        dist.destroy_process_group()
        return
    t0 = time.monotonic()
    try:
        max_over_ranks(3.0)
        outcome = "completed"
    except Exception as exc:                       # gloo: connection closed, or the group's timeout
        outcome = type(exc).__name__
    elapsed = time.monotonic() - t0
    with open(os.path.join(out_dir, "leave.pkl"), "wb") as f:
        pickle.dump((first, outcome, elapsed), f)
    try:
        dist.destroy_process_group()
    except Exception:
        pass


def test_rank_leaving_ends_next_collective_with_error(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_leaving_rank, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    first, outcome, elapsed = pickle.loads((tmp_path / "leave.pkl").read_bytes())
    assert first == 2.0                 # the step both ranks took
    assert outcome != "completed"
    assert elapsed < 30.0               # bounded by the 5 s group timeout (plus teardown)

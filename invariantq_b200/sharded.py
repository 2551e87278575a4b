"""A state vector sharded across GPUs (one process per GPU) by its top qubits.

With P = 2^g ranks, rank r holds the 2^(n-g) amplitudes whose top g physical
index bits equal r; gates run on each rank's slice through the library's C ABI
(every pass local to one GPU).  A gate on a qubit that sits on a global bit
first swaps that qubit with a local one: each rank sends the half of its slice
whose local bit is the other value of the global bit to the partner rank that
differs in that bit and receives the partner's matching half (one pairwise
exchange of half a slice, `iq_statevector_pack_half` / `unpack_half` around a
send/receive).  The mapping logical qubit -> physical bit is kept on the host
and undone when amplitudes are gathered.

The exchange runs through ``torch.distributed`` (NCCL between GPUs; with the
gloo backend the halves travel through host memory).  The reference has no
multi-device state vector (its dense path stops at 16 GiB,
invariantq/simulator/adaptive.py:29,87); this is the path past one GPU.
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np


class TorchComm:
    """Pairwise exchange, sums and gathers over a torch.distributed group."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.host_staged = dist.get_backend(group) == "gloo"

    def exchange(self, send, partner: int):
        """Send tensor `send` to `partner` and return the tensor of the same
        shape received from it."""
        import torch
        src = send.cpu() if (self.host_staged and send.is_cuda) else send
        recv = torch.empty_like(src)
        peer = self.dist.get_global_rank(self.group, partner) if self.group is not None else partner
        ops = [self.dist.P2POp(self.dist.isend, src, peer, self.group),
               self.dist.P2POp(self.dist.irecv, recv, peer, self.group)]
        for req in self.dist.batch_isend_irecv(ops):
            req.wait()
        return recv.to(send.device) if recv.device != send.device else recv

    def all_sum(self, x: np.ndarray) -> np.ndarray:
        import torch
        t = torch.as_tensor(np.asarray(x, np.float64).copy())
        if self.dist.get_backend(self.group) == "nccl":
            t = t.cuda()
        self.dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def gather(self, x: np.ndarray) -> Optional[List[np.ndarray]]:
        """Every rank's array on rank 0 (None elsewhere)."""
        import torch
        t = torch.as_tensor(np.ascontiguousarray(x))
        if self.dist.get_backend(self.group) == "nccl":
            t = t.cuda()
        parts = [torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(parts, t, group=self.group)
        return [p.cpu().numpy() for p in parts] if self.rank == 0 else None


class NativeSlice:
    """One rank's slice on its GPU: a NativeStateVector of the local qubits."""

    def __init__(self, local_bits: int):
        from .binding import NativeStateVector
        self.n = int(local_bits)
        self.sv = NativeStateVector(self.n)

    def apply(self, phys: Sequence[int], matrix) -> None:
        from .simulator import apply_gate_matrix
        apply_gate_matrix(self.sv, list(phys), np.asarray(matrix, np.complex128))

    def set_zero(self, is_origin: bool) -> None:
        self.sv.reset()
        if not is_origin:   # all zeros: the zero matrix on one qubit (the ABI takes any matrix)
            self.sv.apply_1q(0, np.zeros((2, 2), np.complex128))

    def pack(self, bit: int, value: int):
        import torch
        buf = torch.empty((1 << (self.n - 1), 2), dtype=torch.float64, device="cuda")
        self.sv.pack_half(bit, value, buf.data_ptr())
        return buf

    def unpack(self, bit: int, value: int, buf) -> None:
        import torch
        buf = buf.contiguous()
        torch.cuda.synchronize()
        self.sv.unpack_half(bit, value, buf.data_ptr())

    def norm_and_z(self):
        """(sum |a|^2, [sum |a|^2 (1 - 2 bit_b)] for local bits b)."""
        return self.sv.norm_squared(), self.sv.expval_z_all()

    def amplitudes(self) -> np.ndarray:
        return self.sv.get_amplitudes()

    def close(self) -> None:
        self.sv.close()


class ShardedStateVector:
    """n qubits over the ranks of `comm` (a power of two, at most 2^(n-3))."""

    def __init__(self, num_qubits: int, comm=None, backend=NativeSlice):
        self.comm = comm or TorchComm()
        P = self.comm.world
        g = P.bit_length() - 1
        if (1 << g) != P:
            raise ValueError("the number of ranks must be a power of two")
        self.n = int(num_qubits)
        if self.n - g < 3:
            raise ValueError("every rank needs at least 3 local qubits")
        self.g, self.L = g, self.n - g
        self.rank = self.comm.rank
        self.slice = backend(self.L)
        self.pos = list(range(self.n))     # logical qubit -> physical bit
        self.at = list(range(self.n))      # physical bit -> logical qubit
        self.last_use = [0] * self.L       # per local physical bit: step of its last use
        self.step = 0
        self.exchanges = 0
        self.reset()

    def reset(self) -> None:
        """|0...0>: amplitude 1 at index 0, on rank 0."""
        self.slice.set_zero(self.rank == 0)

    def _swap_in(self, logical: int, keep: Sequence[int]) -> None:
        """Move `logical` (on a global bit) onto the least recently used local
        bit whose qubit is not in `keep`."""
        p = self.pos[logical]
        cand = [b for b in range(self.L) if self.at[b] not in keep]
        v = min(cand, key=lambda b: self.last_use[b])
        gbit = p - self.L
        mine = (self.rank >> gbit) & 1
        partner = self.rank ^ (1 << gbit)
        send = self.slice.pack(v, 1 - mine)
        recv = self.comm.exchange(send, partner)
        self.slice.unpack(v, 1 - mine, recv)
        a, b = self.at[p], self.at[v]
        self.pos[a], self.pos[b] = v, p
        self.at[p], self.at[v] = b, a
        self.exchanges += 1

    def apply(self, qubits: Sequence[int], matrix) -> None:
        """A gate in the IR convention (first listed qubit = most significant
        bit of the matrix index), as simulator.apply_gate_matrix takes it."""
        qubits = [int(q) for q in qubits]
        if len(set(qubits)) != len(qubits) or any(not 0 <= q < self.n for q in qubits):
            raise ValueError("invalid qubits")
        if len(qubits) > self.L:
            raise ValueError("a gate is wider than the local qubits")
        self.step += 1
        for q in qubits:
            if self.pos[q] >= self.L:
                self._swap_in(q, qubits)
        phys = [self.pos[q] for q in qubits]
        for b in phys:
            self.last_use[b] = self.step
        self.slice.apply(phys, matrix)

    def norm_squared(self) -> float:
        nrm, _ = self.slice.norm_and_z()
        return float(self.comm.all_sum(np.array([nrm]))[0])

    def expval_z_all(self) -> np.ndarray:
        """<Z_q> for every logical qubit."""
        nrm, z = self.slice.norm_and_z()
        out = np.zeros(self.n)
        for q in range(self.n):
            p = self.pos[q]
            out[q] = z[p] if p < self.L else nrm * (1.0 - 2.0 * ((self.rank >> (p - self.L)) & 1))
        return self.comm.all_sum(out)

    def get_amplitudes(self) -> Optional[np.ndarray]:
        """The full state in logical index order, on rank 0 (None elsewhere)."""
        parts = self.comm.gather(self.slice.amplitudes())
        if parts is None:
            return None
        full = np.concatenate(parts)               # physical index = rank << L | local index
        n = self.n
        t = full.reshape([2] * n)                  # axis j <-> physical bit n-1-j
        axes = [n - 1 - self.pos[n - 1 - j] for j in range(n)]
        return np.ascontiguousarray(t.transpose(axes)).reshape(-1)

    def close(self) -> None:
        self.slice.close()

"""Gate fusion into unitary blocks of up to ``max_fused_qubits`` wires (2..5).

Mirrors the reference compiler's pass interface
(invariantq/compiler/gate_fusion_pass.py:12-23: ``GateFusionPass(max_fused_qubits=2)``,
``run(circuit) -> circuit`` emitting ``FusedGateOp(fused_matrix, original_ops)``),
written from scratch with a correct k-qubit lifting: the reference's
``_lift_unitary`` returns the identity for more than two wires
(gate_fusion_pass.py:136-154) and its contiguous grouping never forms blocks
wider than two on a brick-wall.

Algorithm (greedy, one sweep in program order).  Every wire belongs to at most
one *open* block.  A gate on wires Q merges with the open blocks that own wires
of Q when the union of their wires has at most ``max_fused_qubits`` wires;
open blocks on disjoint wires commute, so merging them is exact.  Otherwise
those blocks are closed -- emitted in creation order -- and the gate opens a
new block.  Measurements, resets, noise and barriers close the blocks on
their wires (a barrier closes all).  A closed block precedes every later
operation on its wires, so the emitted order respects every dependency.

Block matrices are kept LSB-first over the block's wire list and emitted in
the C ABI convention of their width (the convention ``apply_fused`` takes):
k = 1 and k = 2 with the first listed wire the most significant local bit,
k >= 3 with local index bit b on ``qubits[b]`` (core/src/statevector.cpp:
69-72, 133-139).  A block holding a single original gate is emitted as that
gate unchanged.
"""
from __future__ import annotations

import copy
from typing import Dict, List, Optional, Sequence

import numpy as np

from .ir import BarrierOp, CircuitIR, FusedGateOp, GateOp, op_kind


def embed_lsb(u: np.ndarray, sub: Sequence[int], full: Sequence[int]) -> np.ndarray:
    """The 2^m x 2^m matrix of ``u`` (LSB-first over wires ``sub``: local bit b
    is wire sub[b]) acting on wires ``full`` (LSB-first), identity elsewhere."""
    m, k = len(full), len(sub)
    pos = [list(full).index(w) for w in sub]
    dim = 1 << m
    idx = np.arange(dim)
    sub_bits = np.zeros(dim, dtype=np.int64)
    for b, p in enumerate(pos):
        sub_bits |= ((idx >> p) & 1) << b
    mask = 0
    for p in pos:
        mask |= 1 << p
    rest = idx & ~mask
    out = np.zeros((dim, dim), np.complex128)
    same = rest[:, None] == rest[None, :]
    vals = u[sub_bits[:, None], sub_bits[None, :]]
    out[same] = vals[same]
    return out


def msb_to_lsb(u: np.ndarray) -> np.ndarray:
    """Reorder a matrix whose first listed wire is the most significant bit to
    LSB-first over the same wire list (a bit reversal of the local index; the
    same matrix is LSB-first over the reversed wire list)."""
    k = int(round(np.log2(u.shape[0])))
    if k <= 1:
        return np.asarray(u, np.complex128)
    perm = np.zeros(1 << k, dtype=np.int64)
    for i in range(1 << k):
        r = 0
        for b in range(k):
            r |= ((i >> b) & 1) << (k - 1 - b)
        perm[i] = r
    return np.asarray(u, np.complex128)[np.ix_(perm, perm)]


class _Block:
    __slots__ = ("wires", "mat", "ops", "order")

    def __init__(self, wires: List[int], mat: np.ndarray, ops: list, order: int):
        self.wires = wires      # LSB-first wire list
        self.mat = mat          # LSB-first over wires
        self.ops = ops          # original GateOps, program order
        self.order = order      # creation index (emission order among closed blocks)


class GateFusionPass:
    """Fuse gates into unitary blocks of at most ``max_fused_qubits`` wires."""

    def __init__(self, max_fused_qubits: int = 2):
        if not 1 <= int(max_fused_qubits) <= 5:
            raise ValueError("max_fused_qubits must be 1..5 (the C ABI applies blocks of up to 5 wires)")
        self.max_fused_qubits = int(max_fused_qubits)

    def run(self, circuit: CircuitIR) -> CircuitIR:
        out = CircuitIR(getattr(circuit, "name", "circuit") + "_fused")
        for name, size in circuit.qubit_regs.items():
            out.add_qubit_register(name, size)
        for name, size in getattr(circuit, "clbit_regs", {}).items():
            out.add_clbit_register(name, size)
        wire_obj: Dict[int, object] = {}
        for op in circuit.ops:
            for q in op.qubits:
                wire_obj[circuit.get_qubit_index(q)] = q
        open_of: Dict[int, _Block] = {}
        counter = [0]

        def close(blocks: List[_Block]) -> None:
            for b in sorted(set(blocks), key=lambda x: x.order):
                for w in b.wires:
                    if open_of.get(w) is b:
                        del open_of[w]
                out.add_op(self._emit(b, wire_obj))

        for op in circuit.ops:
            kind = op_kind(op)
            wires = [circuit.get_qubit_index(q) for q in op.qubits]
            if kind == "GateOp" and len(wires) <= self.max_fused_qubits:
                # a gate matrix is MSB-first over its listed wires, which is the same
                # index as LSB-first over the reversed list
                lsb = list(reversed(wires))
                u = np.asarray(op.matrix, np.complex128)
                owners = []
                for w in wires:
                    b = open_of.get(w)
                    if b is not None and b not in owners:
                        owners.append(b)
                union: List[int] = []
                for b in owners:
                    union += b.wires
                union += [w for w in lsb if w not in union]
                if len(union) <= self.max_fused_qubits:
                    mat = np.eye(1 << len(union), dtype=np.complex128)
                    ops: list = []
                    for b in sorted(owners, key=lambda x: x.order):
                        mat = embed_lsb(b.mat, b.wires, union) @ mat
                        ops += b.ops
                    mat = embed_lsb(u, lsb, union) @ mat
                    nb = _Block(union, mat, ops + [op], counter[0])
                    counter[0] += 1
                    for w in union:
                        open_of[w] = nb
                    continue
                close(owners)
                nb = _Block(lsb, u, [op], counter[0])
                counter[0] += 1
                for w in lsb:
                    open_of[w] = nb
                continue
            # not fusable here: close what it touches (a barrier closes everything)
            if isinstance(op, BarrierOp) or kind == "BarrierOp":
                close(list(open_of.values()))
            else:
                close([open_of[w] for w in wires if w in open_of])
            out.add_op(copy.copy(op))
        close(list(open_of.values()))
        return out

    @staticmethod
    def _emit(b: _Block, wire_obj: Dict[int, object]):
        if len(b.ops) == 1:
            return copy.copy(b.ops[0])
        k = len(b.wires)
        # k <= 2: first listed wire = most significant bit, i.e. the LSB-first
        # matrix over the reversed list; k >= 3: LSB-first as it is
        wires = list(reversed(b.wires)) if k <= 2 else list(b.wires)
        mat = b.mat
        return FusedGateOp(qubits=[wire_obj[w] for w in wires], fused_matrix=mat, original_ops=list(b.ops))


def fuse(circuit: CircuitIR, max_fused_qubits: int = 2) -> CircuitIR:
    return GateFusionPass(max_fused_qubits).run(circuit)

"""Circuit IR with the reference's shape (invariantq/ir/qir.py:14-355): wires,
gate / measure / reset / barrier / noise / fused ops and ``CircuitIR``.

The simulators in this package accept these objects and, by duck typing on the
class name and fields, the reference's own ``CircuitIR`` objects.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional

import numpy as np

from .gates import gate_matrix

CLIFFORD_GATES = {"h", "s", "sdg", "x", "y", "z", "cx", "cz", "cy", "swap", "cnot", "i", "id"}


@dataclass(frozen=True)
class QWire:
    name: str
    index: int

    def __repr__(self):
        return f"{self.name}[{self.index}]"


@dataclass(frozen=True)
class CWire:
    name: str
    index: int

    def __repr__(self):
        return f"{self.name}[{self.index}]"


@dataclass
class IROp:
    id: int = 0
    qubits: List[QWire] = field(default_factory=list)
    clbits: List[CWire] = field(default_factory=list)
    metadata: Dict[str, Any] = field(default_factory=dict)

    def is_clifford(self) -> bool:
        return False


@dataclass
class GateOp(IROp):
    name: str = "h"
    params: List[float] = field(default_factory=list)
    matrix: Optional[np.ndarray] = None

    def __post_init__(self):
        self.name = self.name.lower()
        if self.matrix is None:
            self.matrix = gate_matrix(self.name, self.params, nqubits=len(self.qubits))

    def is_clifford(self) -> bool:
        return self.name in CLIFFORD_GATES


@dataclass
class MeasureOp(IROp):
    qubit: QWire = field(default_factory=lambda: QWire("q", 0))
    clbit: CWire = field(default_factory=lambda: CWire("c", 0))

    def __post_init__(self):
        self.qubits = [self.qubit]
        self.clbits = [self.clbit]


@dataclass
class ResetOp(IROp):
    qubit: QWire = field(default_factory=lambda: QWire("q", 0))

    def __post_init__(self):
        self.qubits = [self.qubit]


@dataclass
class BarrierOp(IROp):
    pass


@dataclass
class NoiseOp(IROp):
    channel_name: str = "depolarizing"
    params: List[float] = field(default_factory=list)


@dataclass
class FusedGateOp(IROp):
    """A fused unitary block.  ``fused_matrix`` uses the C ABI convention of the
    block's width: k = 2 -> first listed wire is the MSB; k >= 3 -> local index
    bit b is ``qubits[b]`` (core/src/statevector.cpp:133-139)."""
    fused_matrix: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.complex128))
    original_ops: List[GateOp] = field(default_factory=list)


class CircuitIR:
    def __init__(self, name: str = "circuit"):
        self.name = name
        self.qubit_regs: Dict[str, int] = {}
        self.clbit_regs: Dict[str, int] = {}
        self.ops: List[IROp] = []
        self._next_op_id = 0

    def add_qubit_register(self, name: str, size: int):
        self.qubit_regs[name] = size

    def add_clbit_register(self, name: str, size: int):
        self.clbit_regs[name] = size

    @property
    def num_qubits(self) -> int:
        return sum(self.qubit_regs.values())

    @property
    def num_clbits(self) -> int:
        return sum(self.clbit_regs.values())

    def get_qubit_index(self, wire) -> int:
        off = 0
        for reg, size in self.qubit_regs.items():
            if reg == wire.name:
                return off + wire.index
            off += size
        raise KeyError(f"Qubit wire {wire} not found in registers")

    def add_op(self, op: IROp):
        op.id = self._next_op_id
        self._next_op_id += 1
        self.ops.append(op)

    def count_ops(self) -> Dict[str, int]:
        counts: Dict[str, int] = {}
        for op in self.ops:
            key = {"GateOp": getattr(op, "name", "gate"), "MeasureOp": "measure", "FusedGateOp": "fused",
                   "ResetOp": "reset", "BarrierOp": "barrier"}.get(type(op).__name__)
            if type(op).__name__ == "NoiseOp":
                key = f"noise_{op.channel_name}"
            if key:
                counts[key] = counts.get(key, 0) + 1
        return counts


def op_kind(op) -> str:
    """Class name of an op, so reference IR objects dispatch like ours."""
    return type(op).__name__

"""``QCircuit``: the circuit container of ``include/qclab/QCircuit.hpp:22-399``.

``apply`` keeps the reference semantics exactly: gates run in order for
``Op.NoTrans`` and in reverse for ``Op.Trans``/``Op.ConjTrans``, each gate
gets the op, and nested circuits add their ``offset`` to the qubits
(``QCircuit.hpp:130-143``).  The whole (nested) circuit is flattened into
one gate-record list and handed to the CUDA library in a single call.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .gates import PARAMETRIC_KINDS, QObject
from .state import StateVector, apply_records, to_records
from .util import Op, Side, as_op


class QCircuit(QObject):
    def __init__(self, nbQubits: int, offset: int = 0):
        if nbQubits <= 0:
            raise ValueError("nbQubits must be > 0")
        if offset < 0:
            raise ValueError("offset must be >= 0")
        self._n = int(nbQubits)
        self._offset = int(offset)
        self._gates: list[QObject] = []
        self._fixed = False

    # -- QObject interface ---------------------------------------------------
    def nbQubits(self) -> int:
        return self._n

    def fixed(self) -> bool:
        return self._fixed

    def qubit(self) -> int:
        return self._offset

    def qubits(self) -> list[int]:
        return list(range(self._offset, self._offset + self._n))

    def offset(self) -> int:
        return self._offset

    def setOffset(self, offset: int) -> None:
        self._offset = int(offset)

    # -- container -------------------------------------------------------------
    def canInsert(self, gate: QObject) -> bool:
        """All of the gate's qubits lie in [0, nbQubits) (QCircuit.hpp:383-389)."""
        return max(gate.qubits()) < self._n

    def push_back(self, gate: QObject) -> None:
        if not self.canInsert(gate):
            raise ValueError(f"gate {gate!r} does not fit in a {self._n}-qubit circuit")
        self._gates.append(gate)

    def insert(self, pos: int, gate: QObject) -> None:
        if not self.canInsert(gate):
            raise ValueError(f"gate {gate!r} does not fit in a {self._n}-qubit circuit")
        self._gates.insert(pos, gate)

    def erase(self, pos: int) -> None:
        del self._gates[pos]

    def pop_back(self) -> None:
        self._gates.pop()

    def clear(self) -> None:
        self._gates.clear()

    def nbGates(self) -> int:
        return len(self._gates)

    def empty(self) -> bool:
        return not self._gates

    def __len__(self) -> int:
        return len(self._gates)

    def __getitem__(self, i):
        return self._gates[i]

    def __iter__(self):
        return iter(self._gates)

    # -- lowering --------------------------------------------------------------
    def records(self, dtype=np.complex128, offset: int = 0) -> list[tuple]:
        """Flat records of all gates in circuit order, qubits shifted by the
        circuit offset plus ``offset``."""
        out: list[tuple] = []
        for g in self._gates:
            out.extend(g.records(dtype, self._offset + offset))
        return out

    def gate_records(self, dtype=np.complex128, offset: int = 0,
                     number_params: bool = False) -> np.ndarray:
        """GATE_DTYPE array; with ``number_params`` every variable gate gets a
        parameter index in circuit order (the order of ``parameters()``)."""
        recs = to_records(self.records(dtype, offset))
        if number_params:
            k = 0
            for i, g in enumerate(self._flat_gates()):
                if recs[i]["kind"] in PARAMETRIC_KINDS and not g.fixed():
                    recs[i]["param"] = k
                    k += 1
        return recs

    def _flat_gates(self):
        for g in self._gates:
            if isinstance(g, QCircuit):
                yield from g._flat_gates()
            else:
                yield g

    def nbParameters(self) -> int:
        return sum(1 for g in self._flat_gates()
                   if getattr(g, "KIND", None) in PARAMETRIC_KINDS and not g.fixed())

    # -- simulation ------------------------------------------------------------
    def apply(self, op, nbQubits: int, vector, offset: int = 0, fused: bool = False, *rest):
        """QCircuit::apply(op, nbQubits, vector, offset) (QCircuit.hpp:130-143):
        every gate gets offset_ + offset (``records`` adds offset_).

        With a Side first -- apply(side, op, nbQubits, matrix, offset) -- the
        unitary update of QCircuit.hpp:176-204 on a host 2^n x 2^n array (in
        place) or a device matrix object (see ``unitary``)."""
        if isinstance(op, Side) or (isinstance(op, str) and op in ("L", "R")):
            return self._apply_side(op, nbQubits, vector, offset, fused, *rest)
        dtype = vector.numpy_dtype if isinstance(vector, StateVector) else vector.dtype
        recs = self.records(dtype)
        apply_records(recs, as_op(op), nbQubits, vector, offset, fused)
        return vector

    def matrix(self, dtype=np.complex128, fused: bool = False) -> np.ndarray:
        """QCircuit::matrix() (QCircuit.hpp:120-126): the circuit's 2^n x 2^n
        unitary, built on the GPU (eye, then every gate on the right)."""
        from . import unitary as U
        return U.circuit_matrix(self, dtype, fused)

    def simulate(self, vector, fused: bool = False):
        """QCircuit::simulate(vector) (QCircuit.hpp:164-166): in place."""
        return self.apply(Op.NoTrans, self._n, vector, 0, fused)

    def simulate_device(self, state: StateVector, fused: bool = False):
        """QCircuit::simulate_device(T*) (QCircuit.hpp:170-172) on a device state."""
        if not isinstance(state, StateVector):
            raise TypeError("simulate_device needs a StateVector (device memory)")
        return self.apply(Op.NoTrans, self._n, state, 0, fused)

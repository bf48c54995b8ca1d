"""Host front end (QCLAB++ mirror): records, ops, offsets, nesting."""
import numpy as np
import pytest

import oracle
from qclab_b200 import (CNOT, CPhase, Hadamard, Op, QCircuit, RotationY, RotationZ, SWAP,
                        PointerGate1, PauliX)
from qclab_b200 import _lib as L


def test_nested_circuit_offsets_flatten():
    sub = QCircuit(2, offset=1)
    sub.push_back(Hadamard(0))
    sub.push_back(CNOT(0, 1))
    top = QCircuit(4)
    top.push_back(RotationY(0, 0.4))
    top.push_back(sub)
    top.push_back(PointerGate1(PauliX(0), 3))
    recs = top.gate_records(np.complex128)
    assert [int(r["kind"]) for r in recs] == [L.ROTATION_Y, L.HADAMARD, L.CX, L.PAULI_X]
    assert [int(r["qubit0"]) for r in recs] == [0, 1, 1, 3]
    assert int(recs[2]["qubit1"]) == 2


def test_push_back_rejects_out_of_range():
    c = QCircuit(2)
    with pytest.raises(ValueError):
        c.push_back(CNOT(1, 2))


def test_parameter_numbering():
    c = QCircuit(3)
    c.push_back(RotationY(0, 0.1))
    c.push_back(Hadamard(1))
    c.push_back(RotationZ(1, 0.2, fixed=True))
    c.push_back(CPhase(0, 2, 0.3))
    recs = c.gate_records(np.complex128, number_params=True)
    assert [int(r["param"]) for r in recs] == [0, -1, -1, 1]
    assert c.nbParameters() == 2


def test_float_angles_are_rounded_like_qrotation_float():
    g = RotationY(0, 0.7)
    c, s = g._params(np.complex64)
    h = np.float32(np.float32(0.7) / np.float32(2))
    assert c == float(np.float32(np.cos(np.float64(h))))
    assert s == float(np.float32(np.sin(np.float64(h))))


def test_op_conversion():
    from qclab_b200.util import as_op
    assert as_op("C") is Op.ConjTrans
    with pytest.raises(ValueError):
        as_op("X")

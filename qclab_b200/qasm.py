"""OpenQASM front end (``qsv_parse_qasm``), the reader of QCLAB++'s
``QCircuit(filename)`` constructor (``include/qclab/QCircuit.hpp:82-93``).

    n, records = parse(text, np.complex128)
    circuit = read("circuit.qasm")      # QCircuit of gate objects
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _lib as L
from . import gates as G
from .circuit import QCircuit


def parse(text: str, dtype=np.complex128):
    """(nbQubits, GATE_DTYPE records) of OpenQASM text; raises QsvError like
    the reference's reader fails (the records read so far are in the error's
    ``partial`` attribute)."""
    lib = L.load()
    dt = L.DTYPE_OF_NUMPY[np.dtype(dtype)]
    raw = text.encode()
    count, nq = C.c_size_t(), C.c_int()
    st = lib.qsv_parse_qasm(raw, dt, None, 0, C.byref(count), C.byref(nq))
    recs = np.zeros(count.value, dtype=L.GATE_DTYPE)
    st = lib.qsv_parse_qasm(raw, dt, C.c_void_p(recs.ctypes.data) if len(recs) else None,
                            len(recs), C.byref(count), C.byref(nq))
    if st != 0:
        msg = lib.qsv_last_error().decode()
        err = L.QsvError(st, "qsv_parse_qasm", msg)
        err.partial = (nq.value, recs[:count.value])
        raise err
    return nq.value, recs


_CONST1 = {L.HADAMARD: G.Hadamard, L.PAULI_X: G.PauliX, L.PAULI_Y: G.PauliY,
           L.PAULI_Z: G.PauliZ}
_ANGLE1 = {L.ROTATION_X: G.RotationX, L.ROTATION_Y: G.RotationY, L.ROTATION_Z: G.RotationZ,
           L.PHASE: G.Phase}
_CONST2 = {L.CX: G.CX, L.CY: G.CY, L.CZ: G.CZ, L.SWAP: G.SWAP}


def to_circuit(nq: int, recs) -> QCircuit:
    c = QCircuit(nq)
    for r in recs:
        k = int(r["kind"])
        if k in _CONST1:
            c.push_back(_CONST1[k](int(r["qubit0"])))
        elif k in _ANGLE1:
            c.push_back(_ANGLE1[k](int(r["qubit0"]), float(r["cos"]), float(r["sin"])))
        elif k in _CONST2:
            c.push_back(_CONST2[k](int(r["qubit0"]), int(r["qubit1"])))
        else:
            raise ValueError(f"unexpected gate kind {k} from the QASM reader")
    return c


def read(source, dtype=np.complex128) -> QCircuit:
    """QCircuit from a QASM file path or QASM text."""
    p = Path(source) if not isinstance(source, str) or "\n" not in source else None
    text = p.read_text() if p is not None and p.exists() else str(source)
    return to_circuit(*parse(text, dtype))

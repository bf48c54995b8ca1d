"""Unitaries on the GPU: ``QCircuit::matrix()``, ``apply(Side, Op,
nbQubits, SquareMatrix&, offset)`` and ``nrmF`` of ``include/qclab/QCircuit.hpp``.

A 2^n x 2^n matrix lives on the device as a :class:`StateVector` of 2n
qubits holding its entries column-major (entry (r, c) at r + c 2^n), so the
state-vector kernels build and update it (``qsv_apply_matrix``)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .state import StateVector, to_records
from .util import Op, Side, as_op


def as_side(side) -> Side:
    if isinstance(side, Side):
        return side
    if isinstance(side, str) and side in ("L", "R"):
        return Side(side)
    raise ValueError(f"side must be Side.Left/Right or 'L'/'R', got {side!r}")


def identity(nbQubits: int, dtype=np.complex128) -> StateVector:
    """The 2^n x 2^n identity on the device (``qclab::dense::eye``)."""
    m = StateVector(2 * nbQubits, dtype)
    L.check(L.load().qsv_set_identity(m.handle), "qsv_set_identity")
    return m


def upload(matrix: np.ndarray) -> StateVector:
    """A host 2^n x 2^n matrix as a device matrix object."""
    a = np.asarray(matrix)
    N = a.shape[0]
    if a.ndim != 2 or a.shape[1] != N or N & (N - 1):
        raise ValueError("a square matrix of power-of-two size is needed")
    n = N.bit_length() - 1
    m = StateVector(2 * n, a.dtype)
    m.upload(np.ascontiguousarray(a.flatten(order="F")))
    return m


def download(m: StateVector) -> np.ndarray:
    N = 1 << (m.nbQubits // 2)
    return m.download().reshape(N, N, order="F")


def apply_side(m: StateVector, records, side, op, offset: int = 0, fused: bool = False) -> StateVector:
    """``apply(side, op, n, matrix, offset)`` of a gate-record list in circuit
    order on the device matrix ``m`` (in place)."""
    recs = to_records(records)
    ptr = C.c_void_p(recs.ctypes.data) if len(recs) else None
    L.check(L.load().qsv_apply_matrix(m.handle, ptr, len(recs), as_side(side).value.encode(),
                                      as_op(op).value.encode(), int(offset), 1 if fused else 0),
            "qsv_apply_matrix")
    return m


def circuit_matrix_device(circuit, dtype=np.complex128, fused: bool = False) -> StateVector:
    """``QCircuit::matrix()``: eye, then every gate applied on the right."""
    m = identity(circuit.nbQubits(), dtype)
    apply_side(m, circuit.records(dtype), Side.Right, Op.NoTrans, 0, fused)
    return m


def circuit_matrix(circuit, dtype=np.complex128, fused: bool = False) -> np.ndarray:
    with circuit_matrix_device(circuit, dtype, fused) as m:
        return download(m)


def nrmF_device(a: StateVector, b: StateVector) -> float:
    out = C.c_double()
    L.check(L.load().qsv_nrmF(a.handle, b.handle, C.byref(out)), "qsv_nrmF")
    return out.value


def nrmF(circuit1, circuit2, dtype=np.complex128, fused: bool = False) -> float:
    """``qclab::nrmF(circuit1, circuit2)``: Frobenius distance of the two
    circuits' unitaries, built and reduced on the GPU (FP64 reduction)."""
    if circuit1.nbQubits() != circuit2.nbQubits():
        raise ValueError("circuits differ in qubit count")
    with circuit_matrix_device(circuit1, dtype, fused) as a, \
            circuit_matrix_device(circuit2, dtype, fused) as b:
        return nrmF_device(a, b)

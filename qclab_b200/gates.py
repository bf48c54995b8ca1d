"""Gate classes mirroring QCLAB++'s ``qclab::qgates`` on the state-vector path.

Names, constructor arguments and conventions follow the reference:

* qubit q is bit ``n-1-q`` of the amplitude index (qubit 0 = MSB),
  ``src/qgates/apply.hpp:227-238``;
* rotation gates store cos/sin of theta/2 (``include/qclab/QRotation.hpp:44-66``),
  Phase/CPhase store cos/sin of theta (``include/qclab/QAngle.hpp:30-48``);
* rotation and phase gates are variable (trainable) unless ``fixed=True``
  (``include/qclab/qgates/QRotationGate1.hpp:54-59``);
* controlled gates take ``(control, target, ..., controlState=1)``
  (``include/qclab/qgates/QControlledGate2.hpp:30-37``);
* ``qubits()`` is sorted ascending for 2-qubit gates.

Each gate lowers to one ``qsv_gate`` record (``record(dtype)``); amplitudes
are only ever touched by the CUDA library.  ``U2``, ``U3``, ``MatrixGate1``
and ``MatrixGate2`` have no counterpart in QCLAB++.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib as L
from .util import Op, Side, as_op


def _real_of(dtype) -> type:
    dt = np.dtype(dtype)
    return np.float32 if dt in (np.dtype(np.complex64), np.dtype(np.float32)) else np.float64


def _half_angle(theta: float, dtype) -> tuple[float, float]:
    """cos/sin of theta/2 in the state's real precision (QRotation<R>(theta))."""
    R = _real_of(dtype)
    h = R(R(theta) / R(2))
    return float(R(math.cos(float(h)))), float(R(math.sin(float(h))))


def _full_angle(theta: float, dtype) -> tuple[float, float]:
    """cos/sin of theta in the state's real precision (QAngle<R>(theta))."""
    R = _real_of(dtype)
    t = R(theta)
    return float(R(math.cos(float(t)))), float(R(math.sin(float(t))))


class QObject:
    """Base class of all quantum objects (``include/qclab/QObject.hpp:19-89``)."""

    def nbQubits(self) -> int:
        raise NotImplementedError

    def fixed(self) -> bool:
        return True

    def controlled(self) -> bool:
        return False

    def qubits(self) -> list[int]:
        raise NotImplementedError

    def qubit(self) -> int:
        return self.qubits()[0]

    def matrix(self) -> np.ndarray:
        raise NotImplementedError

    def records(self, dtype, offset: int = 0) -> list[tuple]:
        """Flat gate records of this object (with a qubit offset)."""
        raise NotImplementedError

    def apply(self, op, nbQubits: int, vector, offset: int = 0, fused: bool = False, *rest):
        """Applies this object to ``vector`` in place, like
        ``QObject<T>::apply(op, nbQubits, vector, offset)`` (QObject.hpp:52-53).
        ``vector`` is a host numpy array (copied to the GPU and back) or a
        device-resident :class:`StateVector`.

        ``apply(side, op, nbQubits, matrix, offset=0, fused=False)`` (a Side
        first, positional) is the unitary update ``QObject<T>::apply(Side,
        Op, nbQubits, SquareMatrix<T>&, offset)``: side Right gives
        matrix <- op(G) matrix, Left matrix <- matrix op(G)."""
        if isinstance(op, Side) or (isinstance(op, str) and op in ("L", "R")):
            return self._apply_side(op, nbQubits, vector, offset, fused, *rest)
        from .state import apply_records
        op = as_op(op)
        dtype = vector.dtype if not hasattr(vector, "numpy_dtype") else vector.numpy_dtype
        recs = self.records(dtype, 0)
        apply_records(recs, op, nbQubits, vector, offset, fused)
        return vector

    def _apply_side(self, side, op, nbQubits: int, matrix, offset=0, fused=False):
        """The Side form of ``apply`` on a host 2^n x 2^n numpy array (in
        place) or a device matrix object of 2n qubits."""
        from . import unitary as U
        from .state import StateVector
        offset = int(offset)
        if isinstance(matrix, StateVector):
            if matrix.nbQubits != 2 * nbQubits:
                raise ValueError("matrix object does not hold a 2^nbQubits square matrix")
            U.apply_side(matrix, self.records(matrix.numpy_dtype), side, op, offset, bool(fused))
            return matrix
        N = 1 << nbQubits
        if not isinstance(matrix, np.ndarray) or matrix.shape != (N, N):
            raise ValueError("matrix must be a 2^nbQubits x 2^nbQubits numpy array")
        with U.upload(matrix) as m:
            U.apply_side(m, self.records(matrix.dtype), side, op, offset, bool(fused))
            matrix[...] = U.download(m)
        return matrix

    def __repr__(self) -> str:
        return f"{type(self).__name__}({self.qubits()})"


def _rec(kind: int, q0: int, q1: int = -1, cs: int = 1, cos: float = 0.0, sin: float = 0.0,
         matrix=None, param: int = -1) -> tuple:
    m = np.zeros(32)
    if matrix is not None:
        a = np.asarray(matrix, dtype=np.complex128)
        flat = a.flatten(order="F")  # column-major like qclab::dense::SquareMatrix
        m[0:2 * len(flat):2] = flat.real
        m[1:2 * len(flat):2] = flat.imag
    return (kind, q0, q1, cs, cos, sin, m, param, 0)


# ---------------------------------------------------------------------------
# 1-qubit gates
# ---------------------------------------------------------------------------
class QGate1(QObject):
    """1-qubit gate base (``include/qclab/qgates/QGate1.hpp:20``)."""
    KIND = L.MATRIX1

    def __init__(self, qubit: int = 0):
        if qubit < 0:
            raise ValueError("qubit must be >= 0")
        self._qubit = int(qubit)

    def nbQubits(self) -> int:
        return 1

    def qubits(self) -> list[int]:
        return [self._qubit]

    def setQubit(self, qubit: int) -> None:
        if qubit < 0:
            raise ValueError("qubit must be >= 0")
        self._qubit = int(qubit)

    def _params(self, dtype) -> tuple[float, float]:
        return 0.0, 0.0

    def record(self, dtype, offset: int = 0, param: int = -1) -> tuple:
        c, s = self._params(dtype)
        mat = self.matrix() if self.KIND == L.MATRIX1 else None
        return _rec(self.KIND, self._qubit + offset, -1, 1, c, s, mat, param)

    def records(self, dtype, offset: int = 0) -> list[tuple]:
        return [self.record(dtype, offset)]


class Identity(QGate1):
    KIND = L.IDENTITY

    def matrix(self):
        return np.eye(2, dtype=complex)


class Hadamard(QGate1):
    KIND = L.HADAMARD

    def matrix(self):
        s = 1 / math.sqrt(2)
        return np.array([[s, s], [s, -s]], dtype=complex)


class PauliX(QGate1):
    KIND = L.PAULI_X

    def matrix(self):
        return np.array([[0, 1], [1, 0]], dtype=complex)


class PauliY(QGate1):
    KIND = L.PAULI_Y

    def matrix(self):
        return np.array([[0, -1j], [1j, 0]], dtype=complex)


class PauliZ(QGate1):
    KIND = L.PAULI_Z

    def matrix(self):
        return np.array([[1, 0], [0, -1]], dtype=complex)


class Phase45(QGate1):
    """T gate (``include/qclab/qgates/Phase45.hpp``)."""
    KIND = L.PHASE45

    def matrix(self):
        s = 1 / math.sqrt(2)
        return np.array([[1, 0], [0, s + 1j * s]], dtype=complex)


class Phase90(QGate1):
    """S gate (``include/qclab/qgates/Phase90.hpp``)."""
    KIND = L.PHASE90

    def matrix(self):
        return np.array([[1, 0], [0, 1j]], dtype=complex)


class _Angle:
    """Mixin for gates parameterised by one angle.  ``half=True`` stores
    theta/2 (QRotation), ``half=False`` stores theta (QAngle)."""
    HALF = True

    def _init_angle(self, args, fixed: bool):
        self._fixed = bool(fixed)
        if len(args) == 0:
            self._theta, self._cossin = 0.0, None
        elif len(args) == 1:
            self._theta, self._cossin = float(args[0]), None
        elif len(args) == 2:
            c, s = float(args[0]), float(args[1])
            self._cossin = (c, s)
            self._theta = (2.0 if self.HALF else 1.0) * math.atan2(s, c)
        else:
            raise TypeError("expected (theta) or (cos, sin)")

    def theta(self) -> float:
        return self._theta

    def cos(self) -> float:
        return self._cossin[0] if self._cossin else math.cos(self._theta / 2 if self.HALF else self._theta)

    def sin(self) -> float:
        return self._cossin[1] if self._cossin else math.sin(self._theta / 2 if self.HALF else self._theta)

    def update(self, *args) -> None:
        self._init_angle(args, self._fixed)

    def fixed(self) -> bool:
        return self._fixed

    def makeFixed(self) -> None:
        self._fixed = True

    def makeVariable(self) -> None:
        self._fixed = False

    def _params(self, dtype):
        if self._cossin is not None:
            R = _real_of(dtype)
            return float(R(self._cossin[0])), float(R(self._cossin[1]))
        return (_half_angle if self.HALF else _full_angle)(self._theta, dtype)


class RotationX(_Angle, QGate1):
    """exp(-i theta/2 X) (``include/qclab/qgates/RotationX.hpp``)."""
    KIND = L.ROTATION_X

    def __init__(self, qubit: int = 0, *args, fixed: bool = False):
        QGate1.__init__(self, qubit)
        self._init_angle(args, fixed)

    def matrix(self):
        c, s = self.cos(), self.sin()
        return np.array([[c, -1j * s], [-1j * s, c]], dtype=complex)


class RotationY(_Angle, QGate1):
    KIND = L.ROTATION_Y

    def __init__(self, qubit: int = 0, *args, fixed: bool = False):
        QGate1.__init__(self, qubit)
        self._init_angle(args, fixed)

    def matrix(self):
        c, s = self.cos(), self.sin()
        return np.array([[c, -s], [s, c]], dtype=complex)


class RotationZ(_Angle, QGate1):
    KIND = L.ROTATION_Z

    def __init__(self, qubit: int = 0, *args, fixed: bool = False):
        QGate1.__init__(self, qubit)
        self._init_angle(args, fixed)

    def matrix(self):
        c, s = self.cos(), self.sin()
        return np.array([[c - 1j * s, 0], [0, c + 1j * s]], dtype=complex)


class Phase(_Angle, QGate1):
    """diag(1, e^{i theta}) (``include/qclab/qgates/Phase.hpp``)."""
    KIND = L.PHASE
    HALF = False

    def __init__(self, qubit: int = 0, *args, fixed: bool = False):
        QGate1.__init__(self, qubit)
        self._init_angle(args, fixed)

    def matrix(self):
        return np.array([[1, 0], [0, self.cos() + 1j * self.sin()]], dtype=complex)


class MatrixGate1(QGate1):
    """Arbitrary 2x2 unitary (QGate1 with a user matrix; PointerGate1 target)."""
    KIND = L.MATRIX1

    def __init__(self, qubit: int, matrix):
        super().__init__(qubit)
        m = np.asarray(matrix, dtype=complex)
        if m.shape != (2, 2):
            raise ValueError("MatrixGate1 needs a 2x2 matrix")
        self._m = m

    def matrix(self):
        return self._m.copy()


class U3(MatrixGate1):
    """U3(theta, phi, lambda) = [[c, -e^{il} s], [e^{ip} s, e^{i(p+l)} c]],
    c = cos(theta/2), s = sin(theta/2).  Not in QCLAB++."""

    def __init__(self, qubit: int, theta: float, phi: float, lam: float):
        c, s = math.cos(theta / 2), math.sin(theta / 2)
        m = np.array([[c, -np.exp(1j * lam) * s],
                      [np.exp(1j * phi) * s, np.exp(1j * (phi + lam)) * c]], dtype=complex)
        super().__init__(qubit, m)
        self.params = (theta, phi, lam)


class U2(U3):
    """U2(phi, lambda) = U3(pi/2, phi, lambda).  Not in QCLAB++."""

    def __init__(self, qubit: int, phi: float, lam: float):
        super().__init__(qubit, math.pi / 2, phi, lam)


class PointerGate1(QGate1):
    """Forwards to another 1-qubit gate with a qubit offset
    (``include/qclab/qgates/PointerGate1.hpp:16``)."""

    def __init__(self, gate: QGate1, offset: int = 0):
        self._gate = gate
        self._offset = int(offset)

    def qubits(self):
        return [self._gate.qubit() + self._offset]

    def fixed(self):
        return self._gate.fixed()

    def matrix(self):
        return self._gate.matrix()

    def records(self, dtype, offset: int = 0):
        return self._gate.records(dtype, offset + self._offset)

    def record(self, dtype, offset: int = 0, param: int = -1):
        return self._gate.record(dtype, offset + self._offset, param)


# ---------------------------------------------------------------------------
# 2-qubit gates
# ---------------------------------------------------------------------------
class QGate2(QObject):
    """2-qubit gate base (``include/qclab/qgates/QGate2.hpp:17``)."""
    KIND = L.MATRIX2

    def __init__(self, qubit0: int = 0, qubit1: int = 1):
        if qubit0 < 0 or qubit1 < 0 or qubit0 == qubit1:
            raise ValueError("qubits must be distinct and >= 0")
        self._q = (min(qubit0, qubit1), max(qubit0, qubit1))

    def nbQubits(self) -> int:
        return 2

    def qubits(self):
        return list(self._q)

    def setQubits(self, qubits) -> None:
        a, b = qubits
        if a < 0 or b < 0 or a == b:
            raise ValueError("qubits must be distinct and >= 0")
        self._q = (min(a, b), max(a, b))

    def _params(self, dtype):
        return 0.0, 0.0

    def record(self, dtype, offset: int = 0, param: int = -1):
        c, s = self._params(dtype)
        return _rec(self.KIND, self._q[0] + offset, self._q[1] + offset, 1, c, s, None, param)

    def records(self, dtype, offset: int = 0):
        return [self.record(dtype, offset)]


class SWAP(QGate2):
    KIND = L.SWAP

    def matrix(self):
        return np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=complex)


class iSWAP(QGate2):
    KIND = L.ISWAP

    def matrix(self):
        return np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]], dtype=complex)


class _Rot2(_Angle, QGate2):
    def __init__(self, qubit0: int = 0, qubit1: int = 1, *args, fixed: bool = False):
        QGate2.__init__(self, qubit0, qubit1)
        self._init_angle(args, fixed)


class RotationXX(_Rot2):
    """exp(-i theta/2 X⊗X) (``include/qclab/qgates/RotationXX.hpp:136-143``)."""
    KIND = L.ROTATION_XX

    def matrix(self):
        d, o = self.cos(), -1j * self.sin()
        return np.array([[d, 0, 0, o], [0, d, o, 0], [0, o, d, 0], [o, 0, 0, d]], dtype=complex)


class RotationYY(_Rot2):
    KIND = L.ROTATION_YY

    def matrix(self):
        d, o = self.cos(), 1j * self.sin()
        return np.array([[d, 0, 0, o], [0, d, -o, 0], [0, -o, d, 0], [o, 0, 0, d]], dtype=complex)


class RotationZZ(_Rot2):
    KIND = L.ROTATION_ZZ

    def matrix(self):
        a, b = self.cos() - 1j * self.sin(), self.cos() + 1j * self.sin()
        return np.diag([a, b, b, a]).astype(complex)


class MatrixGate2(QObject):
    """Arbitrary 4x4 unitary on (qubit0, qubit1), in the kron basis
    |qubit0 qubit1> (qubit0 the leading factor).  Not in QCLAB++."""

    def __init__(self, qubit0: int, qubit1: int, matrix):
        if qubit0 < 0 or qubit1 < 0 or qubit0 == qubit1:
            raise ValueError("qubits must be distinct and >= 0")
        m = np.asarray(matrix, dtype=complex)
        if m.shape != (4, 4):
            raise ValueError("MatrixGate2 needs a 4x4 matrix")
        self._q = (int(qubit0), int(qubit1))
        self._m = m

    def nbQubits(self):
        return 2

    def qubits(self):
        return sorted(self._q)

    def matrix(self):
        return self._m.copy()

    def record(self, dtype, offset: int = 0, param: int = -1):
        return _rec(L.MATRIX2, self._q[0] + offset, self._q[1] + offset, 1, 0, 0, self._m, param)

    def records(self, dtype, offset: int = 0):
        return [self.record(dtype, offset)]


class PointerGate2(QObject):
    """Forwards to another 2-qubit gate with a qubit offset
    (``include/qclab/qgates/PointerGate2.hpp:62-72``)."""

    def __init__(self, gate, offset: int = 0):
        self._gate = gate
        self._offset = int(offset)

    def nbQubits(self):
        return 2

    def qubits(self):
        return [q + self._offset for q in self._gate.qubits()]

    def fixed(self):
        return self._gate.fixed()

    def matrix(self):
        return self._gate.matrix()

    def record(self, dtype, offset: int = 0, param: int = -1):
        return self._gate.record(dtype, offset + self._offset, param)

    def records(self, dtype, offset: int = 0):
        return self._gate.records(dtype, offset + self._offset)


class QControlledGate2(QObject):
    """Controlled 1-qubit gate (``include/qclab/qgates/QControlledGate2.hpp:18``)."""
    KIND = L.CONTROLLED1

    def __init__(self, control: int, target: int, controlState: int = 1):
        if control < 0 or target < 0 or control == target:
            raise ValueError("control and target must be distinct and >= 0")
        if controlState not in (0, 1):
            raise ValueError("controlState must be 0 or 1")
        self._control, self._target, self._cs = int(control), int(target), int(controlState)

    def nbQubits(self):
        return 2

    def controlled(self):
        return True

    def control(self):
        return self._control

    def target(self):
        return self._target

    def controlState(self):
        return self._cs

    def qubits(self):
        return [min(self._control, self._target), max(self._control, self._target)]

    def gate_matrix(self) -> np.ndarray:
        raise NotImplementedError

    def _params(self, dtype):
        return 0.0, 0.0

    def matrix(self):
        """4x4 in the sorted-qubit basis (QControlledGate2.hpp:64-89)."""
        E0, E1, I2 = np.diag([1, 0]), np.diag([0, 1]), np.eye(2)
        CG = self.gate_matrix()
        if self._cs == 0:
            return (np.kron(E0, CG) + np.kron(E1, I2)) if self._control < self._target \
                else (np.kron(CG, E0) + np.kron(I2, E1))
        return (np.kron(E0, I2) + np.kron(E1, CG)) if self._control < self._target \
            else (np.kron(I2, E0) + np.kron(CG, E1))

    def record(self, dtype, offset: int = 0, param: int = -1):
        c, s = self._params(dtype)
        mat = self.gate_matrix() if self.KIND == L.CONTROLLED1 else None
        return _rec(self.KIND, self._control + offset, self._target + offset, self._cs, c, s,
                    mat, param)

    def records(self, dtype, offset: int = 0):
        return [self.record(dtype, offset)]


class ControlledGate(QControlledGate2):
    """Controlled version of an arbitrary 1-qubit matrix (QControlledGate2
    with a user-supplied target gate)."""

    def __init__(self, control: int, target: int, matrix, controlState: int = 1):
        super().__init__(control, target, controlState)
        self._g = np.asarray(matrix, dtype=complex)

    def gate_matrix(self):
        return self._g


class CX(QControlledGate2):
    KIND = L.CX

    def gate_matrix(self):
        return PauliX().matrix()


CNOT = CX


class CY(QControlledGate2):
    KIND = L.CY

    def gate_matrix(self):
        return PauliY().matrix()


class CZ(QControlledGate2):
    KIND = L.CZ

    def gate_matrix(self):
        return PauliZ().matrix()


class _CAngle(_Angle, QControlledGate2):
    def __init__(self, control: int, target: int, *args, controlState: int = 1,
                 fixed: bool = False):
        QControlledGate2.__init__(self, control, target, controlState)
        self._init_angle(args, fixed)


class CPhase(_CAngle):
    KIND = L.CPHASE
    HALF = False

    def gate_matrix(self):
        return np.array([[1, 0], [0, self.cos() + 1j * self.sin()]], dtype=complex)


class CRotationX(_CAngle):
    KIND = L.CROTATION_X

    def gate_matrix(self):
        c, s = self.cos(), self.sin()
        return np.array([[c, -1j * s], [-1j * s, c]], dtype=complex)


class CRotationY(_CAngle):
    KIND = L.CROTATION_Y

    def gate_matrix(self):
        c, s = self.cos(), self.sin()
        return np.array([[c, -s], [s, c]], dtype=complex)


class CRotationZ(_CAngle):
    KIND = L.CROTATION_Z

    def gate_matrix(self):
        c, s = self.cos(), self.sin()
        return np.array([[c - 1j * s, 0], [0, c + 1j * s]], dtype=complex)


PARAMETRIC_KINDS = {L.ROTATION_X, L.ROTATION_Y, L.ROTATION_Z, L.PHASE, L.CPHASE,
                    L.CROTATION_X, L.CROTATION_Y, L.CROTATION_Z,
                    L.ROTATION_XX, L.ROTATION_YY, L.ROTATION_ZZ}

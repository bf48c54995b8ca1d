"""Unitaries on the GPU against QCLAB++ itself (oracle/_ref): QCircuit::matrix(),
apply(Side, Op, nbQubits, matrix, offset) for both sides and all ops, and
nrmF.  Tolerances: 1e-12 (complex<double>, double), 2e-5 (complex<float>,
float), relative to the matrix scale."""
import numpy as np
import pytest

import oracle
from qclab_b200 import QCircuit, QsvError, StateVector
from qclab_b200 import unitary as U
from qclab_b200 import workloads as W
from qclab_b200.util import Op, Side

pytestmark = pytest.mark.gpu

TOL = {np.dtype(np.complex128): 1e-12, np.dtype(np.float64): 1e-12,
       np.dtype(np.complex64): 2e-5, np.dtype(np.float32): 2e-5}


def circuit(n, seed, real=False, count=None):
    return W.random_mixed(n, count or 6 * n + 4, seed=seed, real=real, adjacent_generic=True)


@pytest.mark.parametrize("fused", [False, True], ids=["unfused", "fused"])
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64, np.float64],
                         ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("n", [1, 2, 3, 5, 6])
def test_matrix_matches_reference(cuda, n, dtype, fused):
    real = np.dtype(dtype).kind == "f"
    c = circuit(n, seed=100 + n, real=real)
    got = c.matrix(dtype, fused=fused)
    ref = oracle.ref_matrix(n, dtype, c.gate_records(dtype))
    assert got.dtype == np.dtype(dtype) and got.shape == (1 << n, 1 << n)
    assert np.max(np.abs(got - ref)) <= TOL[np.dtype(dtype)]


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("op", ["N", "T", "C"])
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=lambda d: np.dtype(d).name)
def test_apply_side_matches_reference(cuda, side, op, dtype):
    nbq, nc, offset = 5, 3, 1
    rng = np.random.default_rng(7)
    N = 1 << nbq
    M0 = (rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N))).astype(dtype)
    c = circuit(nc, seed=11)
    got = M0.copy()
    c.apply(Side(side), Op(op), nbq, got, offset)
    # QCLAB++'s controlled gates ignore `offset` in apply(Side, ...)
    # (src/qgates/QControlledGate2.cpp:48-59 shift qubits[] but loop over
    # control()/target()), so the reference gets the offset in the records.
    ref = oracle.ref_apply_side(M0, c.gate_records(dtype, offset=offset), side, op, nbq, 0,
                                circuit_qubits=nbq)
    scale = max(1.0, float(np.max(np.abs(ref))))
    assert np.max(np.abs(got - ref)) <= TOL[np.dtype(dtype)] * scale


def test_gate_side_apply_and_device_matrix(cuda):
    from qclab_b200 import CNOT, RotationY
    n = 3
    M = U.identity(n, np.complex128)
    g1, g2 = RotationY(1, 0.3), CNOT(0, 2)
    g1.apply(Side.Right, Op.NoTrans, n, M)
    g2.apply(Side.Left, Op.ConjTrans, n, M)      # M = RY . CNOT^+
    host = U.download(M)
    M.close()
    c1 = QCircuit(n)
    c1.push_back(RotationY(1, 0.3))
    c2 = QCircuit(n)
    c2.push_back(CNOT(0, 2))
    expect = oracle.ref_matrix(n, np.complex128, c1.gate_records()) @ \
        oracle.ref_matrix(n, np.complex128, c2.gate_records()).conj().T
    assert np.max(np.abs(host - expect)) < 1e-14


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64, np.float64],
                         ids=lambda d: np.dtype(d).name)
def test_nrmF_matches_reference(cuda, dtype):
    real = np.dtype(dtype).kind == "f"
    n = 4
    a, b = circuit(n, 1, real), circuit(n, 2, real)
    ra, rb = a.gate_records(dtype), b.gate_records(dtype)
    got = U.nrmF(a, b, dtype)
    ref = oracle.ref_nrmF(n, dtype, ra, rb)
    assert abs(got - ref) <= 1e-6 * ref if np.dtype(dtype) == np.complex64 else abs(got - ref) <= 1e-12 * ref
    assert U.nrmF(a, a, dtype) == 0.0
    # same unitary, different gate order: a circuit and its double inverse
    m = a.matrix(dtype)
    assert abs(oracle.nrmF(m, oracle.ref_matrix(n, dtype, ra))) <= TOL[np.dtype(dtype)] * 4 * (1 << n)


def test_unitary_errors(cuda):
    lib_n = 3
    with StateVector(2 * lib_n + 1, np.complex128) as odd:
        with pytest.raises(QsvError) as e:
            U.apply_side(odd, [], "R", "N")
        assert e.value.status == 3
    with U.identity(2, np.complex128) as m:
        c = QCircuit(3)
        from qclab_b200 import Hadamard
        c.push_back(Hadamard(2))
        with pytest.raises(QsvError) as e:
            U.apply_side(m, c.records(np.complex128), "R", "N")
        assert e.value.status == 2
        with pytest.raises(ValueError):
            U.apply_side(m, [], "X", "N")

"""Adjoint gradients on the GPU against parameter shift, central finite
differences (GPU) and a 4-point finite-difference stencil on the CPU oracle.
Gradient tolerance: 1e-9 (complex<double>)."""
import math

import numpy as np
import pytest

import oracle
from qclab_b200 import (CPhase, CRotationX, CRotationY, CRotationZ, CNOT, CZ, Hadamard, Phase,
                        QCircuit, RotationX, RotationXX, RotationY, RotationYY, RotationZ,
                        RotationZZ, StateVector, SWAP)
from qclab_b200 import workloads as W
from qclab_b200.gradients import (_shifted, adjoint_gradient, finite_difference_gradient,
                                  parameter_shift_gradient)
from qclab_b200.observable import Observable, ising

pytestmark = pytest.mark.gpu


def cpu_energy(n, recs, H, dtype=np.complex128):
    x = np.zeros(1 << n, dtype=dtype)
    x[0] = 1
    oracle.apply(x, recs)
    return oracle.expectation(x, H.matrix_free_terms())


def cpu_gradient(n, recs, H, h=1e-3):
    """4-point stencil on the CPU oracle, per gate (error O(h^4))."""
    nparams = int(recs["param"].max()) + 1
    g = np.zeros(nparams)
    for i in range(len(recs)):
        p = int(recs[i]["param"])
        if p < 0:
            continue
        f = [cpu_energy(n, _shifted(recs, i, d * h), H) for d in (-2, -1, 1, 2)]
        g[p] += (f[0] - 8 * f[1] + 8 * f[2] - f[3]) / (12 * h)
    return g


def all_kinds_circuit(n, seed):
    rng = np.random.default_rng(seed)
    c = QCircuit(n)
    for layer in range(2):
        for q in range(n):
            c.push_back(Hadamard(q))
        ang = lambda: float(rng.uniform(0, 2 * math.pi))
        c.push_back(RotationX(0, ang()))
        c.push_back(RotationY(1, ang()))
        c.push_back(RotationZ(2, ang()))
        c.push_back(Phase(3, ang()))
        c.push_back(RotationXX(0, 2, ang()))
        c.push_back(RotationYY(1, 3, ang()))
        c.push_back(RotationZZ(3, 0, ang()))
        c.push_back(CRotationX(1, 0, ang()))
        c.push_back(CRotationY(2, 3, ang(), controlState=0))
        c.push_back(CRotationZ(3, 1, ang()))
        c.push_back(CPhase(0, 3, ang()))
        c.push_back(CPhase(2, 1, ang(), controlState=0))
        c.push_back(CNOT(1, 2))
        c.push_back(CZ(0, 1))
        c.push_back(SWAP(0, 3))
    return c


def test_adjoint_every_parametric_kind(cuda):
    n = 4
    c = all_kinds_circuit(n, 1)
    recs = c.gate_records(np.complex128, number_params=True)
    H = Observable(n).add(0.7, "ZZII").add(-0.3, "XIYI").add(1.1, "IXXZ").add(0.4, "YYII")
    with StateVector(n, np.complex128) as s:
        e, g = adjoint_gradient(s, recs, H)
        assert abs(e - cpu_energy(n, recs, H)) < 1e-12
        ref = cpu_gradient(n, recs, H)
        assert np.max(np.abs(g - ref)) < 1e-9, np.max(np.abs(g - ref))
        # the state is restored to |0...0>
        y = s.download()
        assert abs(y[0] - 1) < 1e-12 and np.max(np.abs(y[1:])) < 1e-12


def test_shared_parameters_accumulate(cuda):
    n = 3
    c = QCircuit(n)
    c.push_back(Hadamard(0))
    c.push_back(RotationY(0, 0.3))
    c.push_back(CNOT(0, 1))
    c.push_back(RotationY(1, 0.3))
    recs = c.gate_records(np.complex128, number_params=True)
    recs["param"] = [-1, 0, -1, 0]
    H = ising(n)
    with StateVector(n, np.complex128) as s:
        e, g = adjoint_gradient(s, recs, H, nparams=1)
    ref = cpu_gradient(n, recs, H)
    assert abs(g[0] - ref[0]) < 1e-9


@pytest.mark.parametrize("n,layers", [(8, 3), (12, 2)])
def test_hea_adjoint_vs_parameter_shift_and_fd(cuda, n, layers):
    c = W.hea(n, layers, seed=n)
    recs = c.gate_records(np.complex128, number_params=True)
    H = ising(n)
    with StateVector(n, np.complex128) as s:
        e, g = adjoint_gradient(s, recs, H)
        ps = parameter_shift_gradient(s, recs, H)
        fd = finite_difference_gradient(s, recs, H, h=1e-5)
    assert abs(e - cpu_energy(n, recs, H)) < 1e-11
    assert np.max(np.abs(g - ps)) < 1e-9
    assert np.max(np.abs(g - fd)) < 1e-8


def test_hea_adjoint_complex64(cuda):
    n = 10
    c = W.hea(n, 2, seed=4)
    H = ising(n)
    r64 = c.gate_records(np.complex64, number_params=True)
    r128 = c.gate_records(np.complex128, number_params=True)
    with StateVector(n, np.complex64) as s, StateVector(n, np.complex128) as d:
        e32, g32 = adjoint_gradient(s, r64, H)
        e64, g64 = adjoint_gradient(d, r128, H)
    assert abs(e32 - e64) < 1e-4
    assert np.max(np.abs(g32 - g64)) < 1e-4


def test_adjoint_rejects_non_parametric(cuda):
    from qclab_b200 import QsvError
    c = QCircuit(2)
    c.push_back(Hadamard(0))
    recs = c.gate_records(np.complex128)
    recs["param"] = [0]
    with StateVector(2, np.complex128) as s:
        with pytest.raises(QsvError) as e:
            adjoint_gradient(s, recs, ising(2), nparams=1)
        assert e.value.status == 8

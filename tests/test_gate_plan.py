"""The gate-specialised engine's plan on the host (no GPU): gate records are
lowered, planned and factored exactly as the GPU executor does it, applied
by the host mirror of the device ops (tests/cpp/gate_plan_test.cpp) and
compared with the C oracle within 1e-12.  Covers every gate class, every
op, offsets, 4- and 5-bit register passes and tile/low-bit shapes, and the
brick circuit of the benchmark."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from qclab_b200 import workloads as W

ROOT = Path(__file__).resolve().parent.parent
CSRC = ROOT / "qclab_b200" / "csrc"


@pytest.fixture(scope="module")
def binary(tmp_path_factory):
    out = tmp_path_factory.mktemp("gp") / "gate_plan_test"
    r = subprocess.run(["g++", "-O2", "-std=c++17", f"-I{ROOT / 'include'}", f"-I{CSRC}",
                        str(ROOT / "tests" / "cpp" / "gate_plan_test.cpp"), str(CSRC / "plan.cpp"),
                        "-o", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return out


def run_plan(binary, tmp_path, n, recs, x, R, m, low, op="N", offset=0):
    rp, sp, op_ = tmp_path / "r.bin", tmp_path / "s.bin", tmp_path / "o.bin"
    rp.write_bytes(np.ascontiguousarray(recs).tobytes())
    sp.write_bytes(np.ascontiguousarray(x, dtype=np.complex128).tobytes())
    r = subprocess.run([str(binary), str(n), str(R), str(m), str(low), op, str(offset), str(rp),
                        str(sp), str(op_)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    stages, passes, ops = (int(v) for v in r.stdout.split())
    return np.frombuffer(op_.read_bytes(), dtype=np.complex128), stages, passes, ops


def rand_state(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return x / np.linalg.norm(x)


@pytest.mark.parametrize("R,m,low", [(4, 8, 2), (4, 10, 3), (5, 9, 3), (5, 11, 4), (4, 6, 1)])
@pytest.mark.parametrize("op", ["N", "T", "C"])
def test_mixed_circuits_match_oracle(binary, tmp_path, R, m, low, op):
    n = 11
    recs = W.random_mixed(n, 400, seed=R * 100 + m).gate_records(np.complex128)
    x = rand_state(n, m)
    want = oracle.apply(x.copy(), recs, op)
    got, stages, passes, ops = run_plan(binary, tmp_path, n, recs, x, R, m, low, op)
    assert stages >= 1 and passes >= stages
    assert np.max(np.abs(got - want)) < 1e-12


def test_offset_and_small_register(binary, tmp_path):
    n = 9
    recs = W.random_mixed(6, 200, seed=3).gate_records(np.complex128)
    x = rand_state(n, 1)
    want = oracle.apply(x.copy(), recs, "N", 3)
    got, *_ = run_plan(binary, tmp_path, n, recs, x, 4, 7, 2, "N", 3)
    assert np.max(np.abs(got - want)) < 1e-12


@pytest.mark.parametrize("R", [4, 5])
def test_brick_circuit(binary, tmp_path, R):
    n = 14
    recs = W.brick(n, 30, seed=2024).gate_records(np.complex128)
    x = np.zeros(1 << n, dtype=np.complex128)
    x[0] = 1
    want = oracle.apply(x.copy(), recs)
    got, stages, passes, ops = run_plan(binary, tmp_path, n, recs, x, R, 12, 2)
    assert np.max(np.abs(got - want)) < 1e-12
    # every gate is one op, plus one scale op per stage
    assert ops <= len(recs) + stages


@pytest.mark.parametrize("R,m,low", [(3, 8, 2), (4, 9, 3), (4, 11, 2)])
def test_adjoint_gradient_terms(binary, tmp_path, R, m, low):
    """The backward list of qsv_adjoint_gradient on two vectors (gradient
    terms as RDX/RDY/RDZ ops) against parameter shift on the oracle."""
    from qclab_b200 import gates as G
    from qclab_b200.circuit import QCircuit
    from qclab_b200.observable import ising
    n = 10
    rng = np.random.default_rng(R * 10 + m)
    c = QCircuit(n)
    for layer in range(3):
        for q in range(n):
            kind = (G.RotationX, G.RotationY, G.RotationZ)[int(rng.integers(0, 3))]
            c.push_back(kind(q, float(rng.uniform(0, 6.28))))
        for q in range(layer % 2, n - 1, 2):
            c.push_back(G.CNOT(q, q + 1) if rng.random() < 0.5 else G.CZ(q, q + 1))
        c.push_back(G.Hadamard(int(rng.integers(0, n))))
    recs = c.gate_records(np.complex128, number_params=True)
    terms = ising(n).matrix_free_terms()
    psi = np.zeros(1 << n, dtype=np.complex128)
    psi[0] = 1
    oracle.apply(psi, recs)
    lam = oracle.observable_apply(psi, terms)
    rp, pp, lp, op_ = (tmp_path / f for f in ("r.bin", "p.bin", "l.bin", "o.bin"))
    rp.write_bytes(recs.tobytes())
    pp.write_bytes(psi.tobytes())
    lp.write_bytes(lam.tobytes())
    r = subprocess.run([str(binary), "adjoint", str(n), str(R), str(m), str(low), str(rp), str(pp),
                        str(lp), str(op_)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    rows = np.frombuffer(op_.read_bytes(), dtype=np.float64)
    params = [int(recs[k]["param"]) for k in range(len(recs) - 1, -1, -1) if recs[k]["param"] >= 0]
    grad = np.zeros(int(recs["param"].max()) + 1)
    for slot, p in enumerate(params):
        grad[p] += rows[slot]

    def energy(rr):
        x = np.zeros(1 << n, dtype=np.complex128)
        x[0] = 1
        oracle.apply(x, rr)
        return oracle.expectation(x, terms)

    from qclab_b200.gradients import _shifted
    for k in range(len(recs)):
        p = int(recs[k]["param"])
        if p < 0:
            continue
        ps = 0.5 * (energy(_shifted(recs, k, np.pi / 2)) - energy(_shifted(recs, k, -np.pi / 2)))
        assert abs(grad[p] - ps) < 1e-10, (p, grad[p], ps)


@pytest.mark.parametrize("R,m,low", [(3, 8, 2), (4, 10, 3)])
def test_adjoint_gradient_terms_any_generator(binary, tmp_path, R, m, low):
    """Gradient terms of every trainable gate class (two-qubit rotations,
    controlled rotations with either control state, Phase and CPhase) as
    generic RDG ops, against central finite differences on the oracle."""
    from qclab_b200 import gates as G
    from qclab_b200.circuit import QCircuit
    from qclab_b200.gradients import _shifted
    from qclab_b200.observable import ising
    n = 9
    rng = np.random.default_rng(R * 100 + m)
    ang = lambda: float(rng.uniform(0, 6.28))  # noqa: E731
    c = QCircuit(n)
    for layer in range(2):
        for q in range(n):
            c.push_back((G.RotationX, G.RotationY, G.RotationZ)[q % 3](q, ang()))
        c.push_back(G.RotationXX(0, n - 1, ang()))
        c.push_back(G.RotationYY(2, 5, ang()))
        c.push_back(G.RotationZZ(1, 7, ang()))
        c.push_back(G.CRotationX(3, 0, ang(), controlState=layer))
        c.push_back(G.CRotationY(8, 2, ang(), controlState=1 - layer))
        c.push_back(G.CRotationZ(4, 6, ang()))
        c.push_back(G.CPhase(0, 4, ang()))
        c.push_back(G.Phase(6, ang()))
        for q in range(layer % 2, n - 1, 2):
            c.push_back(G.CNOT(q, q + 1))
    recs = c.gate_records(np.complex128, number_params=True)
    terms = ising(n).matrix_free_terms()
    psi = np.zeros(1 << n, dtype=np.complex128)
    psi[0] = 1
    oracle.apply(psi, recs)
    lam = oracle.observable_apply(psi, terms)
    rp, pp, lp, op_ = (tmp_path / f for f in ("r.bin", "p.bin", "l.bin", "o.bin"))
    rp.write_bytes(recs.tobytes())
    pp.write_bytes(psi.tobytes())
    lp.write_bytes(lam.tobytes())
    r = subprocess.run([str(binary), "adjoint", str(n), str(R), str(m), str(low), str(rp), str(pp),
                        str(lp), str(op_)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    rows = np.frombuffer(op_.read_bytes(), dtype=np.float64)
    params = [int(recs[k]["param"]) for k in range(len(recs) - 1, -1, -1) if recs[k]["param"] >= 0]
    grad = np.zeros(int(recs["param"].max()) + 1)
    for slot, p in enumerate(params):
        grad[p] += rows[slot]

    def energy(rr):
        x = np.zeros(1 << n, dtype=np.complex128)
        x[0] = 1
        oracle.apply(x, rr)
        return oracle.expectation(x, terms)

    h = 1e-6
    for k in range(len(recs)):
        p = int(recs[k]["param"])
        if p < 0:
            continue
        fd = (energy(_shifted(recs, k, h)) - energy(_shifted(recs, k, -h))) / (2 * h)
        assert abs(grad[p] - fd) < 1e-7, (p, int(recs[k]["kind"]), grad[p], fd)

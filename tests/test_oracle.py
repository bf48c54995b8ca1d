"""The CPU oracle, pinned to the reference (CPU only)."""
import hashlib
import subprocess

import numpy as np
import pytest

import oracle
from cases import DTYPES, circuit_cases, gate_cases, same_bits
from make_golden import HERE, case_digest
from qclab_b200 import MatrixGate2, QCircuit
from qclab_b200 import workloads as W

GOLD = np.load(HERE / "reference_outputs.npz")


@pytest.mark.skipif(not oracle.REF_TESTS.exists(), reason="reference not built here")
def test_reference_own_test_suite_passes():
    """The reference's gate/circuit unit tests (3800+ EXPECTs, with their
    known-answer vectors) pass on the reference build the fixtures come from."""
    r = subprocess.run([str(oracle.REF_TESTS)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:]
    assert "0 failed;" in r.stdout and ", 0 failed," in r.stdout


@pytest.mark.parametrize("dtype", DTYPES, ids=lambda d: np.dtype(d).name)
def test_oracle_bitexact_on_gate_fixtures(dtype):
    name = np.dtype(dtype).name
    outs, digests = [], []
    for n, recs, op, off, x in gate_cases(dtype):
        outs.append(oracle.apply(x.copy(), recs, op, off))
        digests.append(case_digest(recs, op, off, x))
    assert len(outs) == int(GOLD[f"gates_{name}_count"])
    assert hashlib.sha256("".join(digests).encode()).hexdigest() == str(GOLD[f"gates_{name}_digest"])
    got = np.concatenate(outs)
    assert same_bits(got, GOLD[f"gates_{name}"])


@pytest.mark.parametrize("dtype", DTYPES, ids=lambda d: np.dtype(d).name)
def test_oracle_bitexact_on_circuit_fixtures(dtype):
    name = np.dtype(dtype).name
    for cname, n, recs, op, off, x in circuit_cases(dtype):
        assert str(GOLD[f"circ_{name}_{cname}_digest"]) == case_digest(recs, op, off, x)
        y = oracle.apply(x.copy(), recs, op, off)
        assert same_bits(y, GOLD[f"circ_{name}_{cname}"]), cname


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not built here")
@pytest.mark.parametrize("dtype", DTYPES, ids=lambda d: np.dtype(d).name)
def test_oracle_bitexact_vs_reference_random(dtype):
    rng = np.random.default_rng(5)
    real = np.dtype(dtype).kind == "f"
    for seed, n in enumerate([2, 4, 7, 10]):
        for op in "NTC":
            c = W.random_mixed(n - 1, 80, seed=seed, real=real)
            recs = c.gate_records(dtype)
            x = (rng.normal(size=1 << n) + (0 if real else 1j * rng.normal(size=1 << n))).astype(dtype)
            assert same_bits(oracle.apply(x.copy(), recs, op, 1),
                             oracle.ref_apply(x.copy(), recs, op, 1))


def test_matrix_gate2_is_kron_basis():
    """MatrixGate2 (new) acts in the kron basis |qubit0 qubit1>."""
    rng = np.random.default_rng(3)
    U = W.random_unitary(4, rng)
    for a, b in [(0, 2), (2, 0), (1, 2), (2, 1), (0, 1), (1, 0)]:
        c = QCircuit(3)
        c.push_back(MatrixGate2(a, b, U))
        x = rng.normal(size=8) + 1j * rng.normal(size=8)
        y = oracle.apply(x.copy(), c.gate_records(np.complex128))
        ax = "xyz"
        out = "".join("A" if q == a else "B" if q == b else ax[q] for q in range(3))
        ref = np.einsum(f"AB{ax[a]}{ax[b]},xyz->{out}", U.reshape(2, 2, 2, 2),
                        x.reshape(2, 2, 2)).reshape(-1)
        assert np.max(np.abs(ref - y)) < 1e-14


def test_qft_generator_gate_count():
    """examples/qft.cpp:21-35 yields n + n(n-1)/2 + n/2 gates: 220 at n = 20."""
    assert len(W.qft(20)) == 220
    assert len(W.brick(30, 200, seed=0)) == 200 * 30 + 100 * 15 + 100 * 14
    assert len(W.hea(24, 12)) == 12 * (24 + 24 + 23)

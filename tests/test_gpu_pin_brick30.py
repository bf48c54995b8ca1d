"""The headline configuration at full size: the 30-qubit random brick circuit
of depth 200 (8,900 gates, seed 2024, |0...0> input) against QCLAB++'s own
CPU QCircuit::simulate.  tests/golden/make_brick30_pin.py ran the compiled
reference once on that circuit and committed its final state's SHA-256,
FP64 norm, 4096 seeded sample amplitudes and 256-block probability profile.

* qsv_apply (the reference-exact path) over all 8,900 gates gives a state
  whose summary -- digest included -- equals the reference's: bitwise
  parity on the whole 16 GiB state (complex<double>) and 8 GiB state
  (complex<float>, against the reference's complex<float> simulate);
* the fused complex<double> sweep is within 1e-12 max-abs of that state;
* the fused complex<float> sweep (gate parameters in double) is within 1e-5
  max-abs of it, with 1 - |<psi32|psi64>|^2 <= 1e-6, for every engine.

Needs about 40 GiB of device memory and two minutes."""
from pathlib import Path

import numpy as np
import pytest

from qclab_b200 import StateVector
from qclab_b200 import _lib as L
from qclab_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
N, DEPTH, SEED = 30, 200, 2024


def fixture(tag):
    f = GOLDEN / f"brick{N}_d{DEPTH}_s{SEED}_{tag}.npz"
    if not f.exists():
        pytest.fail(f"missing fixture {f.name} (tests/golden/make_brick30_pin.py)")
    return dict(np.load(f))


def assert_summary_equal(got, want):
    assert got["sha256"] == str(want["sha256"]), "digest differs from QCLAB++ simulate"
    assert np.array_equal(got["idx"], want["idx"])
    assert np.array_equal(got["amp"], want["amp"])
    assert np.array_equal(got["block_p"], want["block_p"])
    assert got["norm2"] == float(want["norm2"])


@pytest.fixture(scope="module")
def reference_state(cuda):
    """qsv_apply over the whole circuit, pinned to the reference's digest."""
    want = fixture("c128")
    recs = W.brick(N, DEPTH, seed=SEED).gate_records(np.complex128)
    assert len(recs) == int(want["gates"])
    s = StateVector(N, np.complex128)
    s.apply(recs, "N", 0, fused=False)
    assert_summary_equal(s.summary(want["idx"]), want)
    yield s, recs
    s.close()


def test_reference_exact_path_equals_qclab_simulate(reference_state):
    s, recs = reference_state
    assert s.nbQubits == N and len(recs) == 8900


def test_fused_complex_double_within_1e12(reference_state):
    ref, recs = reference_state
    for opts in (None, L.FuseOpts(engine=5)):
        with StateVector(N, np.complex128) as f:
            f.apply(recs, "N", 0, fused=True, opts=opts)
            ip, maxabs = f.compare(ref)
            assert maxabs <= 1e-12, (opts and opts.engine, maxabs)
            assert abs(1.0 - abs(ip) ** 2) <= 1e-12


def test_fused_complex_float_within_1e5(reference_state):
    ref, recs = reference_state
    for opts in (None, L.FuseOpts(engine=5), L.FuseOpts(engine=5, reg_bits=4)):
        with StateVector(N, np.complex64) as f:
            f.apply(recs, "N", 0, fused=True, opts=opts)
            ip, maxabs = f.compare(ref)
            assert maxabs <= 1e-5, (opts and opts.engine, maxabs)
            assert 1.0 - abs(ip) ** 2 <= 1e-6, (opts and opts.engine, ip)


def test_reference_exact_complex_float_equals_qclab_simulate(cuda):
    want = fixture("c64")
    recs = W.brick(N, DEPTH, seed=SEED).gate_records(np.complex64)
    with StateVector(N, np.complex64) as s:
        s.apply(recs, "N", 0, fused=False)
        assert_summary_equal(s.summary(want["idx"]), want)

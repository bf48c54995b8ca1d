"""QCLAB++'s own gate objects through include/qclab_b200/adapter.hpp: the
C++ drop-in (reference-exact path bitwise, fused within 1e-10) against
QCLAB++'s CPU simulate/apply, for all ops, nested circuits with offsets,
pointer gates and a non-symmetric user QGate2."""
import subprocess

import pytest

import oracle

pytestmark = pytest.mark.gpu
BIN = oracle.HERE / "_ref" / "adapter_test"


@pytest.mark.skipif(not BIN.exists(), reason="adapter test is built where the reference tree exists")
def test_adapter_against_qclab_cpu(cuda):
    r = subprocess.run([str(BIN)], capture_output=True, text=True, timeout=600)
    if r.returncode != 0 or "all passed" not in r.stdout:
        pytest.fail(r.stdout[-6000:] + r.stderr[-2000:], pytrace=False)

"""The sweep timing command (python -m qclab_b200.sweep) on every engine:
plan statistics, timings, and the swept state against the oracle."""
import numpy as np
import pytest

import oracle
from qclab_b200 import sweep
from qclab_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,engine", [("c128", 0), ("c128", 1), ("c128", 5), ("c64", 5),
                                          ("c64", 0), ("c64", 2),
                                          ("c64", 3), ("c64", 4)])
def test_sweep_command(cuda, dtype, engine):
    out = sweep.main(["--qubits", "14", "--depth", "6", "--dtype", dtype, "--engine",
                      str(engine), "--repeat", "1"], keep_state=True)
    assert out["gates"] == 14 * 6 + sum(len(range(l % 2, 13, 2)) for l in range(6))
    assert out["stages"] >= 1 and out["passes"] >= out["stages"]
    assert len(out["ms"]) == 1 and out["gates_per_s"] > 0
    # the swept state: the same seeded circuit through the C oracle in FP64
    recs = W.brick(14, 6, seed=3).gate_records(np.complex128)
    want = np.zeros(1 << 14, dtype=np.complex128)
    want[0] = 1
    oracle.apply(want, recs)
    tol = 1e-12 if dtype == "c128" else 2e-5
    assert np.max(np.abs(out["state"].astype(np.complex128) - want)) < tol


def test_sweep_adjoint_and_batch(cuda):
    out = sweep.main(["--workload", "adjoint", "--qubits", "10", "--depth", "3", "--repeat", "1"])
    assert out["params"] == 10 * 2 * 3 and len(out["ms"]) == 1
    assert -20.0 < out["energy"] < 20.0
    out = sweep.main(["--workload", "batch", "--circuits", "16", "--dtype", "c64", "--repeat", "1"])
    assert out["circuits"] == 16 and out["gates"] > 0 and len(out["ms"]) == 1


def test_sweep_kernels_workload(cuda):
    out = sweep.main(["--workload", "kernels", "--qubits", "12", "--repeat", "1"])
    assert len(out["kernels"]) == 17
    assert all(v["ms"] > 0 for v in out["kernels"].values())

"""Host-side logic of the batched sweep (no GPU): argument validation in
qsv_batch_create (statuses come back before any device call), the
autotuner's candidate list and cache key."""
import numpy as np
import pytest

from qclab_b200 import QsvError
from qclab_b200 import workloads as W
from qclab_b200.batch import Batch, _signature, candidates
from qclab_b200.observable import ising


def test_validation_statuses():
    with pytest.raises(QsvError) as e:
        Batch([W.hea(6, 2)], [ising(6)], np.complex64, tile_bits=13)   # 2^(13-4) threads > 256
    assert e.value.status == 1
    with pytest.raises(QsvError) as e:
        Batch([W.hea(3, 2)], [ising(3)], np.complex64)                  # below the register width
    assert e.value.status == 3
    with pytest.raises(TypeError):
        Batch([W.hea(6, 2)], [ising(6)], np.float64)
    with pytest.raises(ValueError):
        Batch([W.hea(6, 2)], [ising(7)], np.complex64)
    with pytest.raises(ValueError):
        Batch([W.hea(6, 2)], [], np.complex64)


def test_candidates_and_signature():
    c64 = candidates(np.complex64)
    c128 = candidates(np.complex128)
    assert {c["tile_bits"] for c in c64} == {10, 11, 12}
    assert {c["tile_bits"] for c in c128} == {9, 10, 11}
    assert len(c64) == len({tuple(sorted(c.items())) for c in c64})
    circs = [W.hea(8, 3, seed=1), W.hea(10, 2, seed=2)]
    obs = [ising(8), ising(10)]
    k1 = _signature(circs, obs, np.complex64)
    assert k1 == _signature(circs, obs, np.complex64)
    assert k1 != _signature(circs, obs, np.complex128)
    assert k1 != _signature(circs[:1], obs[:1], np.complex64)

"""Batched variational sweeps: every circuit's energy and adjoint gradient
from one persistent launch, against the single-circuit adjoint sweep (GPU)
and the CPU oracle's energy.  Tolerances: 1e-10 (complex<double>), 2e-4
relative to the gradient's scale (complex<float>)."""
import math

import numpy as np
import pytest

import oracle
from qclab_b200 import (CNOT, CPhase, CRotationY, CRotationZ, Hadamard, Phase, QCircuit,
                        RotationX, RotationXX, RotationY, RotationYY, RotationZ, RotationZZ,
                        StateVector)
from qclab_b200 import QsvError
from qclab_b200 import workloads as W
from qclab_b200.batch import Batch, autotune
from qclab_b200.gradients import adjoint_gradient
from qclab_b200.observable import Observable, ising

pytestmark = pytest.mark.gpu


def mixed_circuit(n, seed):
    rng = np.random.default_rng(seed)
    ang = lambda: float(rng.uniform(0, 2 * math.pi))
    c = QCircuit(n)
    for q in range(n):
        c.push_back(Hadamard(q))
    for _ in range(2):
        for q in range(n):
            c.push_back(RotationX(q, ang()) if q % 2 else RotationY(q, ang()))
        for q in range(0, n - 1, 2):
            c.push_back(RotationZZ(q, q + 1, ang()))
        c.push_back(RotationXX(0, n - 1, ang()))
        c.push_back(RotationYY(1, n - 2, ang()))
        c.push_back(CRotationZ(n - 1, 0, ang()))
        c.push_back(CRotationY(2, n - 3, ang(), controlState=0))
        c.push_back(CPhase(0, n // 2, ang()))
        c.push_back(Phase(n - 2, ang()))
        c.push_back(RotationZ(n // 2, ang()))
        for q in range(n - 1):
            c.push_back(CNOT(q, q + 1))
    return c


def random_observable(n, seed, nterms=12):
    rng = np.random.default_rng(seed)
    H = ising(n)
    for _ in range(nterms):
        s = ["I"] * n
        for q in rng.choice(n, size=min(n, 3), replace=False):
            s[q] = "XYZ"[rng.integers(3)]
        H.add(float(rng.normal()), "".join(s))
    return H


def single(circ, H, dtype):
    with StateVector(circ.nbQubits(), dtype) as s:
        return adjoint_gradient(s, circ.gate_records(dtype, number_params=True), H,
                                circ.nbParameters())


def cpu_energy(circ, H):
    x = np.zeros(1 << circ.nbQubits(), dtype=np.complex128)
    x[0] = 1
    oracle.apply(x, circ.gate_records(np.complex128))
    return oracle.expectation(x, H.matrix_free_terms())


@pytest.mark.parametrize("tile_bits", [0, 10])
def test_batch_matches_single_circuit_adjoint_c128(cuda, tile_bits):
    # tile_bits=10 sends the 11..13-qubit circuits through the multi-tile path
    ns = [5, 6, 8, 9, 11, 12, 13, 7]
    circs = [mixed_circuit(n, 10 + i) if i % 2 else W.hea(n, 3 + i % 4, seed=i)
             for i, n in enumerate(ns)]
    obs = [random_observable(n, 20 + i) for i, n in enumerate(ns)]
    with Batch(circs, obs, np.complex128, tile_bits=tile_bits) as b:
        b.run(graph=False)
        e, g = b.results()
    for c, H, ec, gc in zip(circs, obs, e, g):
        e1, g1 = single(c, H, np.complex128)
        assert abs(ec - e1) < 1e-10
        assert abs(ec - cpu_energy(c, H)) < 1e-10
        assert gc.shape == g1.shape
        assert np.max(np.abs(gc - g1)) < 1e-10


def test_batch_c64_against_c128(cuda):
    rng = np.random.default_rng(5)
    ns = [int(x) for x in rng.integers(8, 15, size=24)]
    circs = [W.hea(n, int(rng.integers(4, 9)), seed=100 + i) for i, n in enumerate(ns)]
    obs = [ising(n) for n in ns]
    with Batch(circs, obs, np.complex64) as b:
        b.run()
        e, g = b.results()
    for c, H, ec, gc in zip(circs, obs, e, g):
        e1, g1 = single(c, H, np.complex128)
        scale = max(1.0, np.max(np.abs(g1)))
        assert abs(ec - e1) < 2e-4 * max(1.0, abs(e1))
        assert np.max(np.abs(gc - g1)) < 2e-4 * scale


def test_graph_replay_is_deterministic(cuda):
    ns = [9, 12, 10, 14, 8]
    circs = [W.hea(n, 5, seed=i) for i, n in enumerate(ns)]
    obs = [ising(n) for n in ns]
    with Batch(circs, obs, np.complex64, tile_bits=11) as b:
        b.run(graph=False)
        e0, g0 = b.results()
        for _ in range(3):
            b.run(graph=True)
            e1, g1 = b.results()
            assert np.array_equal(e0, e1)
            assert all(np.array_equal(x, y) for x, y in zip(g0, g1))
        info = b.info()
        assert info["tile_bits"] == 11 and info["blocks"] >= 1
        # work of one launch from the plan: every gate updates 2^n amplitudes
        # forward and 2 x 2^n backward; only the 12- and 14-qubit circuits
        # (larger than the 11-bit tiles) move tiles through global memory
        work = b.work()
        assert work["amplitude_updates"] == sum(3 * len(c) * 2 ** n for c, n in zip(circs, ns))
        assert work["global_bytes"] >= sum(8 * 2 ** n * 6 for n in ns if n > 11)


def test_shared_parameters_accumulate(cuda):
    n = 6
    c = W.hea(n, 3, seed=3)
    recs = c.gate_records(np.complex128, number_params=True)
    recs["param"] = np.where(recs["param"] >= 0, recs["param"] % 4, -1)  # 4 shared angles
    H = ising(n)
    with Batch([(n, recs, 4)], [H], np.complex128) as b:
        b.run()
        e, g = b.results()
    with StateVector(n, np.complex128) as s:
        e1, g1 = adjoint_gradient(s, recs, H, 4)
    assert abs(e[0] - e1) < 1e-12
    assert np.max(np.abs(g[0] - g1)) < 1e-10


def test_batch_errors(cuda):
    H = ising(6)
    with pytest.raises(QsvError) as e:
        Batch([W.hea(6, 2)], [H], np.complex64, tile_bits=13)
    assert e.value.status == 1
    with pytest.raises(QsvError) as e:
        Batch([W.hea(3, 2)], [ising(3)], np.complex64)
    assert e.value.status == 3
    recs = W.hea(6, 2).gate_records(np.complex64, number_params=True)
    with pytest.raises(QsvError) as e:
        Batch([(6, recs, 3)], [H], np.complex64)
    assert e.value.status == 1
    with pytest.raises(TypeError):
        Batch([W.hea(6, 2)], [H], np.float32)


def test_autotune_picks_and_caches(cuda, tmp_path):
    ns = [8, 10, 12, 9]
    circs = [W.hea(n, 4, seed=i) for i, n in enumerate(ns)]
    obs = [ising(n) for n in ns]
    cands = [{"tile_bits": 10, "low_bits": 2, "ctas_per_sm": 0},
             {"tile_bits": 12, "low_bits": 3, "ctas_per_sm": 2}]
    cache = tmp_path / "tune.json"
    best, times = autotune(circs, obs, np.complex64, cands=cands, cache=cache)
    assert best in cands and len(times) == 2
    assert cache.exists()
    best2, _ = autotune(circs, obs, np.complex64, cands=cands, cache=cache,
                        timer=lambda b: pytest.fail("cache not used"))
    assert best2 == best

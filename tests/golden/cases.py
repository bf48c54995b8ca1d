"""Deterministic parity cases shared by the golden-fixture generator
(make_golden.py) and the tests.

Single-gate cases: every gate class x every op x qubit placements
(n = 3: all placements; n = 6: low/high/mixed strides) x control states,
on three inputs: x = 1..2^n (the input pattern of the reference's own gate
tests, e.g. test/qgates/RotationX.cpp:288-300), a seeded random vector and
a vector of signed zeros and small exact values (special_input).
Circuit cases: QFT (examples/qft.cpp:21-35), brick circuits and random
mixed circuits, applied with all three ops and qubit offsets.
"""
from __future__ import annotations

import math

import numpy as np

from qclab_b200 import gates as G
from qclab_b200 import workloads as W
from qclab_b200.circuit import QCircuit

DTYPES = [np.complex128, np.complex64, np.float64, np.float32]


def _one_qubit_gates(q, rng, real):
    th = float(rng.uniform(0, 2 * math.pi))
    gs = [G.Identity(q), G.Hadamard(q), G.PauliX(q), G.PauliZ(q), G.RotationY(q, th),
          G.MatrixGate1(q, np.linalg.qr(rng.normal(size=(2, 2)))[0])]
    if not real:
        gs += [G.PauliY(q), G.RotationX(q, th), G.RotationZ(q, th), G.Phase(q, th),
               G.Phase45(q), G.Phase90(q), G.MatrixGate1(q, W.random_unitary(2, rng)),
               G.U3(q, th, 0.3, 1.1)]
    return gs


def _two_qubit_gates(a, b, rng, real):
    th = float(rng.uniform(0, 2 * math.pi))
    gs = []
    for cs in (0, 1):
        gs += [G.CX(a, b, cs), G.CZ(a, b, cs), G.CRotationY(a, b, th, controlState=cs),
               G.ControlledGate(a, b, np.linalg.qr(rng.normal(size=(2, 2)))[0], cs)]
        if not real:
            gs += [G.CY(a, b, cs), G.CPhase(a, b, th, controlState=cs),
                   G.CRotationX(a, b, th, controlState=cs), G.CRotationZ(a, b, th, controlState=cs),
                   G.ControlledGate(a, b, W.random_unitary(2, rng), cs)]
    gs += [G.SWAP(a, b), G.MatrixGate2(a, b, np.linalg.qr(rng.normal(size=(4, 4)))[0])]
    if not real:
        gs += [G.iSWAP(a, b), G.RotationXX(a, b, th), G.RotationYY(a, b, th),
               G.RotationZZ(a, b, th), G.MatrixGate2(a, b, W.random_unitary(4, rng))]
    return gs


def same_bits(a, b) -> bool:
    """Bitwise equality of two arrays: same dtype, shape and bytes (so -0 and
    +0 differ, where np.array_equal calls them equal)."""
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and a.tobytes() == b.tobytes()


def special_input(n, dtype, seed=0):
    """Components drawn from {+0, -0, 1, -1, 1/2, -1/2, 2}: exact
    cancellations and signed zeros, where a gate's arithmetic form (a swap,
    a real scaling, a negation, a general complex product) shows in the sign
    of zero results."""
    vals = np.array([0.0, -0.0, 1.0, -1.0, 0.5, -0.5, 2.0])
    x = np.zeros(1 << n, dtype=dtype)
    comp = x.view(np.float32 if np.dtype(dtype) in (np.dtype(np.complex64),
                                                    np.dtype(np.float32)) else np.float64)
    comp[:] = np.random.default_rng(1000 + 7 * n + seed).choice(vals, size=comp.size)
    return x


def _inputs(n, dtype, rng):
    N = 1 << n
    iota = np.arange(1, N + 1).astype(dtype)
    if np.dtype(dtype).kind == "c":
        rnd = (rng.normal(size=N) + 1j * rng.normal(size=N)).astype(dtype)
    else:
        rnd = rng.normal(size=N).astype(dtype)
    return [iota, rnd, special_input(n, dtype)]


def gate_cases(dtype):
    """Yields (n, records, op, offset, input) for single-gate cases."""
    rng = np.random.default_rng(1234 + DTYPES.index(dtype))
    real = np.dtype(dtype).kind == "f"
    for n, ones, pairs in [(3, [0, 1, 2], [(a, b) for a in range(3) for b in range(3) if a != b]),
                           (6, [0, 3, 5], [(0, 5), (5, 0), (1, 4), (4, 2), (5, 4)])]:
        for q in ones:
            for g in _one_qubit_gates(q, rng, real):
                recs = QCircuit(n)
                recs.push_back(g)
                r = recs.gate_records(dtype)
                for op in "NTC":
                    for x in _inputs(n, dtype, rng):
                        yield n, r, op, 0, x
        for a, b in pairs:
            for g in _two_qubit_gates(a, b, rng, real):
                recs = QCircuit(n)
                recs.push_back(g)
                r = recs.gate_records(dtype)
                for op in "NTC":
                    for x in _inputs(n, dtype, rng):
                        yield n, r, op, 0, x


def circuit_cases(dtype):
    """Yields (name, n, records, op, offset, input)."""
    rng = np.random.default_rng(99 + DTYPES.index(dtype))
    real = np.dtype(dtype).kind == "f"
    if not real:
        for n in (6, 10):
            c = W.qft(n)
            x = np.zeros(1 << n, dtype=dtype)
            x[W.basis_index(n, seed=n)] = 1
            yield f"qft{n}", n, c.gate_records(dtype), "N", 0, x
        c = W.brick(12, 8, seed=5)
        x = np.zeros(1 << 12, dtype=dtype)
        x[0] = 1
        yield "brick12", 12, c.gate_records(dtype), "N", 0, x
        c = W.hea(9, 3, seed=2)
        x = np.zeros(1 << 9, dtype=dtype)
        x[0] = 1
        yield "hea9", 9, c.gate_records(dtype), "N", 0, x
    for n in (5, 9):
        for op in "NTC":
            for off in (0, 2):
                c = W.random_mixed(n - off, 50, seed=7 * n + off, real=real)
                x = _inputs(n, dtype, rng)[1]
                yield f"mixed{n}{op}{off}", n, c.gate_records(dtype), op, off, x

"""Seeded circuit generators for the benchmark workloads and tests.

* ``qft``: the QFT of ``examples/qft.cpp:21-35`` (Hadamard, CPhase ladder
  with theta = -2*pi/2^j, final SWAP reversal): n + n(n-1)/2 + n/2 gates,
  220 for n = 20.
* ``brick``: random brick circuit -- per layer a gate from
  {Hadamard, RotationX, RotationY, RotationZ} on every qubit (angles uniform
  in [0, 2pi)), then CNOT or CZ (50/50) on (q, q+1) for even q on even
  layers and odd q on odd layers.
* ``hea``: hardware-efficient ansatz -- per layer RotationY and RotationZ on
  every qubit, then a CNOT ladder (i -> i+1).
* ``random_mixed``: every gate class of the library at random qubits, for
  parity tests.
"""
from __future__ import annotations

import math

import numpy as np

from . import gates as G
from .circuit import QCircuit


def qft(n: int) -> QCircuit:
    c = QCircuit(n)
    pi = 4 * math.atan(1)
    for i in range(n):
        c.push_back(G.Hadamard(i))
        for j in range(2, n - i + 1):
            control = j + i - 1
            theta = -2 * pi / (1 << j)
            c.push_back(G.CPhase(control, i, theta))
    for i in range(n // 2):
        c.push_back(G.SWAP(i, n - i - 1))
    return c


def brick(n: int, depth: int, seed: int = 0) -> QCircuit:
    rng = np.random.default_rng(seed)
    c = QCircuit(n)
    for layer in range(depth):
        kinds = rng.integers(0, 4, size=n)
        angles = rng.uniform(0.0, 2 * math.pi, size=n)
        for q in range(n):
            k = int(kinds[q])
            if k == 0:
                c.push_back(G.Hadamard(q))
            elif k == 1:
                c.push_back(G.RotationX(q, float(angles[q])))
            elif k == 2:
                c.push_back(G.RotationY(q, float(angles[q])))
            else:
                c.push_back(G.RotationZ(q, float(angles[q])))
        start = layer % 2
        pairs = list(range(start, n - 1, 2))
        ents = rng.integers(0, 2, size=len(pairs))
        for q, e in zip(pairs, ents):
            c.push_back(G.CNOT(q, q + 1) if e == 0 else G.CZ(q, q + 1))
    return c


def brick_layer_sizes(n: int, depth: int) -> list[int]:
    """Gates per layer of ``brick(n, depth)``: n one-qubit gates plus one
    two-qubit gate per pair (q, q+1), q of the layer's parity."""
    return [n + len(range(layer % 2, n - 1, 2)) for layer in range(depth)]


def hea(n: int, layers: int, seed: int = 0) -> QCircuit:
    rng = np.random.default_rng(seed)
    c = QCircuit(n)
    for _ in range(layers):
        a = rng.uniform(0.0, 2 * math.pi, size=2 * n)
        for q in range(n):
            c.push_back(G.RotationY(q, float(a[q])))
        for q in range(n):
            c.push_back(G.RotationZ(q, float(a[n + q])))
        for q in range(n - 1):
            c.push_back(G.CNOT(q, q + 1))
    return c


def random_unitary(dim: int, rng) -> np.ndarray:
    z = rng.normal(size=(dim, dim)) + 1j * rng.normal(size=(dim, dim))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def random_mixed(n: int, count: int, seed: int = 0, real: bool = False,
                 adjacent_generic: bool = False) -> QCircuit:
    """Random circuit over all gate classes (real-coefficient ones only for
    ``real=True``).  ``adjacent_generic`` puts the generic 2-qubit gates
    (RotationXX/YY/ZZ, MatrixGate2) on neighbouring qubits, the only
    placement QCLAB++'s unitary update of such gates accepts
    (src/qgates/QGate2.cpp:41)."""
    rng = np.random.default_rng(seed)
    c = QCircuit(n)
    one = [G.Identity, G.Hadamard, G.PauliX, G.PauliY, G.PauliZ, G.RotationX, G.RotationY,
           G.RotationZ, G.Phase, G.Phase45, G.Phase90, "M1", "U3"]
    two = [G.CX, G.CY, G.CZ, G.CPhase, G.CRotationX, G.CRotationY, G.CRotationZ, "C1", G.SWAP,
           G.iSWAP, G.RotationXX, G.RotationYY, G.RotationZZ, "M2"]
    if real:
        one = [G.Identity, G.Hadamard, G.PauliX, G.PauliZ, G.RotationY, "M1r"]
        two = [G.CX, G.CZ, G.CRotationY, "C1r", G.SWAP, "M2r"]
    for _ in range(count):
        if n < 2 or rng.random() < 0.55:
            q = int(rng.integers(0, n))
            t = one[int(rng.integers(0, len(one)))]
            th = float(rng.uniform(0, 2 * math.pi))
            if t == "M1":
                c.push_back(G.MatrixGate1(q, random_unitary(2, rng)))
            elif t == "M1r":
                c.push_back(G.MatrixGate1(q, np.linalg.qr(rng.normal(size=(2, 2)))[0]))
            elif t == "U3":
                c.push_back(G.U3(q, th, float(rng.uniform(0, 6.28)), float(rng.uniform(0, 6.28))))
            elif t in (G.RotationX, G.RotationY, G.RotationZ, G.Phase):
                c.push_back(t(q, th))
            else:
                c.push_back(t(q))
        else:
            a, b = (int(x) for x in rng.choice(n, size=2, replace=False))
            t = two[int(rng.integers(0, len(two)))]
            th = float(rng.uniform(0, 2 * math.pi))
            cs = int(rng.integers(0, 2))
            if adjacent_generic and t in (G.RotationXX, G.RotationYY, G.RotationZZ, "M2", "M2r"):
                a = min(a, b, n - 2)
                b = a + 1
            if t == "M2":
                c.push_back(G.MatrixGate2(a, b, random_unitary(4, rng)))
            elif t == "M2r":
                c.push_back(G.MatrixGate2(a, b, np.linalg.qr(rng.normal(size=(4, 4)))[0]))
            elif t == "C1":
                c.push_back(G.ControlledGate(a, b, random_unitary(2, rng), cs))
            elif t == "C1r":
                c.push_back(G.ControlledGate(a, b, np.linalg.qr(rng.normal(size=(2, 2)))[0], cs))
            elif t in (G.CX, G.CY, G.CZ):
                c.push_back(t(a, b, cs))
            elif t in (G.CPhase, G.CRotationX, G.CRotationY, G.CRotationZ):
                c.push_back(t(a, b, th, controlState=cs))
            elif t in (G.RotationXX, G.RotationYY, G.RotationZZ):
                c.push_back(t(a, b, th))
            else:
                c.push_back(t(a, b))
    return c


def basis_index(n: int, seed: int) -> int:
    """A uniformly random n-bit basis index from a seed (qubit 0 = MSB)."""
    rng = np.random.default_rng(seed)
    return int(rng.integers(0, 1 << n))

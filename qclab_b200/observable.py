"""Pauli-sum observables H = sum_t c_t P_t (new: QCLAB++ has none).

A term is a string of nbQubits characters from {I, X, Y, Z}; character q is
the Pauli on qubit q (qubit 0 first, the QCLAB++ order).  Evaluation runs on
the GPU in FP64 (``StateVector.expectation``)."""
from __future__ import annotations

import ctypes as C

import numpy as np


class Observable:
    def __init__(self, nbQubits: int, terms=()):
        self.nbQubits = int(nbQubits)
        self.coefs: list[float] = []
        self.paulis: list[str] = []
        for c, p in terms:
            self.add(c, p)

    def add(self, coef: float, paulis) -> "Observable":
        """Adds coef * P; ``paulis`` is a full string or a {qubit: 'X'} dict."""
        if isinstance(paulis, dict):
            s = ["I"] * self.nbQubits
            for q, c in paulis.items():
                s[q] = c
            paulis = "".join(s)
        paulis = paulis.upper()
        if len(paulis) != self.nbQubits or set(paulis) - set("IXYZ"):
            raise ValueError(f"bad Pauli string {paulis!r}")
        self.coefs.append(float(coef))
        self.paulis.append(paulis)
        return self

    def __len__(self) -> int:
        return len(self.coefs)

    def c_args(self):
        """(char* paulis, double* coefs, nTerms) for the C ABI."""
        buf = "".join(self.paulis).encode()
        coefs = (C.c_double * max(1, len(self.coefs)))(*self.coefs)
        return buf, coefs, len(self.coefs)

    def matrix_free_terms(self):
        return list(zip(self.coefs, self.paulis))


def ising(n: int, J: float = 1.0, h: float = 0.5) -> Observable:
    """Transverse-field Ising chain H = J sum_i Z_i Z_{i+1} + h sum_i X_i
    (open boundary)."""
    H = Observable(n)
    for i in range(n - 1):
        H.add(J, {i: "Z", i + 1: "Z"})
    for i in range(n):
        H.add(h, {i: "X"})
    return H

"""B200-native state-vector backend for QCLAB++.

A drop-in for the reference's ``QCircuit<T,G>::simulate`` /
``QObject<T>::apply(Op, nbQubits, vector, offset)`` path: gates lower to flat
records and run as hand-written sm_100a CUDA kernels behind the C ABI in
``include/qclab_b200.h``.  There is no CPU fallback.
"""
from . import _lib
from ._lib import QsvError
from .util import Op, Side
from .gates import (QObject, QGate1, QGate2, QControlledGate2, Identity, Hadamard, PauliX,
                    PauliY, PauliZ, RotationX, RotationY, RotationZ, Phase, Phase45, Phase90,
                    MatrixGate1, U2, U3, PointerGate1, PointerGate2, SWAP, iSWAP, RotationXX,
                    RotationYY, RotationZZ, MatrixGate2, ControlledGate, CX, CNOT, CY, CZ,
                    CPhase, CRotationX, CRotationY, CRotationZ)
from .circuit import QCircuit
from .state import StateVector, launch_count, tma_launch_count
from .sharded import ShardedStateVector

__all__ = [n for n in dir() if not n.startswith("_")]

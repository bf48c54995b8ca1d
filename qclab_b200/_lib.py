"""ctypes binding of the C ABI declared in ``include/qclab_b200.h``.

The shared library is the product: nothing here computes amplitudes.  If
``libqclab_b200.so`` is missing it is built in place with nvcc (sm_100a);
if that fails, importing raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
# QCLAB_B200_LIB selects another build of the library (no in-place build then)
LIB_PATH = Path(os.environ.get("QCLAB_B200_LIB", _PKG / "libqclab_b200.so"))

# ---- enums (mirror include/qclab_b200.h) ----------------------------------
SUCCESS = 0
STATUS_NAMES = {
    0: "QSV_SUCCESS", 1: "QSV_ERROR_INVALID_VALUE", 2: "QSV_ERROR_QUBIT",
    3: "QSV_ERROR_SIZE", 4: "QSV_ERROR_CUDA", 5: "QSV_ERROR_OUT_OF_MEMORY",
    6: "QSV_ERROR_DTYPE", 7: "QSV_ERROR_TIMEOUT", 8: "QSV_ERROR_NOT_SUPPORTED",
}

C64, C128, F32, F64 = 0, 1, 2, 3
DTYPE_OF_NUMPY = {
    np.dtype(np.complex64): C64, np.dtype(np.complex128): C128,
    np.dtype(np.float32): F32, np.dtype(np.float64): F64,
}
NUMPY_OF_DTYPE = {v: k for k, v in DTYPE_OF_NUMPY.items()}

(IDENTITY, HADAMARD, PAULI_X, PAULI_Y, PAULI_Z, ROTATION_X, ROTATION_Y,
 ROTATION_Z, PHASE, PHASE45, PHASE90, MATRIX1, CX, CY, CZ, CPHASE,
 CROTATION_X, CROTATION_Y, CROTATION_Z, CONTROLLED1, SWAP, ISWAP,
 ROTATION_XX, ROTATION_YY, ROTATION_ZZ, MATRIX2) = range(26)
NUM_GATE_KINDS = 26


class Gate(C.Structure):
    """``qsv_gate``: the flat record of one QCLAB++ gate."""
    _fields_ = [
        ("kind", C.c_int32), ("qubit0", C.c_int32), ("qubit1", C.c_int32),
        ("control_state", C.c_int32), ("cos", C.c_double), ("sin", C.c_double),
        ("matrix", C.c_double * 32), ("param", C.c_int32), ("reserved", C.c_int32),
    ]


class FuseOpts(C.Structure):
    """``qsv_fuse_opts``."""
    _fields_ = [("tile_bits", C.c_int), ("low_bits", C.c_int), ("reg_bits", C.c_int),
                ("max_stage_gates", C.c_int), ("profile", C.c_int), ("engine", C.c_int),
                ("ctas_per_sm", C.c_int), ("tile_copy", C.c_int)]


class BatchOpts(C.Structure):
    """``qsv_batch_opts``."""
    _fields_ = [("tile_bits", C.c_int), ("low_bits", C.c_int), ("ctas_per_sm", C.c_int),
                ("max_team", C.c_int), ("reserved", C.c_int * 4)]


GATE_DTYPE = np.dtype([
    ("kind", np.int32), ("qubit0", np.int32), ("qubit1", np.int32),
    ("control_state", np.int32), ("cos", np.float64), ("sin", np.float64),
    ("matrix", np.float64, (32,)), ("param", np.int32), ("reserved", np.int32),
])
assert GATE_DTYPE.itemsize == C.sizeof(Gate)


class QsvError(RuntimeError):
    """A C-ABI call returned a non-zero qsv_status."""

    def __init__(self, status: int, where: str, message: str):
        self.status = status
        self.status_name = STATUS_NAMES.get(status, f"status {status}")
        super().__init__(f"{where}: {self.status_name}: {message}")


_lock = threading.Lock()
_lib = None


def _declare(lib):
    p, i, sz, d = C.c_void_p, C.c_int, C.c_size_t, C.c_double
    gp = C.c_void_p  # const qsv_gate*
    sigs = {
        "qsv_abi_version": ([], C.c_int),
        "qsv_last_error": ([], C.c_char_p),
        "qsv_status_string": ([i], C.c_char_p),
        "qsv_launch_count": ([], C.c_uint64),
        "qsv_tma_launch_count": ([], C.c_uint64),
        "qsv_create": ([i, i, C.POINTER(p)], i),
        "qsv_wrap": ([i, i, p, C.POINTER(p)], i),
        "qsv_destroy": ([p], i),
        "qsv_set_stream": ([p, p], i),
        "qsv_info": ([p, C.POINTER(i), C.POINTER(i), C.POINTER(p)], i),
        "qsv_upload": ([p, p, sz], i),
        "qsv_download": ([p, p, sz], i),
        "qsv_copy": ([p, p], i),
        "qsv_set_basis": ([p, C.c_uint64], i),
        "qsv_synchronize": ([p], i),
        "qsv_apply": ([p, gp, sz, C.c_char, i], i),
        "qsv_apply_fused": ([p, gp, sz, C.c_char, i, p], i),
        "qsv_plan_stats": ([i, i, gp, sz, C.c_char, i, p, C.POINTER(i), p, i], i),
        "qsv_plan_passes": ([i, i, gp, sz, C.c_char, i, p, C.POINTER(i), C.POINTER(i),
                             C.POINTER(i)], i),
        "qsv_apply_host": ([i, i, p, gp, sz, C.c_char, i, i], i),
        "qsv_last_stage_times": ([C.POINTER(C.c_float), i, C.POINTER(i)], i),
        "qsv_norm2": ([p, C.POINTER(d)], i),
        "qsv_inner": ([p, p, C.POINTER(d)], i),
        "qsv_expectation": ([p, C.c_char_p, C.POINTER(d), sz, C.POINTER(d)], i),
        "qsv_apply_observable": ([p, p, C.c_char_p, C.POINTER(d), sz], i),
        "qsv_expectation_noalloc": ([p, i, i, p, C.c_char_p, C.POINTER(d), sz, C.POINTER(d)], i),
        "qsv_compare": ([p, p, C.POINTER(d)], i),
        "qsv_normalize": ([p, C.POINTER(d)], i),
        "qsv_parse_qasm": ([C.c_char_p, i, p, sz, C.POINTER(sz), C.POINTER(i)], i),
        "qsv_adjoint_gradient": ([p, gp, sz, C.c_char_p, C.POINTER(d), sz, C.POINTER(d), i,
                                  C.POINTER(d)], i),
        "qsv_batch_create": ([i, i, p, gp, p, C.c_char_p, p, p, p, p, C.POINTER(p)], i),
        "qsv_batch_run": ([p, p, i], i),
        "qsv_batch_results": ([p, p, p, p], i),
        "qsv_batch_info": ([p, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(sz)], i),
        "qsv_batch_work": ([p, C.POINTER(C.c_double), C.POINTER(C.c_double)], i),
        "qsv_batch_destroy": ([p], i),
        "qsv_set_identity": ([p], i),
        "qsv_apply_matrix": ([p, gp, sz, C.c_char, C.c_char, i, i], i),
        "qsv_nrmF": ([p, p, C.POINTER(d)], i),
        "qsv_fp64_mma_peak": ([C.POINTER(d)], i),
    }
    for name, (args, res) in sigs.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


def load(build_if_missing: bool = True):
    """Returns the loaded library (building it with nvcc if it is absent)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if build_if_missing and "QCLAB_B200_LIB" not in os.environ:
            from . import build as _build
            _build.build()
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing and could not be built")
        lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | getattr(os, "RTLD_GLOBAL", 0))
        _lib = _declare(lib)
        if _lib.qsv_abi_version() != 1:
            raise ImportError("qclab_b200 ABI version mismatch")
        return _lib


def check(status: int, where: str) -> None:
    if status != SUCCESS:
        msg = load().qsv_last_error()
        raise QsvError(status, where, msg.decode() if msg else "")


def gate_array(records: np.ndarray):
    """(pointer, count) of a GATE_DTYPE array for the C ABI."""
    if records.dtype != GATE_DTYPE:
        raise TypeError("gate records must have GATE_DTYPE")
    records = np.ascontiguousarray(records)
    return records, C.c_void_p(records.ctypes.data), len(records)

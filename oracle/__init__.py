"""CPU oracle for the QCLAB++ state-vector path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker.  The product
(``qclab_b200``) never imports it.

* ``apply``: the plain-C restatement in ``qsv_oracle.c`` (built to
  ``liboracle.so`` with gcc, no FMA contraction).
* ``Ref``: QCLAB++ itself, compiled from its own sources into
  ``_ref/libqclab_ref.so`` (``oracle/Makefile``; only where the reference
  tree exists -- the library then travels with the repository).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libqclab_ref.so"
REF_TESTS = HERE / "_ref" / "ref_tests"

DTYPE_CODE = {np.dtype(np.complex64): 0, np.dtype(np.complex128): 1,
              np.dtype(np.float32): 2, np.dtype(np.float64): 3}

_lock = threading.Lock()
_lib = None
_ref = None


def ref_tree() -> Path | None:
    """The QCLAB++ source tree: $QCLAB_REF, else the tree the last build of
    _ref/ used (recorded in _ref/REF_TREE); None when neither exists."""
    cands = [os.environ.get("QCLAB_REF", "")]
    rec = HERE / "_ref" / "REF_TREE"
    if rec.exists():
        cands.append(rec.read_text().strip())
    for c in cands:
        if c and (Path(c) / "src" / "qgates" / "apply.hpp").exists():
            return Path(c)
    return None


def build() -> None:
    """Builds liboracle.so (always) and _ref/ (when ref_tree() finds the
    reference tree)."""
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    tree = ref_tree()
    if tree is not None:
        env["QCLAB_REF"] = str(tree)
    r = subprocess.run(["make", "-C", str(HERE), "-j8", "all"], capture_output=True, text=True,
                       env=env)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout[-4000:]}\n{r.stderr[-4000:]}")


def _build_oracle_only() -> None:
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    r = subprocess.run(["make", "-C", str(HERE), "liboracle.so"], capture_output=True, text=True,
                       env=env)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout[-4000:]}\n{r.stderr[-4000:]}")


def load():
    global _lib
    with _lock:
        if _lib is None:
            src = HERE / "qsv_oracle.c"
            if not LIB.exists() or LIB.stat().st_mtime < max(
                    src.stat().st_mtime, (HERE / "oracle_impl.h").stat().st_mtime):
                _build_oracle_only()
            lib = C.CDLL(str(LIB))
            lib.oracle_apply.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_size_t,
                                         C.c_char, C.c_int]
            lib.oracle_apply.restype = C.c_int
            lib.oracle_cosf.argtypes = [C.c_float]
            lib.oracle_cosf.restype = C.c_float
            lib.oracle_sinf.argtypes = [C.c_float]
            lib.oracle_sinf.restype = C.c_float
            _lib = lib
        return _lib


def _records(recs):
    from qclab_b200 import _lib as L
    if isinstance(recs, np.ndarray) and recs.dtype == L.GATE_DTYPE:
        return np.ascontiguousarray(recs)
    return np.array(list(recs), dtype=L.GATE_DTYPE)


def apply(state: np.ndarray, recs, op: str = "N", offset: int = 0) -> np.ndarray:
    """Applies gate records to ``state`` (host, in place) with the C oracle."""
    lib = load()
    r = _records(recs)
    n = int(state.size).bit_length() - 1
    if state.size != 1 << n or not state.flags.c_contiguous:
        raise ValueError("state must be a contiguous power-of-two vector")
    st = lib.oracle_apply(n, DTYPE_CODE[state.dtype], state.ctypes.data,
                          r.ctypes.data if len(r) else None, len(r), op.encode(), int(offset))
    if st != 0:
        raise RuntimeError(f"oracle_apply failed with status {st}")
    return state


def ref_available() -> bool:
    return REF_LIB.exists()


def _load_ref():
    global _ref
    with _lock:
        if _ref is None:
            lib = C.CDLL(str(REF_LIB))
            lib.ref_circuit_create.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_size_t,
                                               C.POINTER(C.c_int)]
            lib.ref_circuit_create.restype = C.c_void_p
            lib.ref_circuit_destroy.argtypes = [C.c_void_p]
            lib.ref_vec_create.argtypes = [C.c_int, C.c_uint64]
            lib.ref_vec_create.restype = C.c_void_p
            lib.ref_vec_data.argtypes = [C.c_void_p]
            lib.ref_vec_data.restype = C.c_void_p
            lib.ref_vec_destroy.argtypes = [C.c_void_p]
            lib.ref_circuit_apply.argtypes = [C.c_void_p, C.c_void_p, C.c_char, C.c_int]
            lib.ref_circuit_apply.restype = C.c_int
            lib.ref_circuit_apply_side.argtypes = [C.c_void_p, C.c_char, C.c_char, C.c_int,
                                                   C.c_int, C.c_void_p]
            lib.ref_circuit_apply_side.restype = C.c_int
            lib.ref_circuit_matrix.argtypes = [C.c_void_p, C.c_void_p]
            lib.ref_circuit_matrix.restype = C.c_int
            lib.ref_nrmF.argtypes = [C.c_void_p, C.c_void_p]
            lib.ref_nrmF.restype = C.c_double
            lib.ref_num_threads.restype = C.c_int
            lib.ref_set_num_threads.argtypes = [C.c_int]
            _ref = lib
        return _ref


class RefCircuit:
    """A QCLAB++ ``QCircuit<T>`` built from records, with a driver-owned
    ``std::vector<T>`` state (exposed as a numpy view)."""

    def __init__(self, n: int, dtype, recs):
        self.lib = _load_ref()
        self.n = n
        self.dtype = np.dtype(dtype)
        r = _records(recs)
        st = C.c_int(0)
        self.c = self.lib.ref_circuit_create(n, DTYPE_CODE[self.dtype],
                                             r.ctypes.data if len(r) else None, len(r),
                                             C.byref(st))
        if not self.c:
            raise RuntimeError(f"reference circuit construction failed ({st.value})")
        self.v = self.lib.ref_vec_create(DTYPE_CODE[self.dtype], 1 << n)
        ptr = self.lib.ref_vec_data(self.v)
        buf = (C.c_char * ((1 << n) * self.dtype.itemsize)).from_address(ptr)
        self.state = np.frombuffer(buf, dtype=self.dtype)

    def apply(self, op: str = "N", offset: int = 0) -> None:
        st = self.lib.ref_circuit_apply(self.c, self.v, op.encode(), int(offset))
        if st != 0:
            raise RuntimeError(f"reference apply failed ({st})")

    def close(self) -> None:
        if self.c:
            self.lib.ref_circuit_destroy(self.c)
            self.c = None
        if self.v:
            self.state = None
            self.lib.ref_vec_destroy(self.v)
            self.v = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_apply(state: np.ndarray, recs, op: str = "N", offset: int = 0) -> np.ndarray:
    """Runs the reference's QCircuit::apply on a copy of ``state``."""
    n = int(state.size).bit_length() - 1
    rc = RefCircuit(n, state.dtype, recs)
    rc.state[:] = state
    rc.apply(op, offset)
    out = rc.state.copy()
    rc.close()
    return out


def ref_matrix(n: int, dtype, recs) -> np.ndarray:
    """The reference's ``QCircuit<T>::matrix()`` of a record list."""
    rc = RefCircuit(n, dtype, recs)
    out = np.zeros((1 << n) * (1 << n), dtype=rc.dtype)
    st = rc.lib.ref_circuit_matrix(rc.c, out.ctypes.data)
    rc.close()
    if st:
        raise RuntimeError(f"reference matrix failed ({st})")
    return out.reshape(1 << n, 1 << n, order="F")


def ref_apply_side(matrix: np.ndarray, recs, side: str, op: str, nbq: int, offset: int = 0,
                   circuit_qubits: int | None = None) -> np.ndarray:
    """The reference's ``QCircuit<T>::apply(side, op, nbq, matrix, offset)``
    on a copy of ``matrix`` (the circuit has ``circuit_qubits`` qubits)."""
    rc = RefCircuit(circuit_qubits or nbq, matrix.dtype, recs)
    buf = np.ascontiguousarray(matrix.flatten(order="F"))
    st = rc.lib.ref_circuit_apply_side(rc.c, side.encode(), op.encode(), nbq, offset,
                                       buf.ctypes.data)
    rc.close()
    if st:
        raise RuntimeError(f"reference apply(side) failed ({st})")
    return buf.reshape(matrix.shape, order="F")


def ref_nrmF(n: int, dtype, recs1, recs2) -> float:
    """The reference's ``qclab::nrmF`` of two record lists."""
    a, b = RefCircuit(n, dtype, recs1), RefCircuit(n, dtype, recs2)
    v = float(a.lib.ref_nrmF(a.c, b.c))
    a.close()
    b.close()
    return v


def nrmF(m1: np.ndarray, m2: np.ndarray) -> float:
    """numpy restatement of qclab::nrmF (include/qclab/QCircuit.hpp:407-430)
    on two matrices: scale = max |m1 - m2| (1 if 0), FP64."""
    d = m1.astype(np.complex128) - m2.astype(np.complex128)
    scale = float(np.max(np.abs(d))) if d.size else 0.0
    if scale == 0.0:
        scale = 1.0
    return scale * float(np.sqrt(np.sum((d.real / scale) ** 2 + (d.imag / scale) ** 2)))


def ref_threads() -> int:
    return int(_load_ref().ref_num_threads())


# ---- FP64 reductions (host restatement, numpy) -----------------------------
def pauli_apply(psi: np.ndarray, paulis: str) -> np.ndarray:
    """P psi for a Pauli string (character q acts on qubit q = bit n-1-q)."""
    N = psi.size
    n = N.bit_length() - 1
    f = zy = ny = 0
    for q, c in enumerate(paulis):
        b = 1 << (n - 1 - q)
        if c == "X":
            f |= b
        elif c == "Y":
            f |= b
            zy |= b
            ny += 1
        elif c == "Z":
            zy |= b
    j = np.arange(N, dtype=np.uint64)
    src = j ^ np.uint64(f)
    sign = 1.0 - 2.0 * (np.bitwise_count(src & np.uint64(zy)) & 1).astype(np.float64)
    return (1j ** ny) * sign * psi.astype(np.complex128)[src]


def expectation(psi: np.ndarray, terms) -> float:
    """sum_t c_t <psi|P_t|psi> in FP64; terms = [(coef, pauli string)]."""
    x = psi.astype(np.complex128)
    return float(sum(c * np.vdot(x, pauli_apply(x, p)).real for c, p in terms))


def observable_apply(psi: np.ndarray, terms) -> np.ndarray:
    out = np.zeros(psi.size, dtype=np.complex128)
    for c, p in terms:
        out += c * pauli_apply(psi, p)
    return out

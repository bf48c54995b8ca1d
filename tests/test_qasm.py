"""OpenQASM front end against QCLAB++'s own reader (CPU) and on the GPU."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle
from qclab_b200 import QsvError, StateVector
from qclab_b200 import qasm

QASM = Path(__file__).resolve().parent / "golden" / "qasm"
FILES = ["mixed.qasm", "qft6.qasm"]


def ref_qasm_state(path, dtype, x):
    """QCLAB++: QCircuit<T>(filename) then apply on x (CPU)."""
    lib = oracle._load_ref()
    lib.ref_circuit_from_qasm.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_int)]
    lib.ref_circuit_from_qasm.restype = C.c_void_p
    lib.ref_circuit_nb_gates.argtypes = [C.c_void_p]
    nq = C.c_int()
    c = lib.ref_circuit_from_qasm(str(path).encode(), oracle.DTYPE_CODE[np.dtype(dtype)], C.byref(nq))
    v = lib.ref_vec_create(oracle.DTYPE_CODE[np.dtype(dtype)], 1 << nq.value)
    buf = (C.c_char * (x.nbytes)).from_address(lib.ref_vec_data(v))
    st = np.frombuffer(buf, dtype=dtype)
    st[:] = x
    assert lib.ref_circuit_apply(c, v, b"N", 0) == 0
    out = st.copy()
    ng = lib.ref_circuit_nb_gates(c)
    lib.ref_circuit_destroy(c)
    lib.ref_vec_destroy(v)
    return out, ng


@pytest.mark.parametrize("name", FILES)
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=lambda d: np.dtype(d).name)
def test_reader_matches_reference_reader(name, dtype):
    n, recs = qasm.parse((QASM / name).read_text(), dtype)
    rng = np.random.default_rng(0)
    x = (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)).astype(dtype)
    y = oracle.apply(x.copy(), recs)
    if not oracle.ref_available():
        pytest.skip("reference not built here")
    ref, ng = ref_qasm_state(QASM / name, dtype, x)
    assert ng == len(recs)
    assert np.array_equal(y, ref)


def test_reader_details():
    n, recs = qasm.parse((QASM / "mixed.qasm").read_text())
    assert n == 5
    # s, barrier, measure, creg skipped; 14 gates read
    assert len(recs) == 14
    assert [int(r["qubit0"]) for r in recs[-2:]] == [3, 2]
    with pytest.raises(QsvError) as e:
        qasm.parse((QASM / "bad_angle.qasm").read_text())
    assert e.value.status == 1
    assert len(e.value.partial[1]) == 1  # the reference keeps the gates read so far
    c = qasm.read(QASM / "qft6.qasm")
    assert c.nbQubits() == 6 and len(c) == 8


@pytest.mark.gpu
@pytest.mark.parametrize("name", FILES)
def test_qasm_on_gpu_bitexact(cuda, name):
    c = qasm.read(QASM / name)
    n = c.nbQubits()
    rng = np.random.default_rng(1)
    x = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    ref = oracle.apply(x.copy(), c.gate_records(np.complex128))
    y = x.copy()
    c.simulate(y)
    assert np.array_equal(y, ref)

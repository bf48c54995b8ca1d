"""qsv_expectation_noalloc: the expectation value for callers that cannot
allocate device memory (their framework owns the GPU's memory, or they
cannot pay for cudaMalloc's device synchronisation).  Its work memory is a
fixed array inside the library, so this test checks, through the C ABI,
that it gives the same value as the allocating qsv_expectation (within the
1e-12 relative tolerance of the other FP64 reduction tests) on two calls in
a row, which share that array, and that it rejects an observable too large
for it.  Collected last on purpose; it must also pass alone in a fresh
process."""
import ctypes as C

import numpy as np
import pytest

from qclab_b200 import StateVector
from qclab_b200 import _lib as L
from qclab_b200.observable import Observable, ising

pytestmark = pytest.mark.gpu


def noalloc_expectation(state: StateVector, obs: Observable) -> float:
    buf, coefs, nt = obs.c_args()
    out = C.c_double()
    L.check(L.load().qsv_expectation_noalloc(C.c_void_p(state.device_ptr()), state.nbQubits,
                                             state.qsv_dtype, None, buf, coefs, nt,
                                             C.byref(out)),
            "qsv_expectation_noalloc")
    return out.value


def random_state(n, dtype, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return (x / np.linalg.norm(x)).astype(dtype)


def mixed_observable(n, seed):
    rng = np.random.default_rng(seed)
    H = ising(n)
    for _ in range(6):  # Pauli strings with many X/Y factors (the wide-term path)
        H.add(float(rng.normal()), "".join(rng.choice(list("XYZ"), size=n)))
    return H


def test_noalloc_expectation_matches_allocating_entry_point(cuda):
    cases = [(20, np.complex128, 1), (15, np.complex64, 2)]
    for n, dtype, seed in cases:  # two calls in a row on the shared array
        with StateVector(n, dtype) as s:
            s.upload(random_state(n, dtype, seed))
            H = mixed_observable(n, seed)
            ref = s.expectation(H)
            got = noalloc_expectation(s, H)
            assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)), (n, got, ref)
            assert noalloc_expectation(s, H) == got


def test_noalloc_rejects_oversized_observable(cuda):
    n = 22
    with StateVector(n, np.complex128) as s:
        H = Observable(n)
        for k in range(150):  # 150 wide terms need more partial sums than 1 MiB holds
            H.add(1.0, ("XY" * n)[k % 2:k % 2 + n])
        with pytest.raises(L.QsvError) as e:
            noalloc_expectation(s, H)
        assert e.value.status == 3
        assert "1048576" in str(e.value)

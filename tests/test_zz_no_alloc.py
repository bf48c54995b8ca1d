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

import oracle
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
    if np.dtype(dtype).kind == "f":
        x = rng.normal(size=1 << n)
    else:
        x = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return (x / np.linalg.norm(x)).astype(dtype)


def mixed_observable(n, seed, real=False):
    """Ising H plus six Pauli strings with many X/Y factors (the wide-term
    path); only X and Z for real element types, where an odd number of Y
    factors has no real expectation value."""
    rng = np.random.default_rng(seed)
    H = ising(n)
    for _ in range(6):
        H.add(float(rng.normal()), "".join(rng.choice(list("XZ" if real else "XYZ"), size=n)))
    return H


DTYPES = [np.complex128, np.complex64, np.float64, np.float32]


# n = 3: one tile holds the whole state (a single CTA of 32 threads);
# n = 12: tiles of 2^12 (complex<double>) or 2^13 elements;
# n = 24: more tiles than the 592 CTAs, so every CTA reuses its slot.
@pytest.mark.parametrize("dtype", DTYPES, ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("n", [3, 12, 24])
def test_noalloc_expectation_matches_allocating_entry_point(cuda, n, dtype):
    real = np.dtype(dtype).kind == "f"
    x = random_state(n, dtype, seed=n)
    H = mixed_observable(n, seed=n, real=real)
    with StateVector(n, dtype) as s:
        s.upload(x)
        ref = s.expectation(H)
        got = noalloc_expectation(s, H)
        assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)), (n, got, ref)
        # a second call on the same shared work array gives the same bits
        assert noalloc_expectation(s, H) == got
    if n <= 12:  # and directly against the FP64 host restatement
        want = oracle.expectation(x, H.matrix_free_terms())
        assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (n, got, want)


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

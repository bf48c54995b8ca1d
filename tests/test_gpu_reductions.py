"""FP64 reductions on the GPU against numpy (FP64) restatements."""
import numpy as np
import pytest

import oracle
from qclab_b200 import QsvError, StateVector
from qclab_b200.observable import Observable, ising

pytestmark = pytest.mark.gpu
DTYPES = [np.complex128, np.complex64, np.float64, np.float32]


def rand_state(n, dtype, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=1 << n) + (1j * rng.normal(size=1 << n) if np.dtype(dtype).kind == "c" else 0)
    return (x / np.linalg.norm(x)).astype(dtype)


def rand_observable(n, nterms, seed, allow_y=True):
    rng = np.random.default_rng(seed)
    H = Observable(n)
    letters = "IXYZ" if allow_y else "IXZ"
    for _ in range(nterms):
        H.add(float(rng.normal()), "".join(rng.choice(list(letters), size=n)))
    return H


def rtol(dtype):
    return 1e-12 if np.dtype(dtype) in (np.dtype(np.complex128), np.dtype(np.float64)) else 1e-6


@pytest.mark.parametrize("dtype", DTYPES, ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("n", [1, 5, 13, 20])
def test_norm_and_inner(cuda, dtype, n):
    x, y = rand_state(n, dtype, 1), rand_state(n, dtype, 2)
    with StateVector(n, dtype) as a, StateVector(n, dtype) as b:
        a.upload(x)
        b.upload(y)
        x2, y2 = x.astype(np.complex128), y.astype(np.complex128)
        ref = np.vdot(x2, y2)
        assert abs(a.norm2() - np.vdot(x2, x2).real) < 1e-13
        assert abs(a.inner(b) - ref) < 1e-13
        assert a.norm2() == a.norm2()  # deterministic


@pytest.mark.parametrize("dtype", DTYPES, ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("n", [2, 6, 14, 18])
def test_expectation_random_pauli_sums(cuda, dtype, n):
    x = rand_state(n, dtype, n)
    H = rand_observable(n, 40, seed=n)
    with StateVector(n, dtype) as a:
        a.upload(x)
        e = a.expectation(H)
        ref = oracle.expectation(x, H.matrix_free_terms())
        assert abs(e - ref) <= 1e-12 * max(1.0, abs(ref))
        assert a.expectation(H) == e


@pytest.mark.parametrize("n", [12, 24])
def test_ising_expectation(cuda, n):
    x = rand_state(n, np.complex128, 7)
    H = ising(n)
    assert len(H) == (n - 1) + n
    with StateVector(n, np.complex128) as a:
        a.upload(x)
        assert abs(a.expectation(H) - oracle.expectation(x, H.matrix_free_terms())) < 1e-11


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("n", [3, 11, 17])
def test_apply_observable(cuda, dtype, n):
    x = rand_state(n, dtype, 3)
    H = rand_observable(n, 25, seed=5)
    with StateVector(n, dtype) as a, StateVector(n, dtype) as b:
        a.upload(x)
        b.apply_observable(a, H)
        ref = oracle.observable_apply(x, H.matrix_free_terms())
        tol = 1e-12 if dtype == np.complex128 else 1e-5
        assert np.max(np.abs(b.download() - ref)) <= tol * max(1.0, np.max(np.abs(ref)))


def test_compare_mixed_precision_and_normalize(cuda):
    n = 15
    x = rand_state(n, np.complex128, 9)
    with StateVector(n, np.complex64) as a, StateVector(n, np.complex128) as b:
        xf = (1.01 * x).astype(np.complex64)
        a.upload(xf)
        b.upload(x)
        ip, mx = a.compare(b)
        ref_ip = np.vdot(xf.astype(np.complex128), x)
        assert abs(ip - ref_ip) < 1e-12
        assert abs(mx - np.max(np.abs(xf.astype(np.complex128) - x))) < 1e-15
        before = a.normalize()
        assert abs(before - np.vdot(xf.astype(np.complex128), xf.astype(np.complex128)).real) < 1e-12
        assert abs(a.norm2() - 1.0) < 1e-6
        y = a.download().astype(np.complex128)
        assert np.max(np.abs(y - x)) < 1e-6


def test_reduction_errors(cuda):
    with StateVector(3, np.float64) as a, StateVector(3, np.float64) as b:
        H = Observable(3).add(1.0, "XYZ")
        with pytest.raises(QsvError) as e:
            b.apply_observable(a, H)
        assert e.value.status == 6
        H2 = Observable(3)
        H2.paulis.append("XQZ")
        H2.coefs.append(1.0)
        with pytest.raises(QsvError) as e:
            a.expectation(H2)
        assert e.value.status == 1


def test_copy_and_observable_across_streams(cuda):
    """qsv_copy and qsv_apply_observable between two states whose streams
    differ (non-blocking torch streams) order themselves on the device: each
    is issued while a long circuit is still queued on the other state's
    stream, and the source is overwritten right after the copy."""
    import torch

    from qclab_b200 import workloads as W
    n = 20
    recs = W.brick(n, 60, seed=5).gate_records(np.complex128)
    more = W.brick(n, 20, seed=6).gate_records(np.complex128)
    x = rand_state(n, np.complex128, 9)
    want = oracle.apply(x.copy(), recs)
    H = ising(n)
    want_h = oracle.observable_apply(want, H.matrix_free_terms())
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
    with StateVector(n, np.complex128) as src, StateVector(n, np.complex128) as dst, \
            StateVector(n, np.complex128) as hdst:
        src.set_stream(sa.cuda_stream)
        dst.set_stream(sb.cuda_stream)
        hdst.set_stream(sb.cuda_stream)
        src.upload(x)
        src.apply(recs)            # queued on src's stream
        dst.copy_from(src)         # on dst's stream, after src's queue
        hdst.apply_observable(src, H)  # on src's stream, hdst's stream waits for it
        src.apply(more)            # src's stream waits for the copy's read
        assert np.array_equal(dst.download(), want)
        assert np.max(np.abs(hdst.download() - want_h)) < 1e-12
    torch.cuda.synchronize()

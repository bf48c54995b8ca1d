"""Device-resident state vectors and the record-level apply entry points."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .util import Op, as_op


def to_records(recs) -> np.ndarray:
    """List of record tuples -> contiguous GATE_DTYPE array."""
    if isinstance(recs, np.ndarray) and recs.dtype == L.GATE_DTYPE:
        return np.ascontiguousarray(recs)
    return np.array(list(recs), dtype=L.GATE_DTYPE)


class StateVector:
    """A 2^n-amplitude state in GPU memory (owns a ``qsv_state``).

    The element type is one of complex64, complex128, float32, float64 (the
    QCLAB++ template parameter T).  Created as |0...0>."""

    def __init__(self, nbQubits: int, dtype=np.complex128, *, _handle=None):
        self._lib = L.load()
        self.nbQubits = int(nbQubits)
        self.numpy_dtype = np.dtype(dtype)
        if self.numpy_dtype not in L.DTYPE_OF_NUMPY:
            raise TypeError(f"unsupported dtype {dtype}")
        self.qsv_dtype = L.DTYPE_OF_NUMPY[self.numpy_dtype]
        if _handle is not None:
            self._h = _handle
        else:
            h = C.c_void_p()
            L.check(self._lib.qsv_create(self.nbQubits, self.qsv_dtype, C.byref(h)), "qsv_create")
            self._h = h

    @classmethod
    def wrap(cls, device_ptr: int, nbQubits: int, dtype=np.complex128) -> "StateVector":
        """Non-owning view of caller-owned device memory (simulate_device(T*))."""
        lib = L.load()
        dt = np.dtype(dtype)
        h = C.c_void_p()
        L.check(lib.qsv_wrap(int(nbQubits), L.DTYPE_OF_NUMPY[dt], C.c_void_p(device_ptr),
                             C.byref(h)), "qsv_wrap")
        return cls(nbQubits, dt, _handle=h)

    @property
    def handle(self):
        return self._h

    @property
    def nbytes(self) -> int:
        return (1 << self.nbQubits) * self.numpy_dtype.itemsize

    @property
    def dtype(self):
        return self.numpy_dtype

    def device_ptr(self) -> int:
        p = C.c_void_p()
        L.check(self._lib.qsv_info(self._h, None, None, C.byref(p)), "qsv_info")
        return p.value

    def set_stream(self, stream_handle: int) -> None:
        L.check(self._lib.qsv_set_stream(self._h, C.c_void_p(stream_handle)), "qsv_set_stream")

    def upload(self, host: np.ndarray) -> None:
        host = np.ascontiguousarray(host, dtype=self.numpy_dtype)
        if host.size != 1 << self.nbQubits:
            raise ValueError("host vector size does not match the state")
        L.check(self._lib.qsv_upload(self._h, C.c_void_p(host.ctypes.data), host.nbytes),
                "qsv_upload")

    def upload_ptr(self, host_ptr: int, nbytes: int) -> None:
        L.check(self._lib.qsv_upload(self._h, C.c_void_p(host_ptr), nbytes), "qsv_upload")

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(1 << self.nbQubits, dtype=self.numpy_dtype)
        L.check(self._lib.qsv_download(self._h, C.c_void_p(out.ctypes.data), out.nbytes),
                "qsv_download")
        return out

    def download_ptr(self, host_ptr: int, nbytes: int) -> None:
        L.check(self._lib.qsv_download(self._h, C.c_void_p(host_ptr), nbytes), "qsv_download")

    def set_basis(self, index: int) -> None:
        L.check(self._lib.qsv_set_basis(self._h, int(index)), "qsv_set_basis")

    def copy_from(self, other: "StateVector") -> None:
        L.check(self._lib.qsv_copy(self._h, other._h), "qsv_copy")

    def chunks(self, chunk_qubits: int = 26):
        """Yields the state's elements as host arrays of 2^chunk_qubits
        elements in index order (each downloaded through a non-owning view
        of that part of the device array; one chunk of host memory at a
        time)."""
        self.synchronize()
        k = min(chunk_qubits, self.nbQubits)
        step = (1 << k) * self.numpy_dtype.itemsize
        base = self.device_ptr()
        for i in range(1 << (self.nbQubits - k)):
            view = StateVector.wrap(base + i * step, k, self.numpy_dtype)
            try:
                yield view.download()
            finally:
                view.close()

    def summary(self, idx, blocks: int = 256) -> dict:
        """``util.state_summary`` of this state: SHA-256 of its bytes, FP64
        norm^2, the amplitudes at ``idx`` and per-block probabilities."""
        from .util import state_summary
        return state_summary(self.chunks(), self.nbQubits, idx, blocks)

    def synchronize(self) -> None:
        L.check(self._lib.qsv_synchronize(self._h), "qsv_synchronize")

    def apply(self, records, op=Op.NoTrans, offset: int = 0, fused: bool = False,
              opts: L.FuseOpts | None = None) -> None:
        recs = to_records(records)
        opc = as_op(op).value.encode()
        ptr = C.c_void_p(recs.ctypes.data) if len(recs) else None
        if fused:
            L.check(self._lib.qsv_apply_fused(self._h, ptr, len(recs), opc, int(offset),
                                              C.byref(opts) if opts is not None else None),
                    "qsv_apply_fused")
        else:
            L.check(self._lib.qsv_apply(self._h, ptr, len(recs), opc, int(offset)), "qsv_apply")

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            L.check(self._lib.qsv_destroy(self._h), "qsv_destroy")
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def apply_records(recs, op, nbQubits: int, vector, offset: int = 0, fused: bool = False):
    """Applies gate records to a host numpy vector (in place) or a StateVector."""
    op = as_op(op)
    if isinstance(vector, StateVector):
        if vector.nbQubits != nbQubits:
            raise ValueError("nbQubits does not match the state")
        vector.apply(recs, op, offset, fused)
        return vector
    if not isinstance(vector, np.ndarray) or not vector.flags.c_contiguous:
        raise TypeError("vector must be a contiguous numpy array or a StateVector")
    if vector.dtype not in L.DTYPE_OF_NUMPY:
        raise TypeError(f"unsupported dtype {vector.dtype}")
    if vector.size != 1 << nbQubits:
        raise ValueError(f"vector of {vector.size} elements for {nbQubits} qubits")
    lib = L.load()
    r = to_records(recs)
    ptr = C.c_void_p(r.ctypes.data) if len(r) else None
    L.check(lib.qsv_apply_host(nbQubits, L.DTYPE_OF_NUMPY[vector.dtype],
                               C.c_void_p(vector.ctypes.data), ptr, len(r),
                               op.value.encode(), int(offset), 1 if fused else 0),
            "qsv_apply_host")
    return vector


def launch_count() -> int:
    """Kernel launches issued by the library on this thread."""
    return int(L.load().qsv_launch_count())


def tma_launch_count() -> int:
    """Stage launches on this thread whose tiles moved by TMA."""
    return int(L.load().qsv_tma_launch_count())


def _obs_args(obs):
    from .observable import Observable
    if not isinstance(obs, Observable):
        raise TypeError("expected an Observable")
    return obs.c_args()


def _norm2(self) -> float:
    out = C.c_double()
    L.check(self._lib.qsv_norm2(self._h, C.byref(out)), "qsv_norm2")
    return out.value


def _inner(self, other: "StateVector") -> complex:
    """<self|other> in FP64."""
    out = (C.c_double * 2)()
    L.check(self._lib.qsv_inner(self._h, other._h, out), "qsv_inner")
    return complex(out[0], out[1])


def _expectation(self, obs) -> float:
    """<psi|H|psi> in FP64."""
    buf, coefs, nt = _obs_args(obs)
    if obs.nbQubits != self.nbQubits:
        raise ValueError("observable size does not match the state")
    out = C.c_double()
    L.check(self._lib.qsv_expectation(self._h, buf, coefs, nt, C.byref(out)), "qsv_expectation")
    return out.value


def _apply_observable(self, src: "StateVector", obs) -> None:
    """self = H src."""
    buf, coefs, nt = _obs_args(obs)
    L.check(self._lib.qsv_apply_observable(self._h, src._h, buf, coefs, nt),
            "qsv_apply_observable")


def _compare(self, other: "StateVector"):
    """(<self|other>, max_j |self_j - other_j|) in FP64; dtypes may differ."""
    out = (C.c_double * 3)()
    L.check(self._lib.qsv_compare(self._h, other._h, out), "qsv_compare")
    return complex(out[0], out[1]), out[2]


def _normalize(self) -> float:
    """Scales the state to unit norm (norm in FP64); returns <psi|psi> before."""
    out = C.c_double()
    L.check(self._lib.qsv_normalize(self._h, C.byref(out)), "qsv_normalize")
    return out.value


StateVector.normalize = _normalize
StateVector.compare = _compare
StateVector.norm2 = _norm2
StateVector.inner = _inner
StateVector.expectation = _expectation
StateVector.apply_observable = _apply_observable

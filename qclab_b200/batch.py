"""Batched variational sweeps (new: QCLAB++ runs one circuit at a time).

``Batch`` packs many independent circuits -- each with its own qubit count,
gate list and Pauli-sum observable -- into one plan on the device.  One
persistent kernel launch (``qsv_batch_run``, optionally replayed from a
captured CUDA graph) then gives every circuit's energy <0|U^+ H U|0> and its
full adjoint gradient.  ``autotune`` picks the tile shape and the CTAs per
SM for a batch by timing the candidates on the device.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import time
from pathlib import Path

import numpy as np

from . import _lib as L
from .state import to_records


def _circuit_args(circuit, dtype):
    """(nbQubits, records with numbered params, nParams) of one circuit."""
    if isinstance(circuit, tuple):
        n, recs, nparams = circuit
        return int(n), to_records(recs), int(nparams)
    recs = circuit.gate_records(dtype, number_params=True)
    return circuit.nbQubits(), recs, circuit.nbParameters()


class Batch:
    """Energies and adjoint gradients of many circuits in one launch.

    ``circuits``: QCircuit objects (every variable rotation is a parameter,
    numbered in circuit order) or ``(nbQubits, records, nParams)`` tuples.
    ``observables``: one Observable per circuit.  The input state of every
    circuit is |0...0>."""

    def __init__(self, circuits, observables, dtype=np.complex64, *, tile_bits: int = 0,
                 low_bits: int = 0, ctas_per_sm: int = 0):
        self._lib = L.load()
        self.dtype = np.dtype(dtype)
        if self.dtype not in (np.dtype(np.complex64), np.dtype(np.complex128)):
            raise TypeError("batched sweeps need complex64 or complex128")
        circuits = list(circuits)
        observables = list(observables)
        if len(circuits) != len(observables):
            raise ValueError("one observable per circuit")
        args = [_circuit_args(c, self.dtype) for c in circuits]
        self.nbQubits = np.array([a[0] for a in args], dtype=np.int32)
        self.nParams = np.array([a[2] for a in args], dtype=np.int32)
        gates = [a[1] for a in args]
        self._gates = (np.concatenate(gates) if sum(len(g) for g in gates)
                       else np.zeros(1, dtype=L.GATE_DTYPE))
        self._gate_off = np.zeros(len(args) + 1, dtype=np.uint64)
        self._gate_off[1:] = np.cumsum([len(g) for g in gates])
        for H, n in zip(observables, self.nbQubits):
            if H.nbQubits != n:
                raise ValueError("observable and circuit qubit counts differ")
        self._paulis = "".join("".join(H.paulis) for H in observables).encode()
        self._coefs = np.array([c for H in observables for c in H.coefs] or [0.0], dtype=np.float64)
        self._term_off = np.zeros(len(args) + 1, dtype=np.uint64)
        self._term_off[1:] = np.cumsum([len(H) for H in observables])
        self._grad_off = np.zeros(len(args) + 1, dtype=np.int64)
        self._grad_off[1:] = np.cumsum(self.nParams)
        opts = L.BatchOpts(tile_bits, low_bits, ctas_per_sm)
        h = C.c_void_p()
        L.check(self._lib.qsv_batch_create(
            L.DTYPE_OF_NUMPY[self.dtype], len(args), self.nbQubits.ctypes.data,
            C.c_void_p(self._gates.ctypes.data), self._gate_off.ctypes.data, self._paulis,
            self._coefs.ctypes.data, self._term_off.ctypes.data, self.nParams.ctypes.data,
            C.byref(opts), C.byref(h)), "qsv_batch_create")
        self._h = h

    def __len__(self) -> int:
        return len(self.nbQubits)

    @property
    def handle(self):
        if self._h is None:
            raise ValueError("batch destroyed")
        return self._h

    def run(self, stream: int | None = None, graph: bool = True) -> None:
        """One launch of the whole batch on ``stream`` (a cudaStream_t
        address; None = the default stream)."""
        L.check(self._lib.qsv_batch_run(self.handle, C.c_void_p(stream or 0), int(graph)),
                "qsv_batch_run")

    def results(self, stream: int | None = None):
        """(energies[nCircuits], [gradient of circuit c]) after ``run``."""
        e = np.zeros(len(self), dtype=np.float64)
        g = np.zeros(max(1, int(self._grad_off[-1])), dtype=np.float64)
        L.check(self._lib.qsv_batch_results(self.handle, C.c_void_p(stream or 0), e.ctypes.data,
                                            g.ctypes.data), "qsv_batch_results")
        grads = [g[self._grad_off[c]:self._grad_off[c + 1]].copy() for c in range(len(self))]
        return e, grads

    def info(self) -> dict:
        b, t, m = C.c_int(), C.c_int(), C.c_int()
        w = C.c_size_t()
        L.check(self._lib.qsv_batch_info(self.handle, C.byref(b), C.byref(t), C.byref(m),
                                         C.byref(w)), "qsv_batch_info")
        return {"blocks": b.value, "threads": t.value, "tile_bits": m.value,
                "workspace_bytes": w.value}

    def work(self) -> dict:
        """Work of one launch from the plan (``qsv_batch_work``): global tile
        traffic in bytes and gate x amplitude updates."""
        gb, au = C.c_double(), C.c_double()
        L.check(self._lib.qsv_batch_work(self.handle, C.byref(gb), C.byref(au)), "qsv_batch_work")
        return {"global_bytes": gb.value, "amplitude_updates": au.value}

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            self._lib.qsv_batch_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---- autotuner -----------------------------------------------------------------

def candidates(dtype) -> list[dict]:
    """Tile shapes the batched kernel accepts: 2^m-amplitude tiles with m in
    [10, 12] (complex<float>) or [9, 11] (complex<double>), low bits in
    {2, 3}, and 1, 2, 4 or occupancy-limited CTAs per SM."""
    ms = (10, 11, 12) if np.dtype(dtype) == np.dtype(np.complex64) else (9, 10, 11)
    out = []
    for m in ms:
        for low in (2, 3):
            for cps in (0, 1, 2, 4):
                out.append({"tile_bits": m, "low_bits": low, "ctas_per_sm": cps})
    return out


def _signature(circuits, observables, dtype) -> str:
    args = [_circuit_args(c, np.dtype(dtype)) for c in circuits]
    hist = np.bincount([a[0] for a in args], minlength=31).tolist()
    gates = int(sum(len(a[1]) for a in args))
    terms = int(sum(len(H) for H in observables))
    return f"{np.dtype(dtype).name}:{len(args)}:{gates}:{terms}:{hist}"


def default_cache_path() -> Path:
    return Path(os.environ.get("QCLAB_B200_TUNE_CACHE",
                               Path.home() / ".cache" / "qclab_b200" / "batch_tune.json"))


def autotune(circuits, observables, dtype=np.complex64, *, cands=None, repeats: int = 3,
             cache: Path | str | None = None, timer=None):
    """Times every candidate tile shape on the batch and returns
    (best option dict, {str(option): seconds}).  ``timer(batch)`` returns the
    seconds of one launch (default: host time around run + synchronize, the
    minimum over ``repeats`` after one warm-up).  Results are cached per
    batch signature in ``cache`` (a JSON file)."""
    circuits = list(circuits)
    observables = list(observables)
    cache = Path(cache) if cache is not None else default_cache_path()
    key = _signature(circuits, observables, dtype)
    if cache.exists():
        try:
            hit = json.loads(cache.read_text()).get(key)
            if hit:
                return hit["best"], hit["times"]
        except (OSError, ValueError):
            pass

    def host_timer(b: Batch) -> float:
        b.run(graph=True)
        b.results()
        best = float("inf")
        for _ in range(repeats):
            t0 = time.perf_counter()
            b.run(graph=True)
            b.results()
            best = min(best, time.perf_counter() - t0)
        return best

    timer = timer or host_timer
    times: dict[str, float] = {}
    best, best_t = None, float("inf")
    for opt in (cands or candidates(dtype)):
        try:
            with Batch(circuits, observables, dtype, **opt) as b:
                t = timer(b)
        except L.QsvError:
            continue  # shape not accepted for this batch
        times[json.dumps(opt, sort_keys=True)] = t
        if t < best_t:
            best, best_t = opt, t
    if best is None:
        raise RuntimeError("no candidate tile shape accepted the batch")
    try:
        cache.parent.mkdir(parents=True, exist_ok=True)
        data = json.loads(cache.read_text()) if cache.exists() else {}
        data[key] = {"best": best, "times": times}
        cache.write_text(json.dumps(data, indent=1))
    except (OSError, ValueError):
        pass
    return best, times

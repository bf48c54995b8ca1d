"""Gradients of expectation values with respect to the trainable angles.

* ``adjoint_gradient``: the reverse-mode sweep of the C ABI
  (``qsv_adjoint_gradient``): one forward and one backward fused sweep.
* ``parameter_shift_gradient`` / ``finite_difference_gradient``: the GPU
  baselines the adjoint is checked against -- two full simulations per
  angle (theta +- pi/2 for exp(-i theta P / 2) rotations, theta +- h for
  central differences), each followed by an FP64 expectation value.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L
from .gates import PARAMETRIC_KINDS
from .state import StateVector, to_records

SHIFTABLE = {L.ROTATION_X, L.ROTATION_Y, L.ROTATION_Z, L.ROTATION_XX, L.ROTATION_YY,
             L.ROTATION_ZZ}


def adjoint_gradient(state: StateVector, records, observable, nparams: int | None = None):
    """(E, dE/dtheta) for gate records whose ``param`` fields number the
    trainable angles.  ``state`` holds the input state and is restored."""
    recs = to_records(records)
    if nparams is None:
        nparams = int(recs["param"].max()) + 1 if len(recs) else 0
    buf, coefs, nt = observable.c_args()
    grads = (C.c_double * max(1, nparams))()
    e = C.c_double()
    L.check(L.load().qsv_adjoint_gradient(state.handle, C.c_void_p(recs.ctypes.data) if len(recs) else None,
                                          len(recs), buf, coefs, nt, grads, nparams, C.byref(e)),
            "qsv_adjoint_gradient")
    return e.value, np.array(grads[:nparams])


def _shifted(recs: np.ndarray, i: int, delta: float) -> np.ndarray:
    """Records with gate i's angle theta -> theta + delta (cos/sin of the
    half angle for rotations, of the angle for phase gates)."""
    out = recs.copy()
    r = out[i]
    k = int(r["kind"])
    half = k not in (L.PHASE, L.CPHASE)
    d = delta / 2 if half else delta
    c, s = float(r["cos"]), float(r["sin"])
    out[i]["cos"] = c * math.cos(d) - s * math.sin(d)
    out[i]["sin"] = s * math.cos(d) + c * math.sin(d)
    return out


def _energy(state: StateVector, init: StateVector, recs, observable, fused=True) -> float:
    state.copy_from(init)
    state.apply(recs, "N", 0, fused=fused)
    return state.expectation(observable)


def parameter_shift_gradient(init: StateVector, records, observable, nparams: int | None = None,
                             params=None):
    """dE/dtheta by the parameter-shift rule (E(theta+pi/2) - E(theta-pi/2))/2
    for every rotation gate carrying a param (all on the GPU)."""
    recs = to_records(records)
    if nparams is None:
        nparams = int(recs["param"].max()) + 1
    grads = np.zeros(nparams)
    work = StateVector(init.nbQubits, init.numpy_dtype)
    try:
        for i in range(len(recs)):
            p = int(recs[i]["param"])
            if p < 0 or (params is not None and p not in params):
                continue
            if int(recs[i]["kind"]) not in SHIFTABLE:
                raise ValueError("parameter shift needs exp(-i theta P/2) rotations")
            ep = _energy(work, init, _shifted(recs, i, math.pi / 2), observable)
            em = _energy(work, init, _shifted(recs, i, -math.pi / 2), observable)
            grads[p] += 0.5 * (ep - em)
    finally:
        work.close()
    return grads


def finite_difference_gradient(init: StateVector, records, observable, h: float = 1e-5,
                               nparams: int | None = None, params=None):
    """Central differences (E(theta+h) - E(theta-h)) / 2h on the GPU."""
    recs = to_records(records)
    if nparams is None:
        nparams = int(recs["param"].max()) + 1
    grads = np.zeros(nparams)
    work = StateVector(init.nbQubits, init.numpy_dtype)
    try:
        for i in range(len(recs)):
            p = int(recs[i]["param"])
            if p < 0 or (params is not None and p not in params):
                continue
            ep = _energy(work, init, _shifted(recs, i, h), observable)
            em = _energy(work, init, _shifted(recs, i, -h), observable)
            grads[p] += (ep - em) / (2 * h)
    finally:
        work.close()
    return grads

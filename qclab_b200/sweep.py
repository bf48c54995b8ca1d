"""Times fused sweeps from the command line.

    python -m qclab_b200.sweep --qubits 26 --depth 40 --dtype c64 --engine 3

Runs a seeded random brick circuit (``workloads.brick``) through
``qsv_apply_fused`` on the current GPU, ``--repeat`` times after one warm-up
sweep, and prints one JSON line: gates, stages and tensor-core passes of the
plan (``qsv_plan_passes``), the wall time of each sweep (host planning
included, stream synchronised) and gates/s.  ``--engine`` is
``qsv_fuse_opts.engine``: 0 default (FP64 MMA for complex<double>, mma.sync
TF32 for complex<float>), 1 sparse register passes, 2 FP64 MMA for both,
3 tcgen05 TF32 for complex<float>.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import _lib as L
from . import workloads as W
from .state import StateVector

DTYPES = {"c128": (np.complex128, L.C128), "c64": (np.complex64, L.C64)}


def main(argv=None) -> dict:
    p = argparse.ArgumentParser(prog="python -m qclab_b200.sweep")
    p.add_argument("--qubits", type=int, default=26)
    p.add_argument("--depth", type=int, default=40)
    p.add_argument("--seed", type=int, default=3)
    p.add_argument("--dtype", choices=sorted(DTYPES), default="c128")
    p.add_argument("--engine", type=int, default=0)
    p.add_argument("--tile-bits", type=int, default=0)
    p.add_argument("--repeat", type=int, default=2)
    a = p.parse_args(argv)
    dt, code = DTYPES[a.dtype]
    recs = W.brick(a.qubits, a.depth, seed=a.seed).gate_records(dt)
    opts = L.FuseOpts(engine=a.engine, tile_bits=a.tile_bits)
    lib = L.load()
    arr, ptr, cnt = L.gate_array(recs)
    ns, npas, nops = C.c_int(), C.c_int(), C.c_int()
    L.check(lib.qsv_plan_passes(a.qubits, code, ptr, cnt, b"N", 0, C.byref(opts), C.byref(ns),
                                C.byref(npas), C.byref(nops)), "qsv_plan_passes")
    out = {"qubits": a.qubits, "depth": a.depth, "dtype": a.dtype, "engine": a.engine,
           "gates": int(cnt), "stages": ns.value, "passes": npas.value}
    ms = []
    with StateVector(a.qubits, dt) as s:
        s.apply(recs, "N", 0, fused=True, opts=opts)
        s.synchronize()
        for _ in range(a.repeat):
            s.set_basis(0)
            s.synchronize()
            t = time.perf_counter()
            s.apply(recs, "N", 0, fused=True, opts=opts)
            s.synchronize()
            ms.append((time.perf_counter() - t) * 1e3)
    out["ms"] = [round(v, 3) for v in ms]
    out["gates_per_s"] = cnt / (min(ms) / 1e3) if ms else None
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()

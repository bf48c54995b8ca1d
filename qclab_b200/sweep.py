"""Times fused sweeps from the command line.

    python -m qclab_b200.sweep --qubits 26 --depth 40 --dtype c64 --engine 3
    python -m qclab_b200.sweep --workload adjoint --qubits 22 --depth 12
    python -m qclab_b200.sweep --workload batch --circuits 512

brick (default): a seeded random brick circuit (``workloads.brick``) through
``qsv_apply_fused`` on the current GPU, ``--repeat`` times after one warm-up
sweep; prints one JSON line with the gates, stages and tensor-core passes of
the plan (``qsv_plan_passes``), the wall time of each sweep (host planning
included, stream synchronised) and gates/s.  ``--engine`` is
``qsv_fuse_opts.engine``: 0 default (5 for complex<float>, 2 for
complex<double>), 1 sparse register passes, 2 FP64 MMA dense passes, 3
tcgen05 TF32 for complex<float>, 4 mma.sync TF32 for complex<float>, 5
gate-specialised register passes (``--reg-bits`` 4, or 5 for
complex<float>).

adjoint: energy and full gradient (``qsv_adjoint_gradient``) of the
hardware-efficient ansatz ``workloads.hea(qubits, depth)`` for
H = sum Z_i Z_i+1 + 0.5 sum X_i; prints the time per gradient.

batch: ``--circuits`` ansatz circuits of 8..18 qubits and 4..16 layers in one
persistent launch (``qsv_batch_run``, default tile shape); prints the time
per batch.

kernels: one launch of every reference-exact per-gate kernel shape (pair,
controlled pair and quad at register and lane bits, half-state and
quarter-state phase scales, SWAP/iSWAP) and of the FP64 reductions (norm,
inner product, expectation of the Ising H, state comparison) on a
``--qubits`` complex<double> state; prints each one's best time over
``--repeat`` launches and its achieved GB/s from the bytes the reference's
loop touches (apply.hpp:259-371: 2 N s for pair and quad gates, N s for
controlled pairs, half scales and swaps, N s / 2 for controlled scales).
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


def main(argv=None, keep_state: bool = False) -> dict:
    """Runs the command; with ``keep_state`` the returned dict also holds
    the last sweep's final state (``state``, a host array; not printed)."""
    p = argparse.ArgumentParser(prog="python -m qclab_b200.sweep")
    p.add_argument("--qubits", type=int, default=26)
    p.add_argument("--depth", type=int, default=40)
    p.add_argument("--seed", type=int, default=3)
    p.add_argument("--dtype", choices=sorted(DTYPES), default="c128")
    p.add_argument("--engine", type=int, default=0)
    p.add_argument("--tile-bits", type=int, default=0)
    p.add_argument("--low-bits", type=int, default=0)
    p.add_argument("--reg-bits", type=int, default=0)
    p.add_argument("--ctas-per-sm", type=int, default=0)
    p.add_argument("--tile-copy", type=int, default=0,
                   help="engine 5 tile staging: 0 = TMA where possible, 1 = cp.async")
    p.add_argument("--repeat", type=int, default=2)
    p.add_argument("--workload", choices=["brick", "adjoint", "batch", "kernels"],
                   default="brick")
    p.add_argument("--circuits", type=int, default=512)
    a = p.parse_args(argv)
    if a.workload == "adjoint":
        return _adjoint(a)
    if a.workload == "batch":
        return _batch(a)
    if a.workload == "kernels":
        return _kernels(a)
    dt, code = DTYPES[a.dtype]
    recs = W.brick(a.qubits, a.depth, seed=a.seed).gate_records(dt)
    opts = L.FuseOpts(engine=a.engine, tile_bits=a.tile_bits, low_bits=a.low_bits,
                      reg_bits=a.reg_bits, ctas_per_sm=a.ctas_per_sm, tile_copy=a.tile_copy)
    lib = L.load()
    arr, ptr, cnt = L.gate_array(recs)
    ns, npas, nops = C.c_int(), C.c_int(), C.c_int()
    L.check(lib.qsv_plan_passes(a.qubits, code, ptr, cnt, b"N", 0, C.byref(opts), C.byref(ns),
                                C.byref(npas), C.byref(nops)), "qsv_plan_passes")
    out = {"qubits": a.qubits, "depth": a.depth, "dtype": a.dtype, "engine": a.engine,
           "tile_copy": a.tile_copy, "gates": int(cnt), "stages": ns.value,
           "passes": npas.value}
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
        final = s.download() if keep_state else None
    out["ms"] = [round(v, 3) for v in ms]
    out["gates_per_s"] = cnt / (min(ms) / 1e3) if ms else None
    print(json.dumps(out), flush=True)
    if keep_state:
        out["state"] = final
    return out


def _timed(fn, repeat):
    fn()
    ms = []
    for _ in range(repeat):
        t = time.perf_counter()
        fn()
        ms.append((time.perf_counter() - t) * 1e3)
    return [round(v, 3) for v in ms]


def _adjoint(a) -> dict:
    from .gradients import adjoint_gradient
    from .observable import ising
    dt, _ = DTYPES[a.dtype]
    recs = W.hea(a.qubits, a.depth, seed=a.seed).gate_records(dt, number_params=True)
    nparams = int(recs["param"].max()) + 1
    H = ising(a.qubits)
    out = {"workload": "adjoint", "qubits": a.qubits, "layers": a.depth, "dtype": a.dtype,
           "gates": len(recs), "params": nparams}
    with StateVector(a.qubits, dt) as s:
        res = {}

        def run():
            res["e"], res["g"] = adjoint_gradient(s, recs, H, nparams)
        out["ms"] = _timed(run, a.repeat)
        out["energy"] = res["e"]
    print(json.dumps(out), flush=True)
    return out


def _batch(a) -> dict:
    from .batch import Batch
    from .observable import ising
    dt, _ = DTYPES[a.dtype]
    rng = np.random.default_rng(a.seed)
    ns = rng.integers(8, 19, size=a.circuits)
    ls = rng.integers(4, 17, size=a.circuits)
    circs = [W.hea(int(n), int(l), seed=a.seed * 100003 + i) for i, (n, l) in enumerate(zip(ns, ls))]
    obs = [ising(int(n)) for n in ns]
    out = {"workload": "batch", "circuits": a.circuits, "dtype": a.dtype,
           "gates": int(sum(len(c.gate_records(dt)) for c in circs))}
    with Batch(circs, obs, dt, tile_bits=a.tile_bits, ctas_per_sm=a.ctas_per_sm) as b:
        out["launch_shape"] = b.info()

        def run():
            b.run()
            b.results()
        out["ms"] = _timed(run, a.repeat)
    print(json.dumps(out), flush=True)
    return out


def _kernels(a) -> dict:
    from . import gates as G
    from .circuit import QCircuit
    from .observable import ising
    n = a.qubits
    N = 1 << n
    s16 = N * 16
    hi, lo = 0, n - 1  # qubit 0 is the top index bit (register kernels), n-1 bit 0 (lanes)
    cases = [
        ("k_pair_reg  Hadamard(top)", [G.Hadamard(hi)], 2 * s16),
        ("k_pair_lane Hadamard(bit 0)", [G.Hadamard(lo)], 2 * s16),
        ("k_pair_reg  CNOT(top)", [G.CNOT(hi, hi + 1)], s16),
        ("k_pair_lane CNOT(bit 0)", [G.CNOT(lo - 1, lo)], s16),
        ("k_scale     PauliZ (half)", [G.PauliZ(3)], s16),
        ("k_scale     CZ (quarter)", [G.CZ(2, 3)], s16 // 2),
        ("k_quad_reg2 RotationXX(top)", [G.RotationXX(hi, hi + 1, 0.3)], 2 * s16),
        ("k_quad_reg1 RotationXX(reg, lane)", [G.RotationXX(n - 6, lo, 0.3)], 2 * s16),
        ("k_quad_lane RotationXX(lanes)", [G.RotationXX(lo - 2, lo, 0.3)], 2 * s16),
        ("k_swap_reg2 SWAP(top)", [G.SWAP(hi, hi + 1)], s16),
        ("k_swap_reg1 iSWAP(reg, lane)", [G.iSWAP(n - 6, lo)], s16),
        ("k_swap_lane SWAP(lanes)", [G.SWAP(lo - 2, lo)], s16),
    ]
    out = {"workload": "kernels", "qubits": n, "dtype": "c128", "kernels": {}}
    H = ising(n)

    def best(fn):
        fn()
        st.synchronize()
        ms = []
        for _ in range(max(1, a.repeat)):
            t = time.perf_counter()
            fn()
            st.synchronize()
            ms.append((time.perf_counter() - t) * 1e3)
        return min(ms)

    with StateVector(n, np.complex128) as st, StateVector(n, np.complex128) as other:
        st.set_basis(0)
        for name, gl, nbytes in cases:
            c = QCircuit(n)
            for g in gl:
                c.push_back(g)
            recs = c.gate_records(np.complex128)
            ms = best(lambda: st.apply(recs, "N", 0, fused=False))
            out["kernels"][name] = {"ms": round(ms, 4), "gbs": nbytes / (ms / 1e3) / 1e9}
        reds = [("k_norm2 (norm)", lambda: st.norm2(), s16),
                ("k_inner (inner product)", lambda: st.inner(other), 2 * s16),
                ("k_compare (state comparison)", lambda: st.compare(other), 2 * s16),
                ("k_expect* (Ising H, tiled groups)", lambda: st.expectation(H), None),
                ("k_observable* (Ising H psi, tiled groups)", lambda: other.apply_observable(st, H),
                 None)]
        for name, fn, nbytes in reds:
            ms = best(fn)
            out["kernels"][name] = {"ms": round(ms, 4),
                                    "gbs": (nbytes / (ms / 1e3) / 1e9) if nbytes else None}
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()

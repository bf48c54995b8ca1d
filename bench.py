"""Benchmark of the B200 state-vector backend (one JSON line on rank 0).

Workload (the headline configuration): a seeded random brick circuit on
30 qubits, complex<double> (16 GiB state), depth 200 -- per layer one gate
from {Hadamard, RotationX, RotationY, RotationZ} on every qubit, then CNOT
or CZ on alternating neighbour pairs: 8,900 gates.  One step = reset to
|0...0> + the whole circuit through the fused sweep, state resident in HBM.
The state (16 GiB) is far larger than L2 (126 MB), so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun, one rank per GPU) every rank simulates its own
circuit (replicas, weak scaling; the path has no exchange step); time is the
max over ranks.  ``--impl reference`` times QCLAB++'s own CPU simulate
(compiled from its sources into oracle/_ref) on the host cores instead.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "gates/s & HBM GB/s vs 8TB/s at 30q; adjoint grads/s vs param-shift @1e-9"
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--qubits", type=int, default=30)
    p.add_argument("--depth", type=int, default=200)
    p.add_argument("--seed", type=int, default=2024)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--unfused-gates", type=int, default=45)
    p.add_argument("--parity-layers", type=int, default=10)
    p.add_argument("--no-extras", action="store_true",
                   help="skip the adjoint (24q) and precision (32q) measurements")
    p.add_argument("--ps-params", type=int, default=0,
                   help="angles timed for the parameter-shift baseline (0 = all 576)")
    return p.parse_args()


def adjoint_extra(torch, stream, ps_params, fd_params=48, fd_h=1e-5):
    """Adjoint gradient on the 24-qubit hardware-efficient ansatz (12 layers of
    RotationY/RotationZ on every qubit + a CNOT ladder: 852 gates, 576
    angles), complex<double>, H = sum Z_i Z_{i+1} + 0.5 sum X_i, checked
    against the GPU parameter-shift gradient on every angle (`ps_params` = 0;
    a positive count times that many evenly spaced angles and extrapolates)
    and central finite differences (h = `fd_h`) on `fd_params` seeded angles."""
    from qclab_b200 import StateVector
    from qclab_b200 import workloads as W
    from qclab_b200.gradients import (adjoint_gradient, finite_difference_gradient,
                                      parameter_shift_gradient)
    from qclab_b200.observable import ising
    n = 24
    recs = W.hea(n, 12, seed=7).gate_records(np.complex128, number_params=True)
    nparams = int(recs["param"].max()) + 1
    H = ising(n)
    with StateVector(n, np.complex128) as s:
        s.set_stream(stream.cuda_stream)
        for _ in range(2):
            adjoint_gradient(s, recs, H)
        torch.cuda.synchronize()
        reps = 5
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            s.set_basis(0)
            e, g = adjoint_gradient(s, recs, H)
        b.record(stream)
        torch.cuda.synchronize()
        adj_ms = a.elapsed_time(b) / reps
        s.set_basis(0)
        subset = (set(range(nparams)) if ps_params <= 0
                  else set(range(0, nparams, max(1, nparams // ps_params))))
        parameter_shift_gradient(s, recs, H, params={0})  # warm-up
        torch.cuda.synchronize()
        a.record(stream)
        ps = parameter_shift_gradient(s, recs, H, params=subset)
        b.record(stream)
        torch.cuda.synchronize()
        ps_ms = a.elapsed_time(b) * nparams / len(subset)
        rng = np.random.default_rng(24)
        fd_set = set(int(v) for v in rng.choice(nparams, size=min(fd_params, nparams),
                                                replace=False))
        fd = finite_difference_gradient(s, recs, H, h=fd_h, params=fd_set)
    # the same gradient on a complex<float> state (FP64 reductions), against
    # the complex<double> one
    recs32 = W.hea(n, 12, seed=7).gate_records(np.complex64, number_params=True)
    with StateVector(n, np.complex64) as s32:
        s32.set_stream(stream.cuda_stream)
        for _ in range(2):
            adjoint_gradient(s32, recs32, H)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(reps):
            s32.set_basis(0)
            e32, g32 = adjoint_gradient(s32, recs32, H)
        b.record(stream)
        torch.cuda.synchronize()
        adj32_ms = a.elapsed_time(b) / reps
    err = float(max(abs(g[p] - ps[p]) for p in subset))
    fd_err = float(max(abs(g[p] - fd[p]) for p in fd_set))
    return {"workload": "hea24_12layers_c128_ising", "gates": len(recs), "params": nparams,
            "energy": e, "adjoint_ms": adj_ms, "grads_per_s": 1e3 / adj_ms,
            "param_shift_ms": ps_ms, "param_shift_params_timed": len(subset),
            "param_shift_extrapolated": len(subset) < nparams,
            "speedup_vs_param_shift": ps_ms / adj_ms,
            "max_abs_grad_diff_vs_param_shift": err,
            "central_fd": {"h": fd_h, "params": len(fd_set), "seed": 24,
                           "max_abs_grad_diff_vs_adjoint": fd_err},
            "max_abs_grad": float(np.max(np.abs(g))),
            "complex_float": {"adjoint_ms": adj32_ms,
                              "max_abs_grad_diff_vs_c128": float(np.max(np.abs(g32 - g))),
                              "energy_diff_vs_c128": abs(e32 - e)}}


def plan_counts(n, code, recs, opts=None):
    """(stages, register passes) of the fused plan qsv_apply_fused would run."""
    from qclab_b200 import _lib as L
    lib = L.load()
    st_, ps_, op_ = C.c_int(), C.c_int(), C.c_int()
    L.check(lib.qsv_plan_passes(n, code, C.c_void_p(recs.ctypes.data), len(recs), b"N", 0,
                                C.byref(opts) if opts is not None else None, C.byref(st_),
                                C.byref(ps_), C.byref(op_)), "qsv_plan_passes")
    return st_.value, ps_.value


def precision_extra(torch, stream, n=32, depth=100, seed=11):
    """Precision study: the brick generator at n qubits, depth `depth`, run in
    complex<float> and complex<double> (fused), compared in FP64.  Both runs
    take the circuit's gate parameters in double, so the difference is the
    state's precision (and the engine's arithmetic) alone.  Each
    complex<float> engine gets its HBM roofline (stages x one read + one
    write of the 32 GiB state over its time), and the plain unfused
    complex<double> path (qsv_apply) is timed on the circuit's first layer
    at the same size."""
    from qclab_b200 import StateVector
    from qclab_b200 import _lib as L
    from qclab_b200 import workloads as W
    from qclab_b200.observable import Observable
    circ = W.brick(n, depth, seed=seed)
    r128 = circ.gate_records(np.complex128)
    zz = Observable(n).add(1.0, {0: "Z", 1: "Z"})
    peak, peak_kind = peaks()
    out = {"workload": f"brick{n}_depth{depth}", "gates": len(r128)}

    def timed(fn):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1])

    with StateVector(n, np.complex128) as d, StateVector(n, np.complex64) as f:
        d.set_stream(stream.cuda_stream)
        f.set_stream(stream.cuda_stream)
        c128_ms = timed(lambda: d.apply(r128, "N", 0, fused=True))
        d_norm2 = d.norm2()
        zd = d.expectation(zz)
        engines = [("default (gate passes, 5 bits)", None),
                   ("gate passes, 4 bits", L.FuseOpts(engine=5, reg_bits=4)),
                   ("fp64_mma", L.FuseOpts(engine=2)),
                   ("tf32_mma_sync", L.FuseOpts(engine=4))]
        runs = {}
        for name, opts in engines:
            f.set_basis(0)
            f.apply(r128[:1], "N", 0, fused=True, opts=opts)  # loads the kernel
            f.set_basis(0)
            ms = timed(lambda: f.apply(r128, "N", 0, fused=True, opts=opts))
            ip, maxabs = f.compare(d)
            zf = f.expectation(zz)
            nf = f.norm2()
            stages, passes = plan_counts(n, L.C64, r128, opts)
            achieved = stages * 2 * (1 << n) * 8 / (ms / 1e3) / 1e9
            runs[name] = {"ms": ms, "gates_per_s": len(r128) / (ms / 1e3),
                          "infidelity": 1.0 - abs(ip) ** 2, "max_abs_error": maxabs,
                          "zz01_error": abs(zf - zd), "norm2_c64": nf,
                          "stages": stages, "passes": passes,
                          "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                                       "unit": "GB/s", "frac": achieved / peak,
                                       "peak_source": f"{peak_kind} hbm_gbs"}}
        # the plain unfused complex<double> path on the circuit's first layer
        layer = r128[:W.brick_layer_sizes(n, 1)[0]]
        d.set_basis(0)
        d.apply(layer[:1], "N", 0, fused=False)
        d.set_basis(0)
        u_ms = timed(lambda: d.apply(layer, "N", 0, fused=False))
        u_bytes = sum((2 if int(r["kind"]) in (L.HADAMARD, L.ROTATION_X, L.ROTATION_Y,
                                                L.ROTATION_Z) else 1 if int(r["kind"]) == L.CX
                       else 0.5) * (1 << n) * 16 for r in layer)
        unfused = {"gates": len(layer), "ms": u_ms, "gates_per_s": len(layer) / (u_ms / 1e3),
                   "hbm_gbs": u_bytes / (u_ms / 1e3) / 1e9, "path": "qsv_apply (bit-exact)"}
    best = runs["default (gate passes, 5 bits)"]
    out.update({"c64_ms": best["ms"], "c128_ms": c128_ms,
                "c64_gates_per_s": best["gates_per_s"],
                "c128_gates_per_s": len(r128) / (c128_ms / 1e3),
                "infidelity": best["infidelity"], "max_abs_error": best["max_abs_error"],
                "zz01_c128": zd, "zz01_error": best["zz01_error"],
                "norm2_c64": best["norm2_c64"], "norm2_c128": d_norm2,
                "roofline_c64": best["roofline"], "c64_engines": runs,
                "unfused_c128_first_layer": unfused,
                "c64_fused_vs_unfused_c128": best["gates_per_s"] / unfused["gates_per_s"],
                "note": "infidelity = 1 - |<psi32|psi64>|^2 of the states as computed, "
                        "without renormalisation; TF32 is opt-in (its accumulation truncates)"})
    return out


def batch_extra(torch, stream, ncirc=4096, seed=21, check=16, loop_sample=64):
    """Batched variational sweep: `ncirc` hardware-efficient circuits with
    qubit counts uniform in 8..18 and 4..16 layers (RotationY/RotationZ on
    every qubit + a CNOT ladder), complex<float> states with FP64
    reductions, H = sum Z_i Z_{i+1} + 0.5 sum X_i: the energy and full
    adjoint gradient of every circuit from one persistent, graph-captured
    launch whose tile shape the autotuner picks.  Checked on `check`
    circuits against the single-circuit complex<double> adjoint; the
    one-circuit-at-a-time GPU loop (qsv_adjoint_gradient, complex<float>) is
    timed on `loop_sample` circuits and scaled to the batch."""
    import tempfile
    from pathlib import Path
    from qclab_b200 import StateVector
    from qclab_b200 import workloads as W
    from qclab_b200.batch import Batch, autotune
    from qclab_b200.gradients import adjoint_gradient
    from qclab_b200.observable import ising
    peak, peak_kind = peaks()
    rng = np.random.default_rng(seed)
    ns = rng.integers(8, 19, size=ncirc)
    ls = rng.integers(4, 17, size=ncirc)
    circs = [W.hea(int(n), int(l), seed=seed * 100003 + i) for i, (n, l) in enumerate(zip(ns, ls))]
    obs = [ising(int(n)) for n in ns]
    s = stream.cuda_stream
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def ev_timer(b, reps=3):
        b.run(s, graph=True)
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(reps):
            b.run(s, graph=True)
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / reps / 1e3

    # the persistent kernel fits at most two CTAs per SM: 0 (the occupancy
    # limit) and 1 are the distinct choices
    cands = [{"tile_bits": m, "low_bits": 2, "ctas_per_sm": c} for m in (10, 11, 12) for c in (0, 1)]
    t0 = time.perf_counter()
    best, times = autotune(circs, obs, np.complex64, cands=cands, timer=ev_timer,
                           cache=Path(tempfile.mkdtemp()) / "tune.json")
    tune_s = time.perf_counter() - t0
    with Batch(circs, obs, np.complex64, **best) as b:
        sec = ev_timer(b, reps=5)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.run(s, graph=True)
        e, g = b.results(s)
        e2e = time.perf_counter() - t0
        info = b.info()
        work = b.work()
    idx = list(range(0, ncirc, max(1, ncirc // check)))[:check]
    err_e = err_g = 0.0
    for i in idx:
        with StateVector(circs[i].nbQubits(), np.complex128) as st:
            e1, g1 = adjoint_gradient(st, circs[i].gate_records(np.complex128, number_params=True),
                                      obs[i])
        err_e = max(err_e, abs(e[i] - e1))
        err_g = max(err_g, float(np.max(np.abs(g[i] - g1))))
    loop_idx = list(range(0, ncirc, max(1, ncirc // loop_sample)))[:loop_sample]
    recs = [circs[i].gate_records(np.complex64, number_params=True) for i in loop_idx]

    def loop_once():
        for i, r in zip(loop_idx, recs):
            with StateVector(circs[i].nbQubits(), np.complex64) as st:
                adjoint_gradient(st, r, obs[i])

    loop_once()  # untimed: the first pass pays allocation and start-up costs (2-5x)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loop_once()
    torch.cuda.synchronize()
    loop_s = (time.perf_counter() - t0) * ncirc / len(loop_idx)
    nparams = int(sum(2 * int(n) * int(l) for n, l in zip(ns, ls)))
    return {"workload": f"hea_batch{ncirc}_q8-18_l4-16_c64_ising", "circuits": ncirc,
            "gates": int(sum(len(c) for c in circs)), "angles": nparams,
            "launch_ms": sec * 1e3, "circuits_per_s": ncirc / sec,
            "angle_derivatives_per_s": nparams / sec, "e2e_ms_with_results_copy": e2e * 1e3,
            "autotuned": best, "autotune_s": tune_s,
            "amplitude_updates_per_s": work["amplitude_updates"] / sec,
            "roofline": {"bound": "hbm", "achieved": work["global_bytes"] / sec / 1e9,
                         "peak": peak, "unit": "GB/s",
                         "frac": work["global_bytes"] / sec / 1e9 / peak,
                         "peak_source": f"{peak_kind} hbm_gbs",
                         "traffic_note": "tile traffic of the circuits larger than a tile "
                                         "(the others stay in shared memory): "
                                         f"{work['global_bytes'] / 1e9:.2f} GB per launch"},
            "autotune_ms": {k: v * 1e3 for k, v in times.items()}, "launch_shape": info,
            "max_abs_energy_err_vs_c128": err_e, "max_abs_grad_err_vs_c128": err_g,
            "checked_circuits": len(idx),
            "per_circuit_loop_s_extrapolated": loop_s, "speedup_vs_per_circuit_loop": loop_s / sec}


def peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def traffic_per_launch(n, elem_bytes):
    """DRAM bytes per fused-stage launch from the committed ncu summary,
    scaled to this state size (traffic grows with the amplitudes moved)."""
    f = ROOT / "profiles" / "k_stage_traffic.json"
    if not f.exists():
        return None
    d = json.loads(f.read_text())
    per_amp = d.get("dram_bytes_per_amplitude", {}).get(str(elem_bytes))
    if per_amp is None:
        return None
    return float(per_amp) * (1 << n)


class Clocks:
    """nvidia-smi sampler for the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(f"/tmp/qsv_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        self.path.unlink(missing_ok=True)
        if not rows:
            return None
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        smax = max((num(r[2]) for r in rows if num(r[2]) is not None), default=None)
        power = [num(r[3]) for r in rows if num(r[3]) is not None]
        loaded = [s for s, p in zip(sm, power) if p is not None and p > 250] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": reasons, "samples": len(rows)}


class CpuBrickSample:
    """QCLAB++'s CPU simulate (oracle/_ref, OpenMP, all host threads) timed
    on WHOLE brick layers of the circuit, so the sample has the circuit's own
    gate mix (per layer n one-qubit gates, which stream the state twice, and
    n/2 CNOT/CZ, which stream it once or half).  The state is allocated and
    first-touched once, outside the timed calls; each ``run()`` resets it to
    |0...0> (untimed) and times QCircuit::simulate over the sampled layers.
    Without oracle/_ref the C restatement (one thread) is timed instead at
    24 qubits on whole layers of a 24-qubit brick and scaled by 2^(n-24)."""

    def __init__(self, n, recs, layer_sizes, budget_s=15.0):
        import oracle
        self.oracle = oracle
        self.n = n
        self.kind = "reference" if oracle.ref_available() else "port"
        if self.kind == "port":
            from qclab_b200 import workloads as W
            self.n_s = min(n, 24)
            sizes = W.brick_layer_sizes(self.n_s, 2)
            self.recs = W.brick(self.n_s, 2, seed=0).gate_records(np.complex128)
            self.layers = 2
            self.threads = 1
            self.x = np.zeros(1 << self.n_s, dtype=np.complex128)
            self.gates = sum(sizes)
            return
        try:
            import psutil
            avail = psutil.virtual_memory().available
        except Exception:
            avail = 1 << 40
        self.n_s = n
        while self.n_s > 20 and (1 << self.n_s) * 16 * 2.5 > avail:
            self.n_s -= 1
        # size the sample from one timed layer: as many whole layers as fit the budget
        first = recs[:layer_sizes[0]]
        rc = oracle.RefCircuit(self.n_s, np.complex128, first)
        rc.state[:] = 0
        rc.state[0] = 1
        t0 = time.perf_counter()
        rc.apply()
        per_layer = time.perf_counter() - t0
        rc.close()
        self.layers = int(max(1, min(len(layer_sizes), budget_s // max(per_layer, 1e-6))))
        self.gates = sum(layer_sizes[:self.layers])
        self.rc = oracle.RefCircuit(self.n_s, np.complex128, recs[:self.gates])
        self.threads = oracle.ref_threads()

    def run(self):
        """Gates/s of one timed simulate over the sampled layers."""
        if self.kind == "port":
            self.x[:] = 0
            self.x[0] = 1
            t0 = time.perf_counter()
            self.oracle.apply(self.x, self.recs)
            dt = time.perf_counter() - t0
        else:
            self.rc.state[:] = 0
            self.rc.state[0] = 1
            t0 = time.perf_counter()
            self.rc.apply()
            dt = time.perf_counter() - t0
        return self.gates / dt * (1 << self.n_s) / (1 << self.n)

    def describe(self):
        if self.kind == "port":
            return (f"C oracle, 1 thread, 2 whole brick layers ({self.gates} gates) at "
                    f"{self.n_s} qubits, scaled by 2^{self.n - self.n_s}")
        return (f"QCLAB++ QCircuit::simulate (g++ -O3 -fopenmp), {self.threads} threads, the "
                f"first {self.layers} whole brick layer(s) ({self.gates} gates, the circuit's "
                f"gate mix) at {self.n_s} qubits"
                + (f", scaled by 2^{self.n - self.n_s}" if self.n_s != self.n else ""))

    def close(self):
        if getattr(self, "rc", None) is not None:
            self.rc.close()
            self.rc = None


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    from qclab_b200 import workloads as W
    recs = W.brick(args.qubits, args.depth, seed=args.seed).gate_records(np.complex128)
    sample = CpuBrickSample(args.qubits, recs, W.brick_layer_sizes(args.qubits, args.depth),
                            budget_s=8.0)
    vals = []
    for i in range(args.warmup + args.steps):
        v = sample.run()
        if i >= args.warmup:
            vals.append(v)
    sample.close()
    value = statistics.median(vals)
    threads, kind, txt = sample.threads, sample.kind, sample.describe()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "gates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128", "data": "synthetic: seeded random brick circuit, |0...0> input",
        "config": workload_config(args, len(recs), world),
        "cpu_baseline": {"value": value, "unit": "gates/s", "cores": threads, "kind": kind,
                         "sample": txt},
        "e2e": {"value": value, "unit": "gates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def full_size_parity(torch, stream, n, args, recs, sv):
    """Parity of the fused complex<double> sweep (run again in the bench's
    state `sv`) and of a fused complex<float> sweep against the
    reference-exact path; the latter is
    checked against the committed summary of QCLAB++'s CPU simulate on the
    same circuit (tests/golden/make_brick30_pin.py) when that fixture exists
    for this workload."""
    from qclab_b200 import StateVector
    fix = ROOT / "tests" / "golden" / f"brick{n}_d{args.depth}_s{args.seed}_c128.npz"
    want = dict(np.load(fix)) if fix.exists() else None
    sub = recs if want is not None else recs[:sum(
        n + len(range(l % 2, n - 1, 2)) for l in range(max(args.parity_layers, 1)))]
    out = {"gates": len(sub)}
    with StateVector(n, np.complex128) as ref:
        ref.set_stream(stream.cuda_stream)
        ref.apply(sub, "N", 0, fused=False)
        if want is not None:
            got = ref.summary(want["idx"])
            bitwise = (got["sha256"] == str(want["sha256"]) and
                       bool(np.array_equal(got["amp"], want["amp"])) and
                       bool(np.array_equal(got["block_p"], want["block_p"])))
            out.update({"against": "QCLAB++ QCircuit::simulate digest (SHA-256 of the final "
                                   "state, samples, block profile)",
                        "bitwise": bitwise, "sha256": got["sha256"],
                        "reference_cpu_seconds": float(want["seconds"])})
        else:
            out.update({"against": "qsv_apply (bitwise equal to QCLAB++ CPU apply in tests)",
                        "bitwise": None})
        # the fused complex<double> sweep of the same gates, in the bench's state
        # infidelity as computed (1 - |<a|b>|^2; negative when rounding left
        # the fused state's norm slightly above 1) and with both norms divided out
        ref_n2 = ref.norm2()
        sv.set_basis(0)
        sv.apply(sub, "N", 0, fused=True)
        ip, maxabs = sv.compare(ref)
        n2 = sv.norm2()
        out["c128_fused"] = {"max_abs_error": maxabs, "infidelity": 1.0 - abs(ip) ** 2,
                             "infidelity_normalised": 1.0 - abs(ip) ** 2 / (n2 * ref_n2),
                             "norm2": n2, "bound": 1e-12}
        with StateVector(n, np.complex64) as f:
            f.set_stream(stream.cuda_stream)
            f.apply(sub, "N", 0, fused=True)
            ip, maxabs = f.compare(ref)
            n2 = f.norm2()
        out["c64_fused"] = {"max_abs_error": maxabs, "infidelity": 1.0 - abs(ip) ** 2,
                            "infidelity_normalised": 1.0 - abs(ip) ** 2 / (n2 * ref_n2),
                            "norm2": n2, "bound": 1e-5}
    return out


def workload_config(args, ngates, world):
    return {"workload": f"brick{args.qubits}_depth{args.depth}_c128", "qubits": args.qubits,
            "depth": args.depth, "gates": ngates, "seed": args.seed,
            "parallelism": f"replicas{world}" if world > 1 else "single",
            "path": "fused sweep (qsv_apply_fused)",
            "l2": "no flush: the 16 GiB state is larger than L2 (126 MB)"}


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    from qclab_b200 import StateVector, launch_count
    from qclab_b200 import _lib as L
    from qclab_b200 import workloads as W
    from qclab_b200.replicas import job_throughput, job_time_ms, replica_seed

    n = args.qubits
    circ = W.brick(n, args.depth, seed=replica_seed(args.seed, rank))
    recs = circ.gate_records(np.complex128)
    ngates = len(recs)
    stream = torch.cuda.current_stream()
    sv = StateVector(n, np.complex128)
    sv.set_stream(stream.cuda_stream)
    opts = L.FuseOpts(profile=1)
    lib = L.load()

    def step():
        sv.set_basis(0)
        sv.apply(recs, "N", 0, fused=True, opts=opts)

    def stage_times():
        cnt = C.c_int(0)
        lib.qsv_last_stage_times(None, 0, C.byref(cnt))
        buf = (C.c_float * cnt.value)()
        lib.qsv_last_stage_times(buf, cnt.value, C.byref(cnt))
        return list(buf)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    launches0 = launch_count()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0.record(stream)
    stage_ms = []
    for _ in range(args.steps):
        step()
        stage_ms.extend(stage_times())
    t1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = t0.elapsed_time(t1)
    launches = launch_count() - launches0
    clk = clocks.stop()
    ms = job_time_ms(ms, dist if world > 1 else None, device="cuda")
    ms_per_step = ms / args.steps
    value = job_throughput(ngates, args.steps, ms, world)

    # roofline of the dominant kernel: the fused stage sweep, which runs its
    # register passes on the FP64 tensor cores (k_dmma3).  HBM: one read and
    # one write of the state per stage launch.  Tensor: each pass applies a
    # 16x16 real matrix to every 8-amplitude group, 64 flops per amplitude.
    n_stages = len(stage_ms) // max(args.steps, 1)
    state_bytes = (1 << n) * 16
    alg_bytes = 2 * state_bytes
    avg_stage_ms = statistics.mean(stage_ms) if stage_ms else float("nan")
    achieved = alg_bytes / (avg_stage_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    traffic = traffic_per_launch(n, 16)
    st_, ps_, op_ = C.c_int(), C.c_int(), C.c_int()
    L.check(lib.qsv_plan_passes(n, L.C128, C.c_void_p(recs.ctypes.data), len(recs), b"N", 0,
                                None, C.byref(st_), C.byref(ps_), C.byref(op_)), "qsv_plan_passes")
    flops_step = ps_.value * (1 << n) * 64.0
    tc_peak = C.c_double()
    L.check(lib.qsv_fp64_mma_peak(C.byref(tc_peak)), "qsv_fp64_mma_peak")
    tc_achieved = flops_step / (sum(stage_ms) / max(args.steps, 1) / 1e3) / 1e12
    roofline = {"bound": "hbm", "kernel": "k_dmma3<double2> (fused stage sweep, FP64 tensor cores)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} hbm_gbs", "traffic": traffic,
                "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_stage_ms,
                "launches_per_step": n_stages,
                "tensor_fp64": {"achieved": tc_achieved, "peak": tc_peak.value, "unit": "TFLOP/s",
                                "frac": tc_achieved / tc_peak.value,
                                "peak_source": "measured live (qsv_fp64_mma_peak, mma.sync m8n8k4 f64)",
                                "flops_per_step": flops_step, "passes_per_step": ps_.value}}

    # unfused reference-exact path on the first layer (side measurement)
    unf = None
    if args.unfused_gates > 0:
        sub = recs[:args.unfused_gates]
        sv.set_basis(0)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sv.apply(sub, "N", 0, fused=False)
        b.record(stream)
        torch.cuda.synchronize()
        ums = a.elapsed_time(b)
        unf_bytes = 0
        for r in sub:
            k = int(r["kind"])
            unf_bytes += state_bytes * (2 if k in (L.HADAMARD, L.ROTATION_X, L.ROTATION_Y, L.ROTATION_Z)
                                        else 1 if k == L.CX else 0.5)
        unf = {"gates": len(sub), "gates_per_s": len(sub) / (ums / 1e3),
               "hbm_gbs": unf_bytes / (ums / 1e3) / 1e9, "path": "qsv_apply (bit-exact)"}

    # parity at full size: the reference-exact path over the whole circuit,
    # pinned to QCLAB++'s own simulate by the committed digest when this is
    # the pinned workload (else over the first layers), then the fused
    # complex<double> state (this step's result) and a fused complex<float>
    # sweep compared with it
    parity = None
    if args.parity_layers != 0 and world == 1:
        parity = full_size_parity(torch, stream, n, args, recs, sv)

    # end to end through the C ABI with host buffers (copies inside the timed region)
    e2e = None
    if not args.no_e2e:
        # every rank takes the same barrier + reduction even if its own
        # pinned allocation fails (its time is then +inf)
        e_steps = max(1, min(args.steps, 2))
        err = None
        host = None
        try:
            host = torch.zeros(1 << n, dtype=torch.complex128, pin_memory=True)
            host[0] = 1
        except Exception as ex:  # pinned allocation can fail on small hosts
            err = str(ex)[:200]
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ems = float("inf")
        if host is not None:
            hp = host.data_ptr()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(e_steps):
                sv.upload_ptr(hp, state_bytes)
                sv.apply(recs, "N", 0, fused=True)
                sv.download_ptr(hp, state_bytes)
            b.record(stream)
            torch.cuda.synchronize()
            ems = a.elapsed_time(b)
            del host
        ems = job_time_ms(ems, dist if world > 1 else None, device="cuda")
        e2e = {"value": job_throughput(ngates, e_steps, ems, world) if math.isfinite(ems) else None,
               "unit": "gates/s", "h2d_bytes_per_step": state_bytes,
               "d2h_bytes_per_step": state_bytes, "steps": e_steps, "ms_per_step": ems / e_steps,
               "api": "qsv_upload + qsv_apply_fused + qsv_download (pinned host buffer)"}
        if err or not math.isfinite(ems):
            e2e["error"] = err or "a rank could not allocate its pinned host buffer"

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sample = CpuBrickSample(n, recs, W.brick_layer_sizes(n, args.depth))
        v = sample.run()
        cpu = {"value": v, "unit": "gates/s", "cores": sample.threads, "kind": sample.kind,
               "sample": sample.describe()}
        sample.close()

    sv.close()
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        for name, fn in (("adjoint", lambda: adjoint_extra(torch, stream, args.ps_params)),
                         ("precision", lambda: precision_extra(torch, stream)),
                         ("batch", lambda: batch_extra(torch, stream))):
            try:
                extras[name] = fn()
            except Exception as ex:  # reported, not fatal: the headline line still prints
                extras[name] = {"error": f"{type(ex).__name__}: {ex}"[:300]}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "gates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic: seeded random brick circuit, |0...0> input",
            "config": workload_config(args, ngates, world),
            "hbm_gbs_algorithmic": n_stages * alg_bytes / (ms_per_step / 1e3) / 1e9,
            "hbm_gbs_effective_unfused_equivalent": None,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": launches, "unfused_first_layer": unf,
            "parity_vs_reference_exact": parity,
        }
        line.update(extras)
        eff = 0
        for r in recs:
            k = int(r["kind"])
            eff += state_bytes * (2 if k in (L.HADAMARD, L.ROTATION_X, L.ROTATION_Y, L.ROTATION_Z)
                                  else 1 if k == L.CX else 0.5)
        line["hbm_gbs_effective_unfused_equivalent"] = eff / (ms_per_step / 1e3) / 1e9
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Pins the headline brick circuit at full size by running QCLAB++ itself.

The workload is the 30-qubit random brick circuit of depth 200 (seed 2024,
8,900 gates, |0...0> input; ``qclab_b200.workloads.brick``).  This script
builds the reference's own ``QCircuit<T>`` from the same gate records
(oracle/_ref/libqclab_ref.so, compiled from the reference's sources by
oracle/Makefile), runs its CPU ``QCircuit::simulate`` (OpenMP, all host
threads; include/qclab/QCircuit.hpp:164-166) once, and stores a fixture small
enough to commit:

* ``sha256``      digest of the final state's bytes (2^30 elements of T);
* ``norm2``       FP64 sum of |a_i|^2;
* ``idx``/``amp`` 4096 seeded sample indices and their amplitudes;
* ``block_p``     FP64 sum of |a_i|^2 over each of 256 contiguous blocks of
                  2^22 amplitudes (a probability profile of the whole state).

The GPU tests hash the reference-exact path's 30-qubit state and compare it
with ``sha256`` (bitwise parity at full size), then check the fused sweeps
against that state within the stated tolerances.  One run takes about an
hour per element type on 8 cores and needs 2^30 * sizeof(T) bytes of host
memory (16 GiB for complex<double>).

    python tests/golden/make_brick30_pin.py --dtype c128
    python tests/golden/make_brick30_pin.py --dtype c64
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

import oracle  # noqa: E402
from qclab_b200 import util  # noqa: E402
from qclab_b200 import workloads as W  # noqa: E402

QUBITS, DEPTH, SEED = 30, 200, 2024
SAMPLES, SAMPLE_SEED = 4096, 7
BLOCKS = 256
DTYPES = {"c128": np.complex128, "c64": np.complex64}


def fixture_path(tag: str) -> Path:
    return HERE / f"brick{QUBITS}_d{DEPTH}_s{SEED}_{tag}.npz"


def sample_indices(n: int = QUBITS) -> np.ndarray:
    rng = np.random.default_rng(SAMPLE_SEED)
    idx = rng.choice(1 << n, size=SAMPLES - 2, replace=False)
    return np.unique(np.concatenate([idx, [0, (1 << n) - 1]])).astype(np.int64)


def state_summary(state: np.ndarray) -> dict:
    """Digest, norm, samples and block profile of one final state (the same
    routine the GPU side runs on its downloaded chunks)."""
    n = int(state.size).bit_length() - 1
    chunk = 1 << min(n, 26)
    return util.state_summary((state[s:s + chunk] for s in range(0, state.size, chunk)), n,
                              sample_indices(n), BLOCKS)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--dtype", choices=sorted(DTYPES), default="c128")
    args = ap.parse_args()
    dt = np.dtype(DTYPES[args.dtype])
    if not oracle.ref_available():
        oracle.build()
    recs = W.brick(QUBITS, DEPTH, seed=SEED).gate_records(dt)
    rc = oracle.RefCircuit(QUBITS, dt, recs)
    rc.state[0] = 1
    threads = rc.lib.ref_num_threads()
    t0 = time.perf_counter()
    rc.apply("N", 0)
    secs = time.perf_counter() - t0
    out = state_summary(rc.state)
    rc.close()
    out.update({"qubits": QUBITS, "depth": DEPTH, "seed": SEED, "gates": len(recs),
                "records_sha256": hashlib.sha256(recs.tobytes()).hexdigest(),
                "seconds": secs, "threads": threads, "host_cpus": os.cpu_count()})
    np.savez_compressed(fixture_path(args.dtype), **{k: np.asarray(v) for k, v in out.items()})
    print(f"{args.dtype}: {len(recs)} gates in {secs:.0f} s on {threads} threads; "
          f"sha256 {out['sha256']}; norm2 {out['norm2']:.17g}")


if __name__ == "__main__":
    main()

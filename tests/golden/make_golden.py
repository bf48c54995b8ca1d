"""Generates the golden fixtures in tests/golden/ by running QCLAB++ itself.

The reference is compiled from its own sources into oracle/_ref/ by
oracle/Makefile (needs the reference tree, present only on the development
machine).  For every case of tests/golden/cases.py the reference's
QCircuit<T>::apply output is stored, so the tests can pin the oracle and the
GPU library to the reference on machines without it.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE))

import oracle  # noqa: E402
from cases import DTYPES, circuit_cases, gate_cases  # noqa: E402


def case_digest(records, op, offset, x) -> str:
    h = hashlib.sha256()
    h.update(records.tobytes())
    h.update(op.encode())
    h.update(str(offset).encode())
    h.update(x.tobytes())
    return h.hexdigest()[:16]


def main() -> None:
    if not oracle.ref_available():
        oracle.build()
    out = {}
    for dt in DTYPES:
        name = np.dtype(dt).name
        outs, digests = [], []
        for n, recs, op, off, x in gate_cases(dt):
            outs.append(oracle.ref_apply(x.copy(), recs, op, off))
            digests.append(case_digest(recs, op, off, x))
        out[f"gates_{name}"] = np.concatenate(outs)
        out[f"gates_{name}_digest"] = np.array(
            hashlib.sha256("".join(digests).encode()).hexdigest())
        out[f"gates_{name}_count"] = np.array(len(outs))
        for cname, n, recs, op, off, x in circuit_cases(dt):
            out[f"circ_{name}_{cname}"] = oracle.ref_apply(x.copy(), recs, op, off)
            out[f"circ_{name}_{cname}_digest"] = np.array(case_digest(recs, op, off, x))
    np.savez_compressed(HERE / "reference_outputs.npz", **out)
    print(f"wrote {HERE / 'reference_outputs.npz'} with {len(out)} arrays")


if __name__ == "__main__":
    main()

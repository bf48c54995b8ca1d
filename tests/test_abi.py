"""The C ABI library: loads, exports every declared symbol, host-side
lowering and planning (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from qclab_b200 import _lib as L
from qclab_b200 import workloads as W

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        names |= set(re.findall(r"\b(qsv_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = L.load()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_and_status_strings():
    lib = L.load()
    assert lib.qsv_abi_version() == 1
    assert lib.qsv_status_string(2) == b"QSV_ERROR_QUBIT"


def test_gate_record_layout():
    assert C.sizeof(L.Gate) == L.GATE_DTYPE.itemsize == 296


def plan(n, recs, dtype=L.C128, op=b"N", offset=0, opts=None, cap=4096):
    lib = L.load()
    ns = C.c_int(0)
    sg = (C.c_int * cap)()
    st = lib.qsv_plan_stats(n, dtype, C.c_void_p(recs.ctypes.data), len(recs), op, offset,
                            C.byref(opts) if opts else None, C.byref(ns), sg, cap)
    return st, ns.value, list(sg[:ns.value])


def test_planner_covers_every_gate_once():
    lib = L.load()
    for n, depth in [(8, 5), (20, 10), (30, 4)]:
        c = W.brick(n, depth, seed=1)
        recs = c.gate_records(np.complex128)
        # sparse register passes: one op per gate
        st, ns, sg = plan(n, recs, opts=L.FuseOpts(engine=1))
        assert st == 0
        assert sum(sg) == len(recs)
        assert ns <= len(recs)
        # tensor-core engine: one dense op per pass, no more passes than gates
        stages, passes, ops = C.c_int(), C.c_int(), C.c_int()
        assert lib.qsv_plan_passes(n, L.C128, C.c_void_p(recs.ctypes.data), len(recs), b"N", 0,
                                   None, C.byref(stages), C.byref(passes), C.byref(ops)) == 0
        assert ops.value == passes.value <= len(recs)
        assert 0 < stages.value <= passes.value


def test_tensor_plans_need_no_more_passes_than_greedy():
    """The tensor-core engine picks each pass's bits by a greedy rollout, which
    never needs more passes than the plain in-order greedy planner.  The
    bounds are that planner's pass counts for these circuits."""
    lib = L.load()
    cases = [(W.brick(30, 200, seed=3), 1992), (W.qft(30), 251),
             (W.random_mixed(24, 2000, seed=1), 565)]
    for c, greedy in cases:
        recs = c.gate_records(np.complex128)
        stages, passes, ops = C.c_int(), C.c_int(), C.c_int()
        assert lib.qsv_plan_passes(c.nbQubits(), L.C128, C.c_void_p(recs.ctypes.data), len(recs),
                                   b"N", 0, None, C.byref(stages), C.byref(passes),
                                   C.byref(ops)) == 0
        assert 0 < passes.value <= greedy


def test_planner_errors_are_status_codes():
    c = W.brick(6, 2, seed=1)
    recs = c.gate_records(np.complex128)
    st, _, _ = plan(5, recs)           # gates on qubit 5 do not fit 5 qubits
    assert st == 2
    st, _, _ = plan(6, recs, op=b"X")  # bad op
    assert st == 1
    st, _, _ = plan(6, recs, offset=1)  # offset pushes qubit 5 out
    assert st == 2
    from qclab_b200 import QCircuit, RotationX
    c = QCircuit(2)
    c.push_back(RotationX(0, 0.3))
    st, _, _ = plan(2, c.gate_records(np.float64), dtype=L.F64)
    assert st == 6                     # complex gate on a real state
    bad = c.gate_records(np.complex128)
    bad[0]["kind"] = 99
    st, _, _ = plan(2, bad)
    assert st == 1

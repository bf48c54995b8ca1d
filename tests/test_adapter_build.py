"""The C++ front end compiles against the reference's headers (CPU only)."""
import subprocess
from pathlib import Path

import pytest

import oracle

ROOT = Path(__file__).resolve().parent.parent
TREE = oracle.ref_tree()


@pytest.mark.skipif(TREE is None, reason="reference tree not present (set QCLAB_REF)")
def test_adapter_header_compiles(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text('#include "qclab_b200/adapter.hpp"\n'
                   "template void qclab_b200::simulate(const qclab::QCircuit<std::complex<double>>&,"
                   " std::vector<std::complex<double>>&, bool);\n"
                   "template void qclab_b200::simulate(const qclab::QCircuit<float>&,"
                   " std::vector<float>&, bool);\n")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", f"-I{ROOT / 'include'}",
                        f"-I{TREE / 'include'}", str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]

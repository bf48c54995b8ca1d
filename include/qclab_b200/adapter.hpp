// qclab_b200/adapter.hpp -- QCLAB++ front end for the B200 backend.
//
// Header-only C++17.  Include it in a translation unit that already sees the
// QCLAB++ headers (include/qclab/...) and link libqclab_b200.so.  It lowers a
// qclab::QObject<T> tree -- QCircuit (nested, with offsets), every gate class
// of qclab::qgates, PointerGate1/2 and user subclasses of QGate1 / QGate2 /
// QControlledGate2 -- to qsv_gate records and runs them through the C ABI.
//
//   qclab_b200::simulate(circuit, vec)       ~ circuit.simulate(vec)
//                                              (include/qclab/QCircuit.hpp:164-166)
//   qclab_b200::apply(obj, op, n, vec, off)  ~ obj.apply(op, n, vec, off)
//                                              (include/qclab/QObject.hpp:52-53)
//   qclab_b200::simulate_device(circuit, p)  ~ circuit.simulate_device(p)
//                                              (include/qclab/QCircuit.hpp:170-172)
//
// The reference-exact path (default) gives the same bits as QCLAB++'s CPU
// apply; `fused = true` selects the fused sweep (within 1e-12 for
// complex<double>).  Failures throw qclab_b200::Error (QCLAB++ itself only
// asserts).
#pragma once

#include <complex>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "qclab/QCircuit.hpp"
#include "qclab/qgates/CPhase.hpp"
#include "qclab/qgates/CRotationX.hpp"
#include "qclab/qgates/CRotationY.hpp"
#include "qclab/qgates/CRotationZ.hpp"
#include "qclab/qgates/CX.hpp"
#include "qclab/qgates/CY.hpp"
#include "qclab/qgates/CZ.hpp"
#include "qclab/qgates/Hadamard.hpp"
#include "qclab/qgates/Identity.hpp"
#include "qclab/qgates/PauliX.hpp"
#include "qclab/qgates/PauliY.hpp"
#include "qclab/qgates/PauliZ.hpp"
#include "qclab/qgates/Phase.hpp"
#include "qclab/qgates/Phase45.hpp"
#include "qclab/qgates/Phase90.hpp"
#include "qclab/qgates/PointerGate1.hpp"
#include "qclab/qgates/PointerGate2.hpp"
#include "qclab/qgates/RotationX.hpp"
#include "qclab/qgates/RotationXX.hpp"
#include "qclab/qgates/RotationY.hpp"
#include "qclab/qgates/RotationYY.hpp"
#include "qclab/qgates/RotationZ.hpp"
#include "qclab/qgates/RotationZZ.hpp"
#include "qclab/qgates/SWAP.hpp"
#include "qclab/qgates/iSWAP.hpp"
#include "qclab_b200.h"

namespace qclab_b200 {

class Error : public std::runtime_error {
 public:
  Error(qsv_status s, const std::string& where)
      : std::runtime_error(where + ": " + qsv_status_string(s) + ": " + qsv_last_error()),
        status(s) {}
  qsv_status status;
};

inline void check(qsv_status s, const char* where) {
  if (s != QSV_SUCCESS) throw Error(s, where);
}

template <typename T> constexpr qsv_dtype dtype_of();
template <> constexpr qsv_dtype dtype_of<std::complex<float>>() { return QSV_C64; }
template <> constexpr qsv_dtype dtype_of<std::complex<double>>() { return QSV_C128; }
template <> constexpr qsv_dtype dtype_of<float>() { return QSV_F32; }
template <> constexpr qsv_dtype dtype_of<double>() { return QSV_F64; }

namespace detail {

inline qsv_gate blank(int kind) {
  qsv_gate g;
  std::memset(&g, 0, sizeof(g));
  g.kind = kind;
  g.qubit1 = -1;
  g.control_state = 1;
  g.param = -1;
  return g;
}

template <typename T>
void put(double* m, int idx, const T& v) {
  if constexpr (qclab::is_complex_v<T>) {
    m[2 * idx] = (double)v.real();
    m[2 * idx + 1] = (double)v.imag();
  } else {
    m[2 * idx] = (double)v;
    m[2 * idx + 1] = 0.0;
  }
}

// SquareMatrix (column-major, SquareMatrix.hpp:125-132) -> record matrix
template <typename T>
void put_matrix(double* m, const qclab::dense::SquareMatrix<T>& A) {
  const int d = (int)A.rows();
  for (int c = 0; c < d; ++c)
    for (int r = 0; r < d; ++r) put(m, r + c * d, A(r, c));
}

template <typename T>
void lower(const qclab::QObject<T>& o, int offset, std::vector<qsv_gate>& out);

template <typename T>
bool lower_circuit(const qclab::QObject<T>& o, int offset, std::vector<qsv_gate>& out) {
  if (auto* c = dynamic_cast<const qclab::QCircuit<T>*>(&o)) {
    for (auto it = c->begin(); it != c->end(); ++it) lower<T>(**it, offset + c->offset(), out);
    return true;
  }
  return false;
}

template <typename T>
void lower(const qclab::QObject<T>& o, int offset, std::vector<qsv_gate>& out) {
  using namespace qclab::qgates;
  if (lower_circuit<T>(o, offset, out)) return;
  if (auto* p = dynamic_cast<const PointerGate1<T>*>(&o)) {
    lower<T>(*p->ptr(), offset + p->offset(), out);
    return;
  }
  if (auto* p = dynamic_cast<const PointerGate2<T>*>(&o)) {
    lower<T>(*p->ptr(), offset + p->offset(), out);
    return;
  }
  constexpr bool cplx = qclab::is_complex_v<T>;
  const std::vector<int> qs = o.qubits();
  // ---- 1-qubit classes ------------------------------------------------------
  if (o.nbQubits() == 1) {
    const int q = qs[0] + offset;
    qsv_gate g = blank(QSV_MATRIX1);
    g.qubit0 = q;
    if (dynamic_cast<const Identity<T>*>(&o)) g.kind = QSV_IDENTITY;
    else if (dynamic_cast<const Hadamard<T>*>(&o)) g.kind = QSV_HADAMARD;
    else if (dynamic_cast<const PauliX<T>*>(&o)) g.kind = QSV_PAULI_X;
    else if (dynamic_cast<const PauliZ<T>*>(&o)) g.kind = QSV_PAULI_Z;
    else if (auto* r = dynamic_cast<const RotationY<T>*>(&o)) {
      g.kind = QSV_ROTATION_Y; g.cos = r->cos(); g.sin = r->sin();
    } else if constexpr (cplx) {
      if (dynamic_cast<const PauliY<T>*>(&o)) g.kind = QSV_PAULI_Y;
      else if (auto* r = dynamic_cast<const RotationX<T>*>(&o)) {
        g.kind = QSV_ROTATION_X; g.cos = r->cos(); g.sin = r->sin();
      } else if (auto* r = dynamic_cast<const RotationZ<T>*>(&o)) {
        g.kind = QSV_ROTATION_Z; g.cos = r->cos(); g.sin = r->sin();
      } else if (auto* r = dynamic_cast<const Phase<T>*>(&o)) {
        g.kind = QSV_PHASE; g.cos = r->cos(); g.sin = r->sin();
      } else if (dynamic_cast<const Phase45<T>*>(&o)) g.kind = QSV_PHASE45;
      else if (dynamic_cast<const Phase90<T>*>(&o)) g.kind = QSV_PHASE90;
      else put_matrix(g.matrix, o.matrix());     // QGate1 subclass: lambda_QGate1 path
    } else {
      put_matrix(g.matrix, o.matrix());
    }
    out.push_back(g);
    return;
  }
  // ---- controlled classes ---------------------------------------------------
  if (auto* cg = dynamic_cast<const QControlledGate2<T>*>(&o)) {
    qsv_gate g = blank(QSV_CONTROLLED1);
    g.qubit0 = cg->control() + offset;
    g.qubit1 = cg->target() + offset;
    g.control_state = cg->controlState();
    if (dynamic_cast<const CX<T>*>(&o)) g.kind = QSV_CX;
    else if (dynamic_cast<const CZ<T>*>(&o)) g.kind = QSV_CZ;
    else if (auto* r = dynamic_cast<const CRotationY<T>*>(&o)) {
      g.kind = QSV_CROTATION_Y; g.cos = r->cos(); g.sin = r->sin();
    } else if constexpr (cplx) {
      if (dynamic_cast<const CY<T>*>(&o)) g.kind = QSV_CY;
      else if (auto* r = dynamic_cast<const CPhase<T>*>(&o)) {
        g.kind = QSV_CPHASE; g.cos = r->cos(); g.sin = r->sin();
      } else if (auto* r = dynamic_cast<const CRotationX<T>*>(&o)) {
        g.kind = QSV_CROTATION_X; g.cos = r->cos(); g.sin = r->sin();
      } else if (auto* r = dynamic_cast<const CRotationZ<T>*>(&o)) {
        g.kind = QSV_CROTATION_Z; g.cos = r->cos(); g.sin = r->sin();
      } else put_matrix(g.matrix, cg->gate()->matrix());
    } else {
      put_matrix(g.matrix, cg->gate()->matrix());
    }
    out.push_back(g);
    return;
  }
  // ---- uncontrolled 2-qubit classes -----------------------------------------
  if (o.nbQubits() == 2) {
    qsv_gate g = blank(QSV_MATRIX2);
    g.qubit0 = qs[0] + offset;
    g.qubit1 = qs[1] + offset;
    if (dynamic_cast<const SWAP<T>*>(&o)) g.kind = QSV_SWAP;
    else if constexpr (cplx) {
      if (dynamic_cast<const iSWAP<T>*>(&o)) g.kind = QSV_ISWAP;
      else if (auto* r = dynamic_cast<const RotationXX<T>*>(&o)) {
        g.kind = QSV_ROTATION_XX; g.cos = r->cos(); g.sin = r->sin();
      } else if (auto* r = dynamic_cast<const RotationYY<T>*>(&o)) {
        g.kind = QSV_ROTATION_YY; g.cos = r->cos(); g.sin = r->sin();
      } else if (auto* r = dynamic_cast<const RotationZZ<T>*>(&o)) {
        g.kind = QSV_ROTATION_ZZ; g.cos = r->cos(); g.sin = r->sin();
      }
    }
    if (g.kind == QSV_MATRIX2) {
      // A user QGate2: QCLAB++'s vector apply (apply4 + lambda_QGate2) pairs
      // matrix() entries with the amplitudes |00>,|10>,|01>,|11> of the
      // sorted qubits.  MATRIX2 is in the kron basis, so pass P M P (P swaps
      // basis states 1 and 2) to reproduce that behaviour exactly.
      const auto M = o.matrix();
      const int p[4] = {0, 2, 1, 3};
      for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) put(g.matrix, r + c * 4, M(p[r], p[c]));
    }
    out.push_back(g);
    return;
  }
  throw Error(QSV_ERROR_NOT_SUPPORTED, "qclab_b200::lower: unsupported QObject");
}

}  // namespace detail

// Flat qsv_gate records of a QCLAB++ object (circuit order, offsets applied).
template <typename T>
std::vector<qsv_gate> records(const qclab::QObject<T>& o, int offset = 0) {
  std::vector<qsv_gate> out;
  detail::lower<T>(o, offset, out);
  return out;
}

// obj.apply(op, nbQubits, vector, offset) on the GPU; the vector is copied to
// the device and back.
template <typename T>
void apply(const qclab::QObject<T>& o, qclab::Op op, int nbQubits, std::vector<T>& vector,
           int offset = 0, bool fused = false) {
  const std::vector<qsv_gate> g = records<T>(o, 0);
  if (vector.size() != (size_t(1) << nbQubits))
    throw Error(QSV_ERROR_SIZE, "qclab_b200::apply: vector size");
  check(qsv_apply_host(nbQubits, dtype_of<T>(), vector.data(), g.data(), g.size(),
                       static_cast<char>(op), offset, fused ? 1 : 0),
        "qclab_b200::apply");
}

// circuit.simulate(vector) on the GPU.
template <typename T, typename G>
void simulate(const qclab::QCircuit<T, G>& c, std::vector<T>& vector, bool fused = false) {
  apply<T>(c, qclab::Op::NoTrans, c.nbQubits(), vector, 0, fused);
}

// obj.apply_device(op, nbQubits, device_vector, offset) -- the QObject<T>
// virtual of the offload build (include/qclab/QObject.hpp:56-59) and its
// QCircuit<T,G> loop (include/qclab/QCircuit.hpp:146-160): in place on
// caller-owned device memory of 2^nbQubits elements of T on the current
// device; the gate list runs in reverse order for [Conj]Trans and every gate
// gets the circuits' offset_ plus `offset`.  Returns after the device work
// has finished, as the reference's synchronous offload loops do.
template <typename T>
void apply_device(const qclab::QObject<T>& o, qclab::Op op, int nbQubits, T* device_vector,
                  int offset = 0, bool fused = false) {
  const std::vector<qsv_gate> g = records<T>(o, 0);
  qsv_state s = nullptr;
  check(qsv_wrap(nbQubits, dtype_of<T>(), device_vector, &s), "qsv_wrap");
  const char opc = static_cast<char>(op);
  qsv_status st = fused ? qsv_apply_fused(s, g.data(), g.size(), opc, offset, nullptr)
                        : qsv_apply(s, g.data(), g.size(), opc, offset);
  if (st == QSV_SUCCESS) st = qsv_synchronize(s);
  qsv_destroy(s);
  check(st, "qclab_b200::apply_device");
}

// circuit.simulate_device(ptr) (include/qclab/QCircuit.hpp:169-172): in place
// on caller-owned device memory.
template <typename T, typename G>
void simulate_device(const qclab::QCircuit<T, G>& c, T* device_vector, bool fused = false) {
  apply_device<T>(c, qclab::Op::NoTrans, c.nbQubits(), device_vector, 0, fused);
}

}  // namespace qclab_b200

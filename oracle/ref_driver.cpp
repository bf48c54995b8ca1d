// ref_driver.cpp -- extern "C" driver around QCLAB++ itself.
//
// TEST INFRASTRUCTURE ONLY.  Compiled together with the reference's own
// sources (src/qgates/*.cpp, src/io/*.cpp) into oracle/_ref/libqclab_ref.so
// by oracle/Makefile.  It turns qsv_gate records into the reference's gate
// objects (qclab::qgates::*) and runs the reference's QCircuit::apply /
// simulate on a std::vector<T> it owns, so tests can compare the oracle and
// the GPU library with the reference, and bench.py can time the reference's
// CPU path (OpenMP, all host threads).  It contains no arithmetic of its
// own beyond building the gate objects.
#include <omp.h>

#include <complex>
#include <cstring>
#include <memory>
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
#include "qclab/qgates/QControlledGate2.hpp"
#include "qclab/qgates/RotationX.hpp"
#include "qclab/qgates/RotationXX.hpp"
#include "qclab/qgates/RotationY.hpp"
#include "qclab/qgates/RotationYY.hpp"
#include "qclab/qgates/RotationZ.hpp"
#include "qclab/qgates/RotationZZ.hpp"
#include "qclab/qgates/SWAP.hpp"
#include "qclab/qgates/iSWAP.hpp"
#include "qclab_b200.h"

namespace {

using qclab::Op;

template <typename T>
T entry(const double* m, int dim, int r, int c) {
  const double* p = m + 2 * (r + c * dim);
  if constexpr (qclab::is_complex_v<T>) {
    using R = qclab::real_t<T>;
    return T((R)p[0], (R)p[1]);
  } else {
    return (T)p[0];
  }
}

// A user 1-qubit gate: how a QCLAB++ user adds a custom matrix gate.  Its
// vector apply is the reference's generic QGate1::apply.
template <typename T>
class UserGate1 : public qclab::qgates::QGate1<T> {
 public:
  UserGate1(int qubit, const double* m)
      : qclab::qgates::QGate1<T>(qubit),
        mat_(entry<T>(m, 2, 0, 0), entry<T>(m, 2, 0, 1), entry<T>(m, 2, 1, 0),
             entry<T>(m, 2, 1, 1)) {}
  bool fixed() const override { return true; }
  qclab::dense::SquareMatrix<T> matrix() const override { return mat_; }
  void print() const override {}
  int toQASM(std::ostream&, const int = 0) const override { return -1; }

 protected:
  bool equals(const qclab::QObject<T>&) const override { return false; }
  qclab::dense::SquareMatrix<T> mat_;
};

// A user 2-qubit gate (generic QGate2::apply).  `m` is in the order the
// reference's apply4 lambda uses (x1..x4 = |00>,|10>,|01>,|11> of the
// sorted qubits).
// The state path (apply4) pairs slots differently from the kron basis, so
// the gate carries two matrices: `m` in apply4 slot order for the vector
// apply, `k` in the kron basis of the sorted qubits for the unitary update
// apply(Side, ...), whose loops use the kron order (src/qgates/QGate2.cpp:32-108).
template <typename T>
class UserGate2 : public qclab::qgates::QGate2<T> {
 public:
  UserGate2(int q0, int q1, const T* m, const T* k)
      : q_{std::min(q0, q1), std::max(q0, q1)},
        mat_(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8], m[9], m[10], m[11], m[12],
             m[13], m[14], m[15]),
        kron_(k[0], k[1], k[2], k[3], k[4], k[5], k[6], k[7], k[8], k[9], k[10], k[11], k[12],
              k[13], k[14], k[15]) {}
  bool fixed() const override { return true; }
  bool controlled() const override { return false; }
  int qubit() const override { return q_[0]; }
  std::vector<int> qubits() const override { return {q_[0], q_[1]}; }
  void setQubits(const int* q) override { q_[0] = q[0]; q_[1] = q[1]; }
  qclab::dense::SquareMatrix<T> matrix() const override { return side_ ? kron_ : mat_; }
  int toQASM(std::ostream&, const int = 0) const override { return -1; }
  using qclab::qgates::QGate2<T>::apply;
  void apply(qclab::Side side, qclab::Op op, const int nbQubits,
             qclab::dense::SquareMatrix<T>& matrix, const int offset = 0) const override {
    side_ = true;
    qclab::qgates::QGate2<T>::apply(side, op, nbQubits, matrix, offset);
    side_ = false;
  }

 protected:
  bool equals(const qclab::QObject<T>&) const override { return false; }
  int q_[2];
  qclab::dense::SquareMatrix<T> mat_, kron_;
  mutable bool side_ = false;
};

// A user controlled gate (generic QControlledGate2::apply).
template <typename T>
class UserControlled : public qclab::qgates::QControlledGate2<T> {
 public:
  UserControlled(int control, int target, const double* m, int cs)
      : qclab::qgates::QControlledGate2<T>(control, cs), gate_(target, m) {}
  bool fixed() const override { return true; }
  int qubit() const override { return std::min(this->control(), gate_.qubit()); }
  int target() const override { return gate_.qubit(); }
  const qclab::qgates::QGate1<T>* gate() const override { return &gate_; }
  void setTarget(const int t) override { gate_.setQubit(t); }
  void print() const override {}
  int toQASM(std::ostream&, const int = 0) const override { return -1; }

 protected:
  bool equals(const qclab::QObject<T>&) const override { return false; }
  UserGate1<T> gate_;
};

template <typename T>
int add_gate(qclab::QCircuit<T>& c, const qsv_gate& g) {
  using namespace qclab::qgates;
  using R = qclab::real_t<T>;
  const R cs = (R)g.cos, sn = (R)g.sin;
  const int q = g.qubit0, a = g.qubit0, b = g.qubit1, st = g.control_state;
  constexpr bool cplx = qclab::is_complex_v<T>;
  std::unique_ptr<qclab::QObject<T>> p;
  switch (g.kind) {
    case QSV_IDENTITY: p = std::make_unique<Identity<T>>(q); break;
    case QSV_HADAMARD: p = std::make_unique<Hadamard<T>>(q); break;
    case QSV_PAULI_X: p = std::make_unique<PauliX<T>>(q); break;
    case QSV_PAULI_Z: p = std::make_unique<PauliZ<T>>(q); break;
    case QSV_ROTATION_Y: p = std::make_unique<RotationY<T>>(q, cs, sn); break;
    case QSV_MATRIX1: p = std::make_unique<UserGate1<T>>(q, g.matrix); break;
    case QSV_CX: p = std::make_unique<CX<T>>(a, b, st); break;
    case QSV_CZ: p = std::make_unique<CZ<T>>(a, b, st); break;
    case QSV_CROTATION_Y: p = std::make_unique<CRotationY<T>>(a, b, cs, sn, st); break;
    case QSV_CONTROLLED1: p = std::make_unique<UserControlled<T>>(a, b, g.matrix, st); break;
    case QSV_SWAP: p = std::make_unique<SWAP<T>>(a, b); break;
    case QSV_MATRIX2: {
      // kron basis |qubit0 qubit1> -> apply4 slot order of the sorted qubits
      const int q0 = std::min(a, b);
      T m[16];
      int slot_of[4];
      for (int s = 0; s < 4; ++s) {
        const int bq0 = s & 1, bq1 = s >> 1;
        const int bfirst = (a == q0) ? bq0 : bq1, bsecond = (a == q0) ? bq1 : bq0;
        slot_of[s] = 2 * bfirst + bsecond;
      }
      for (int r = 0; r < 4; ++r)
        for (int cc = 0; cc < 4; ++cc) m[r * 4 + cc] = entry<T>(g.matrix, 4, slot_of[r], slot_of[cc]);
      // kron basis of the sorted qubits: index 2 bit(min) + bit(max)
      T k[16];
      auto kron_of = [&](int s) { return (a == q0) ? s : (((s & 1) << 1) | (s >> 1)); };
      for (int r = 0; r < 4; ++r)
        for (int cc = 0; cc < 4; ++cc) k[r * 4 + cc] = entry<T>(g.matrix, 4, kron_of(r), kron_of(cc));
      p = std::make_unique<UserGate2<T>>(a, b, m, k);
      break;
    }
    default:
      if constexpr (cplx) {
        switch (g.kind) {
          case QSV_PAULI_Y: p = std::make_unique<PauliY<T>>(q); break;
          case QSV_ROTATION_X: p = std::make_unique<RotationX<T>>(q, cs, sn); break;
          case QSV_ROTATION_Z: p = std::make_unique<RotationZ<T>>(q, cs, sn); break;
          case QSV_PHASE: p = std::make_unique<Phase<T>>(q, cs, sn); break;
          case QSV_PHASE45: p = std::make_unique<Phase45<T>>(q); break;
          case QSV_PHASE90: p = std::make_unique<Phase90<T>>(q); break;
          case QSV_CY: p = std::make_unique<CY<T>>(a, b, st); break;
          case QSV_CPHASE: p = std::make_unique<CPhase<T>>(a, b, cs, sn, st); break;
          case QSV_CROTATION_X: p = std::make_unique<CRotationX<T>>(a, b, cs, sn, st); break;
          case QSV_CROTATION_Z: p = std::make_unique<CRotationZ<T>>(a, b, cs, sn, st); break;
          case QSV_ISWAP: p = std::make_unique<iSWAP<T>>(a, b); break;
          case QSV_ROTATION_XX: p = std::make_unique<RotationXX<T>>(a, b, cs, sn); break;
          case QSV_ROTATION_YY: p = std::make_unique<RotationYY<T>>(a, b, cs, sn); break;
          case QSV_ROTATION_ZZ: p = std::make_unique<RotationZZ<T>>(a, b, cs, sn); break;
          default: return 1;
        }
      } else {
        return 6;
      }
  }
  if (!c.canInsert(*p)) return 2;
  c.push_back(std::move(p));
  return 0;
}

struct AnyCircuit {
  int dtype;
  std::shared_ptr<void> c;
};
struct AnyVec {
  int dtype;
  std::shared_ptr<void> v;
  void* data;
};

template <typename T>
AnyCircuit* make_circuit(int n, int dtype, const qsv_gate* g, size_t count, int* status) {
  auto c = std::make_shared<qclab::QCircuit<T>>(n);
  for (size_t i = 0; i < count; ++i) {
    const int st = add_gate<T>(*c, g[i]);
    if (st) {
      *status = st;
      return nullptr;
    }
  }
  *status = 0;
  return new AnyCircuit{dtype, c};
}

template <typename T>
int run(AnyCircuit* ac, AnyVec* av, char op, int offset) {
  auto* c = static_cast<qclab::QCircuit<T>*>(ac->c.get());
  auto* v = static_cast<std::vector<T>*>(av->v.get());
  if (op == 'N' && offset == 0) {
    c->simulate(*v);  // QCircuit::simulate, include/qclab/QCircuit.hpp:164-166
  } else {
    c->apply(static_cast<Op>(op), c->nbQubits(), *v, offset);
  }
  return 0;
}

// QCircuit<T>::apply(side, op, nbQubits, SquareMatrix<T>&, offset)
// (include/qclab/QCircuit.hpp:176-204) on a caller-held column-major matrix.
template <typename T>
int run_side(AnyCircuit* ac, char side, char op, int nbq, int offset, void* data) {
  auto* c = static_cast<qclab::QCircuit<T>*>(ac->c.get());
  const int64_t N = int64_t(1) << nbq;
  T* d = static_cast<T*>(data);
  qclab::dense::SquareMatrix<T> M(N);
  for (int64_t j = 0; j < N; ++j)
    for (int64_t i = 0; i < N; ++i) M(i, j) = d[i + j * N];
  c->apply(static_cast<qclab::Side>(side), static_cast<qclab::Op>(op), nbq, M, offset);
  for (int64_t j = 0; j < N; ++j)
    for (int64_t i = 0; i < N; ++i) d[i + j * N] = M(i, j);
  return 0;
}

// QCircuit<T>::matrix() (include/qclab/QCircuit.hpp:120-126), column-major.
template <typename T>
int run_matrix(AnyCircuit* ac, void* data) {
  auto* c = static_cast<qclab::QCircuit<T>*>(ac->c.get());
  const auto M = c->matrix();
  T* d = static_cast<T*>(data);
  for (int64_t j = 0; j < M.cols(); ++j)
    for (int64_t i = 0; i < M.rows(); ++i) d[i + j * M.rows()] = M(i, j);
  return 0;
}

template <typename T>
double run_nrmf(AnyCircuit* a, AnyCircuit* b) {
  return qclab::nrmF(*static_cast<qclab::QCircuit<T>*>(a->c.get()),
                     *static_cast<qclab::QCircuit<T>*>(b->c.get()));
}

}  // namespace

extern "C" {

int ref_num_threads(void) { return omp_get_max_threads(); }
void ref_set_num_threads(int n) { omp_set_num_threads(n); }

void* ref_circuit_create(int n, int dtype, const qsv_gate* gates, size_t count, int* status) {
  switch (dtype) {
    case QSV_C128: return make_circuit<std::complex<double>>(n, dtype, gates, count, status);
    case QSV_C64: return make_circuit<std::complex<float>>(n, dtype, gates, count, status);
    case QSV_F64: return make_circuit<double>(n, dtype, gates, count, status);
    case QSV_F32: return make_circuit<float>(n, dtype, gates, count, status);
  }
  *status = 1;
  return nullptr;
}

void ref_circuit_destroy(void* c) { delete static_cast<AnyCircuit*>(c); }

// QCircuit<T>(filename): the reference's own OpenQASM reader
// (include/qclab/QCircuit.hpp:82-93).
void* ref_circuit_from_qasm(const char* filename, int dtype, int* nbQubits) {
  switch (dtype) {
    case QSV_C128: {
      auto c = std::make_shared<qclab::QCircuit<std::complex<double>>>(std::string(filename));
      *nbQubits = c->nbQubits();
      return new AnyCircuit{dtype, c};
    }
    case QSV_C64: {
      auto c = std::make_shared<qclab::QCircuit<std::complex<float>>>(std::string(filename));
      *nbQubits = c->nbQubits();
      return new AnyCircuit{dtype, c};
    }
  }
  return nullptr;
}

int ref_circuit_nb_gates(void* c) {
  auto* ac = static_cast<AnyCircuit*>(c);
  if (ac->dtype == QSV_C128)
    return (int)static_cast<qclab::QCircuit<std::complex<double>>*>(ac->c.get())->nbGates();
  if (ac->dtype == QSV_C64)
    return (int)static_cast<qclab::QCircuit<std::complex<float>>*>(ac->c.get())->nbGates();
  return -1;
}

void* ref_vec_create(int dtype, uint64_t count) {
  auto* av = new AnyVec{dtype, nullptr, nullptr};
  switch (dtype) {
    case QSV_C128: { auto v = std::make_shared<std::vector<std::complex<double>>>(count); av->data = v->data(); av->v = v; break; }
    case QSV_C64: { auto v = std::make_shared<std::vector<std::complex<float>>>(count); av->data = v->data(); av->v = v; break; }
    case QSV_F64: { auto v = std::make_shared<std::vector<double>>(count); av->data = v->data(); av->v = v; break; }
    case QSV_F32: { auto v = std::make_shared<std::vector<float>>(count); av->data = v->data(); av->v = v; break; }
    default: delete av; return nullptr;
  }
  return av;
}

void* ref_vec_data(void* v) { return static_cast<AnyVec*>(v)->data; }
void ref_vec_destroy(void* v) { delete static_cast<AnyVec*>(v); }

// QCircuit<T>::apply(op, nbQubits, vector, offset) on the driver-owned vector.
int ref_circuit_apply(void* c, void* v, char op, int offset) {
  auto* ac = static_cast<AnyCircuit*>(c);
  auto* av = static_cast<AnyVec*>(v);
  if (ac->dtype != av->dtype) return 1;
  switch (ac->dtype) {
    case QSV_C128: return run<std::complex<double>>(ac, av, op, offset);
    case QSV_C64: return run<std::complex<float>>(ac, av, op, offset);
    case QSV_F64: return run<double>(ac, av, op, offset);
    case QSV_F32: return run<float>(ac, av, op, offset);
  }
  return 1;
}

int ref_circuit_apply_side(void* c, char side, char op, int nbQubits, int offset, void* data) {
  auto* ac = static_cast<AnyCircuit*>(c);
  switch (ac->dtype) {
    case QSV_C128: return run_side<std::complex<double>>(ac, side, op, nbQubits, offset, data);
    case QSV_C64: return run_side<std::complex<float>>(ac, side, op, nbQubits, offset, data);
    case QSV_F64: return run_side<double>(ac, side, op, nbQubits, offset, data);
    case QSV_F32: return run_side<float>(ac, side, op, nbQubits, offset, data);
  }
  return 1;
}

int ref_circuit_matrix(void* c, void* data) {
  auto* ac = static_cast<AnyCircuit*>(c);
  switch (ac->dtype) {
    case QSV_C128: return run_matrix<std::complex<double>>(ac, data);
    case QSV_C64: return run_matrix<std::complex<float>>(ac, data);
    case QSV_F64: return run_matrix<double>(ac, data);
    case QSV_F32: return run_matrix<float>(ac, data);
  }
  return 1;
}

// qclab::nrmF(circuit1, circuit2) (include/qclab/QCircuit.hpp:407-430).
double ref_nrmF(void* a, void* b) {
  auto* x = static_cast<AnyCircuit*>(a);
  auto* y = static_cast<AnyCircuit*>(b);
  if (x->dtype != y->dtype) return -1.0;
  switch (x->dtype) {
    case QSV_C128: return run_nrmf<std::complex<double>>(x, y);
    case QSV_C64: return run_nrmf<std::complex<float>>(x, y);
    case QSV_F64: return run_nrmf<double>(x, y);
    case QSV_F32: return run_nrmf<float>(x, y);
  }
  return -1.0;
}

}  // extern "C"

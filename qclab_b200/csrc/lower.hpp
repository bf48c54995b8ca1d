// Host-side lowering of qsv_gate records to amplitude-kernel launches.
//
// QCLAB++ maps every gate class to a (lambda, index loop) pair
// (src/qgates/apply.hpp:9-371).  Here each gate + op is lowered once, on the
// host, to one of six index shapes with its coefficients already rounded to
// the state's real type R, exactly as the reference lambdas compute them:
//
//   SH_PAIR  : 2x2 on (a, a|t)                 apply2    apply.hpp:259-272
//   SH_HALF  : x *= lambda on the t=1 half      apply2b   apply.hpp:275-287
//   SH_QUAD  : 4x4 on (a, a|b1, a|c1, a|b1|c1)  apply4    apply.hpp:290-308
//   SH_CPAIR : 2x2 on the target pair where control == state
//                                               apply4    apply.hpp:311-332
//   SH_CHALF : x *= lambda where control == state and target == 1
//                                               apply4b   apply.hpp:335-352
//   SH_SWAP  : swap (a|b1, a|c1), optionally times lambda
//                                               apply4bc  apply.hpp:355-371
//
// Matrices are stored row-major as (re, im) pairs.  Each PAIR/CPAIR/HALF/
// CHALF gate also carries its lambda's arithmetic form (ExactForm): a
// generic complex product m11*x1 + m12*x2, (ac - bd, ad + bc) without FMA,
// has the values of every specialised lambda, but its extra 0 * x terms can
// turn a -0 component into +0 where the lambda's own operations (Hadamard's
// real scaling, PauliX's swap, PauliZ's negation, ...) keep the sign; the
// kernels therefore evaluate each form as its lambda does.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include "qclab_b200.h"

namespace qsv {

enum Shape : int {
  SH_NONE = 0, SH_PAIR = 1, SH_HALF = 2, SH_QUAD = 3,
  SH_CPAIR = 4, SH_CHALF = 5, SH_SWAP = 6,
  SH_RED = 7   // gradient reduction w * Im(i^ny <lam| Pi P |psi>) (adjoint sweep)
};

// Arithmetic of a PAIR/CPAIR (a, b = rows 0, 1; x1, x2 = the pair) or
// HALF/CHALF gate as its reference lambda evaluates it (apply.hpp:9-128):
enum ExactForm : int {
  EF_GENERAL = 0,  // a = m11*x1 + m12*x2, b = m21*x1 + m22*x2 (lambda_QGate1);
                   // HALF: x *= lambda (Phase, Phase45, Phase90, CPhase)
  EF_HADAMARD,     // a = s*x1 + s*x2, b = s*x1 - s*x2, s real
  EF_ROTX,         // a = c*x1 + s*x2, b = s*x1 + c*x2, c real, s complex
  EF_ROTY,         // a = c*x1 + s1*x2, b = s2*x1 + c*x2, all real
  EF_DIAG,         // a = x1 * l1, b = x2 * l2 (RotationZ, CRotationZ)
  EF_SWAP,         // a = x2, b = x1 (PauliX, CX)
  EF_SWAP_MUL,     // a = x2 * l1, b = x1 * l2 (PauliY, CY)
  EF_NEG           // HALF: x = -x (PauliZ, CZ)
};

// Generator of a parametric gate for the adjoint gradient:
// d/dtheta U(theta) = c * Pi * P * U with P a Pauli string (flip mask f,
// sign mask zy, ny factors of Y) and Pi a projector onto index bits
// (pm, pv).  dE/dtheta = w * Im(i^ny <lam| Pi P |psi>) with
//   w = 1  for exp(-i theta/2 P) rotations (c = -i/2),
//   w = -2 for Phase/CPhase (c = i, P = I, Pi onto the |1> target).
struct Generator {
  uint64_t f = 0, zy = 0, pm = 0, pv = 0;
  int ny = 0;
  int w = 1;
};

// One lowered gate.  Bit positions are amplitude-index bits (qubit q of an
// n-qubit register is bit n-1-q).
struct Lowered {
  int shape = SH_NONE;
  int t0 = 0;      // PAIR/HALF/CPAIR/CHALF: target bit; QUAD/SWAP: bit of qubits[0]
  int t1 = 0;      // QUAD/SWAP: bit of qubits[1]; CPAIR/CHALF: control bit
  int cval = 1;    // control state
  int mul = 0;     // SWAP: multiply the swapped pair by lambda (iSWAP)
  int diag = 0;    // PAIR/CPAIR: matrix is diagonal (RotationZ-type)
  int form = EF_GENERAL;  // PAIR/CPAIR/HALF/CHALF: the lambda's arithmetic
  int real = 1;    // all coefficients have zero imaginary part
  double m[32];    // row-major complex coefficients (already rounded to R)
  int qubits[2] = {-1, -1};  // qubits touched (after offset), -1 if unused
  int param = -1;  // trainable parameter index of the source gate
  int kind = 0;    // source gate kind
  char op = 'N';
  Generator gen;   // SH_RED: the generator to reduce
  int slot = -1;   // SH_RED: output row
};

// Generator of gate g (qubits with offset) in an n-qubit register; returns
// false if the gate kind has no trainable angle.
inline bool generator_of(const qsv_gate& g, int offset, int n, Generator* out) {
  Generator G;
  auto bit = [n](int q) { return 1ull << (n - 1 - q); };
  const uint64_t a = bit(g.qubit0 + offset);
  switch (g.kind) {
    case QSV_ROTATION_X: G.f = a; break;
    case QSV_ROTATION_Y: G.f = a; G.zy = a; G.ny = 1; break;
    case QSV_ROTATION_Z: G.zy = a; break;
    case QSV_PHASE: G.pm = a; G.pv = a; G.w = -2; break;
    case QSV_ROTATION_XX:
    case QSV_ROTATION_YY:
    case QSV_ROTATION_ZZ: {
      const uint64_t ab = a | bit(g.qubit1 + offset);
      if (g.kind == QSV_ROTATION_XX) G.f = ab;
      if (g.kind == QSV_ROTATION_YY) { G.f = ab; G.zy = ab; G.ny = 2; }
      if (g.kind == QSV_ROTATION_ZZ) G.zy = ab;
      break;
    }
    case QSV_CROTATION_X:
    case QSV_CROTATION_Y:
    case QSV_CROTATION_Z:
    case QSV_CPHASE: {
      const uint64_t t = bit(g.qubit1 + offset);
      G.pm = a;
      G.pv = g.control_state ? a : 0;
      if (g.kind == QSV_CROTATION_X) G.f = t;
      if (g.kind == QSV_CROTATION_Y) { G.f = t; G.zy = t; G.ny = 1; }
      if (g.kind == QSV_CROTATION_Z) G.zy = t;
      if (g.kind == QSV_CPHASE) { G.pm |= t; G.pv |= t; G.w = -2; }
      break;
    }
    default:
      return false;
  }
  *out = G;
  return true;
}

inline bool valid_op(char op) { return op == 'N' || op == 'T' || op == 'C'; }

namespace detail {

template <typename R> struct C { R re, im; };

template <typename R>
inline C<R> cx(R re, R im) { return C<R>{re, im}; }

template <typename R>
inline C<R> conj(C<R> z) { return C<R>{z.re, -z.im}; }

// operateInPlace(op, A) for a dim x dim row-major matrix
// (include/qclab/dense/transpose.hpp:13-35): conjugate for 'C', then
// transpose for 'T' and 'C'.
template <typename R>
inline void operate(char op, C<R>* A, int dim) {
  if (op == 'N') return;
  if (op == 'C')
    for (int i = 0; i < dim * dim; ++i) A[i] = conj(A[i]);
  for (int i = 0; i < dim; ++i)
    for (int j = i + 1; j < dim; ++j) std::swap(A[i * dim + j], A[j * dim + i]);
}

template <typename R>
inline void store(Lowered* L, const C<R>* A, int count) {
  L->real = 1;
  for (int i = 0; i < count; ++i) {
    L->m[2 * i] = (double)A[i].re;
    L->m[2 * i + 1] = (double)A[i].im;
    if (A[i].im != R(0)) L->real = 0;
  }
}

// column-major (re,im) input matrix -> row-major C<R>, rounded to R
template <typename R>
inline void load_colmajor(const double* src, C<R>* A, int dim) {
  for (int r = 0; r < dim; ++r)
    for (int c = 0; c < dim; ++c) {
      const double* p = src + 2 * (r + c * dim);
      A[r * dim + c] = C<R>{(R)p[0], (R)p[1]};
    }
}

}  // namespace detail

// Lowers gate g (with op and qubit offset) for an n-qubit state of real
// type R.  `is_real` marks a real-valued state (float/double): gates whose
// coefficients are complex are rejected with QSV_ERROR_DTYPE, as QCLAB++
// only instantiates those gate classes for std::complex.
template <typename R>
inline qsv_status lower_gate(const qsv_gate& g, char op, int offset, int n,
                             bool is_real, Lowered* out) {
  using namespace detail;
  Lowered L;
  std::memset(L.m, 0, sizeof(L.m));
  L.kind = g.kind;
  L.param = g.param;
  L.op = op;
  if (!valid_op(op)) return QSV_ERROR_INVALID_VALUE;
  const R cs = (R)g.cos, sn = (R)g.sin;
  const R one = R(1), zero = R(0);
  auto bit = [n](int q) { return n - 1 - q; };
  auto check1 = [&](int q) { return q >= 0 && q < n; };

  const int k = g.kind;
  if (k < 0 || k >= QSV_NUM_GATE_KINDS) return QSV_ERROR_INVALID_VALUE;

  const bool one_qubit = (k <= QSV_MATRIX1);
  if (one_qubit) {
    const int q = g.qubit0 + offset;
    if (!check1(q)) return QSV_ERROR_QUBIT;
    L.qubits[0] = q;
    L.t0 = bit(q);
    C<R> A[4];
    switch (k) {
      case QSV_IDENTITY:
        L.shape = SH_NONE;
        *out = L;
        return QSV_SUCCESS;
      case QSV_HADAMARD: {  // lambda_Hadamard, apply.hpp:30-42
        const R s = R(1) / std::sqrt(R(2));
        A[0] = cx(s, zero); A[1] = cx(s, zero);
        A[2] = cx(s, zero); A[3] = cx(-s, zero);
        L.shape = SH_PAIR;
        L.form = EF_HADAMARD;
        break;
      }
      case QSV_PAULI_X:  // lambda_PauliX, apply.hpp:46-52
        A[0] = cx(zero, zero); A[1] = cx(one, zero);
        A[2] = cx(one, zero);  A[3] = cx(zero, zero);
        L.shape = SH_PAIR;
        L.form = EF_SWAP;
        break;
      case QSV_PAULI_Y: {  // lambda_PauliY, apply.hpp:56-68
        C<R> l1 = cx(zero, -one), l2 = cx(zero, one);
        if (op == 'T') std::swap(l1, l2);
        A[0] = cx(zero, zero); A[1] = l1;
        A[2] = l2;             A[3] = cx(zero, zero);
        L.shape = SH_PAIR;
        L.form = EF_SWAP_MUL;
        break;
      }
      case QSV_PAULI_Z:  // lambda_PauliZ + apply2b, apply.hpp:72-78
        A[0] = cx(-one, zero);
        L.shape = SH_HALF;
        L.form = EF_NEG;
        break;
      case QSV_ROTATION_X: {  // lambda_RotationX, apply.hpp:82-95
        C<R> s = cx(zero, -sn);
        if (op == 'C') s = conj(s);
        A[0] = cx(cs, zero); A[1] = s;
        A[2] = s;            A[3] = cx(cs, zero);
        L.shape = SH_PAIR;
        L.form = EF_ROTX;
        break;
      }
      case QSV_ROTATION_Y: {  // lambda_RotationY, apply.hpp:99-113
        R s1 = -sn, s2 = sn;
        if (op != 'N') std::swap(s1, s2);
        A[0] = cx(cs, zero); A[1] = cx(s1, zero);
        A[2] = cx(s2, zero); A[3] = cx(cs, zero);
        L.shape = SH_PAIR;
        L.form = EF_ROTY;
        break;
      }
      case QSV_ROTATION_Z: {  // lambda_RotationZ + apply2, apply.hpp:117-128
        C<R> l1 = cx(cs, -sn), l2 = cx(cs, sn);
        if (op == 'C') std::swap(l1, l2);
        A[0] = l1;             A[1] = cx(zero, zero);
        A[2] = cx(zero, zero); A[3] = l2;
        L.shape = SH_PAIR;
        L.diag = 1;
        L.form = EF_DIAG;
        break;
      }
      case QSV_PHASE: {  // lambda_Phase, apply.hpp:132-140
        C<R> l = cx(cs, sn);
        if (op == 'C') l = conj(l);
        A[0] = l;
        L.shape = SH_HALF;
        break;
      }
      case QSV_PHASE45: {  // lambda_Phase45, apply.hpp:144-155
        const R s = R(1) / std::sqrt(R(2));
        C<R> l = cx(s, s);
        if (op == 'C') l = conj(l);
        A[0] = l;
        L.shape = SH_HALF;
        break;
      }
      case QSV_PHASE90: {  // lambda_Phase90, apply.hpp:159-168
        C<R> l = cx(zero, one);
        if (op == 'C') l = conj(l);
        A[0] = l;
        L.shape = SH_HALF;
        break;
      }
      case QSV_MATRIX1: {  // lambda_QGate1, apply.hpp:11-26
        load_colmajor<R>(g.matrix, A, 2);
        operate<R>(op, A, 2);
        L.shape = SH_PAIR;
        break;
      }
      default:
        return QSV_ERROR_INVALID_VALUE;
    }
    store<R>(&L, A, L.shape == SH_PAIR ? 4 : 1);
    if (is_real && !L.real) return QSV_ERROR_DTYPE;
    *out = L;
    return QSV_SUCCESS;
  }

  // ---- 2-qubit gates -------------------------------------------------------
  if (n < 2) return QSV_ERROR_QUBIT;
  const int qa = g.qubit0 + offset, qb = g.qubit1 + offset;
  if (!check1(qa) || !check1(qb) || qa == qb) return QSV_ERROR_QUBIT;
  const bool controlled =
      (k >= QSV_CX && k <= QSV_CONTROLLED1);
  if (controlled) {
    if (g.control_state != 0 && g.control_state != 1)
      return QSV_ERROR_INVALID_VALUE;
    const int control = qa, target = qb;
    L.qubits[0] = std::min(control, target);
    L.qubits[1] = std::max(control, target);
    L.t0 = bit(target);
    L.t1 = bit(control);
    L.cval = g.control_state;
    C<R> A[4];
    int count = 4;
    switch (k) {
      case QSV_CX:  // CX.cpp:8-18: lambda_PauliX + apply4(ctrl)
        A[0] = cx(zero, zero); A[1] = cx(one, zero);
        A[2] = cx(one, zero);  A[3] = cx(zero, zero);
        L.shape = SH_CPAIR;
        L.form = EF_SWAP;
        break;
      case QSV_CY: {  // CY.cpp:8-18: lambda_PauliY + apply4(ctrl)
        C<R> l1 = cx(zero, -one), l2 = cx(zero, one);
        if (op == 'T') std::swap(l1, l2);
        A[0] = cx(zero, zero); A[1] = l1;
        A[2] = l2;             A[3] = cx(zero, zero);
        L.shape = SH_CPAIR;
        L.form = EF_SWAP_MUL;
        break;
      }
      case QSV_CZ:  // CZ.cpp:8-18: lambda_PauliZ + apply4b
        A[0] = cx(-one, zero);
        count = 1;
        L.shape = SH_CHALF;
        L.form = EF_NEG;
        break;
      case QSV_CPHASE: {  // CPhase.cpp:8-19: lambda_Phase + apply4b
        C<R> l = cx(cs, sn);
        if (op == 'C') l = conj(l);
        A[0] = l;
        count = 1;
        L.shape = SH_CHALF;
        break;
      }
      case QSV_CROTATION_X: {  // QControlledGate2.cpp:8-20 with RotationX::matrix
        A[0] = cx(cs, zero);   A[1] = cx(zero, -sn);
        A[2] = cx(zero, -sn);  A[3] = cx(cs, zero);
        operate<R>(op, A, 2);
        L.shape = SH_CPAIR;
        break;
      }
      case QSV_CROTATION_Y: {  // QControlledGate2.cpp:8-20 with RotationY::matrix
        A[0] = cx(cs, zero);   A[1] = cx(-sn, zero);
        A[2] = cx(sn, zero);   A[3] = cx(cs, zero);
        operate<R>(op, A, 2);
        L.shape = SH_CPAIR;
        break;
      }
      case QSV_CROTATION_Z: {  // CRotationZ.cpp:8-19: lambda_RotationZ + apply4(ctrl)
        C<R> l1 = cx(cs, -sn), l2 = cx(cs, sn);
        if (op == 'C') std::swap(l1, l2);
        A[0] = l1;             A[1] = cx(zero, zero);
        A[2] = cx(zero, zero); A[3] = l2;
        L.shape = SH_CPAIR;
        L.diag = 1;
        L.form = EF_DIAG;
        break;
      }
      case QSV_CONTROLLED1: {  // QControlledGate2.cpp:8-20
        load_colmajor<R>(g.matrix, A, 2);
        operate<R>(op, A, 2);
        L.shape = SH_CPAIR;
        break;
      }
      default:
        return QSV_ERROR_INVALID_VALUE;
    }
    store<R>(&L, A, count);
    if (is_real && !L.real) return QSV_ERROR_DTYPE;
    *out = L;
    return QSV_SUCCESS;
  }

  // uncontrolled 2-qubit gates: qubits sorted ascending (QRotationGate2.hpp:142-147,
  // SWAP.hpp:60-66); qubits[0] is the more significant bit.
  const int q0 = std::min(qa, qb), q1 = std::max(qa, qb);
  L.qubits[0] = q0;
  L.qubits[1] = q1;
  L.t0 = bit(q0);
  L.t1 = bit(q1);
  switch (k) {
    case QSV_SWAP: {  // SWAP.cpp:9-16: lambda_SWAP + apply4bc
      C<R> l = cx(one, zero);
      store<R>(&L, &l, 1);
      L.shape = SH_SWAP;
      L.mul = 0;
      break;
    }
    case QSV_ISWAP: {  // iSWAP.cpp:11-18: lambda_iSWAP + apply4bc
      C<R> l = cx(zero, one);
      if (op == 'C') l = cx(zero, -one);
      store<R>(&L, &l, 1);
      L.shape = SH_SWAP;
      L.mul = 1;
      break;
    }
    case QSV_ROTATION_XX:
    case QSV_ROTATION_YY:
    case QSV_ROTATION_ZZ:
    case QSV_MATRIX2: {  // QGate2.cpp:8-15: lambda_QGate2 + apply4
      C<R> A[16];
      const C<R> Z = cx(zero, zero);
      for (int i = 0; i < 16; ++i) A[i] = Z;
      if (k == QSV_ROTATION_XX) {  // RotationXX.hpp:136-143
        const C<R> d = cx(cs, zero), o = cx(zero, -sn);
        A[0] = d;  A[3] = o;  A[5] = d;  A[6] = o;
        A[9] = o;  A[10] = d; A[12] = o; A[15] = d;
      } else if (k == QSV_ROTATION_YY) {  // RotationYY.hpp:136-143
        const C<R> d = cx(cs, zero), o = cx(zero, sn), mo = cx(-zero, -sn);
        A[0] = d;   A[3] = o;  A[5] = d;  A[6] = mo;
        A[9] = mo;  A[10] = d; A[12] = o; A[15] = d;
      } else if (k == QSV_ROTATION_ZZ) {  // RotationZZ.hpp:136-143
        const C<R> a = cx(cs, -sn), b = cx(cs, sn);
        A[0] = a; A[5] = b; A[10] = b; A[15] = a;
      } else {
        // MatrixGate2: given in the kron basis |qubit0 qubit1>.  Reorder to
        // the basis of the sorted qubits, then to the amplitude order used
        // by apply4 (x1..x4 = |00>,|10>,|01>,|11> of (q0,q1)).
        C<R> K[16];
        load_colmajor<R>(g.matrix, K, 4);
        // kron index of basis state (bit of qubit0, bit of qubit1)
        // -> apply4 slot
        int slot_of[4];
        for (int s = 0; s < 4; ++s) {
          // slot s: bit(q0) = s & 1, bit(q1) = s >> 1
          const int bq0 = s & 1, bq1 = s >> 1;
          const int b_first = (qa == q0) ? bq0 : bq1;   // bit of qubit0
          const int b_second = (qa == q0) ? bq1 : bq0;  // bit of qubit1
          slot_of[s] = 2 * b_first + b_second;
        }
        for (int r = 0; r < 4; ++r)
          for (int c = 0; c < 4; ++c) A[r * 4 + c] = K[slot_of[r] * 4 + slot_of[c]];
      }
      operate<R>(op, A, 4);
      store<R>(&L, A, 16);
      L.shape = SH_QUAD;
      break;
    }
    default:
      return QSV_ERROR_INVALID_VALUE;
  }
  if (is_real && !L.real) return QSV_ERROR_DTYPE;
  *out = L;
  return QSV_SUCCESS;
}

// Applies op to a gate list: 'N' keeps the order, 'T'/'C' reverse it
// (include/qclab/QCircuit.hpp:130-143).
template <typename R>
inline qsv_status lower_list(const qsv_gate* gates, size_t count, char op,
                             int offset, int n, bool is_real, Lowered* out,
                             size_t* bad_index) {
  for (size_t i = 0; i < count; ++i) {
    const size_t src = (op == 'N') ? i : count - 1 - i;
    qsv_status st = lower_gate<R>(gates[src], op, offset, n, is_real, &out[i]);
    if (st != QSV_SUCCESS) {
      if (bad_index) *bad_index = src;
      return st;
    }
  }
  return QSV_SUCCESS;
}

}  // namespace qsv

// Host side of the gate-specialised stage engine (apply_gates.cu): op codes,
// the factorisation of lowered gates into cheap register-pass ops, the
// packed plan, and a host mirror of the device semantics (used by the CPU
// test tests/cpp/gate_plan_test.cpp).  Plain C++: no CUDA types.
//
// A stage (plan.hpp) is run tile by tile in shared memory, in register
// passes of R tile bits: each thread holds the 2^R amplitudes of one group
// in registers and applies the pass's ops to them.  Every op is one switch
// case whose register indices are compile-time (op kind x register
// positions), so an op costs its arithmetic plus one indirect branch.
//
// One-qubit gates are factored so that a gate costs two multiply-adds per
// amplitude component: a matrix c [[1, a], [b, 1]] is applied as
// (x1 + a x2, b x1 + x2) and the scalar c is multiplied into the stage's
// scale kappa, which the stage applies once at the end (kappa commutes with
// every gate).  The forms, by the structure of the lowered 2x2 matrix
// M = [[m00, m01], [m10, m11]] (QCLAB++'s lambdas, src/qgates/apply.hpp:11-128):
//   H       m00 = m01 = m10 = -m11          (x1 + x2, x1 - x2),          kappa *= m00
//   SHEAR   real, m00 = m11, |m00| largest  (x1 + a x2, b x1 + x2),      kappa *= m00
//   SHEARO  real, m01 = -m10, |m10| largest (a x1 - x2, x1 + b x2),      kappa *= m10
//   ISHEAR  RotationX-like, m00 = m11       (x1 + i a x2, i b x1 + x2),  kappa *= m00
//   ISHEARO RotationX-like, m01 = m10       (a x1 - i x2, -i x1 + b x2), kappa *= -Im m01
//   PHASE   diagonal                        x2 *= m11 / m00,             kappa *= m00
//   X, Z    PauliX swap, x2 = -x2
//   REAL2 / GEN2: any other real / complex 2x2 (no factoring).
// RotationY takes SHEAR or SHEARO and RotationX ISHEAR or ISHEARO, whichever
// keeps |a|, |b| <= 1; RotationZ is a PHASE with kappa = e^{-i theta/2}.
#pragma once

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#include "lower.hpp"
#include "plan.hpp"

namespace qsv {
namespace gx {

using cplx = std::complex<double>;

// one-qubit kinds (register position p)
enum Kind1 : int { G_H, G_SHEAR, G_SHEARO, G_ISHEAR, G_ISHEARO, G_PHASE, G_GEN2, G_REAL2, G_X,
                   G_Z, G_N1 };
// controlled kinds (target t, control c, control value cv): CX swaps the
// target pair, CGEN2 applies a complex 2x2 to it, CNEG negates and CPH
// multiplies by z the amplitudes with target 1 and control cv
enum Kind2 : int { G_CX, G_CGEN2, G_CNEG, G_CPH, G_N2 };
// two-qubit kinds on positions p0 > p1, slots (j, j|p0, j|p1, j|p0|p1):
// SWAP/ISWAP exchange slots 1 and 2 (ISWAP times z), GEN4 a 4x4 (row-major)
enum Kind4 : int { G_SWAP, G_ISWAP, G_GEN4, G_N4 };
// gradient terms of the two-vector (adjoint) sweeps at register position p:
// Im <lam| X_p |psi>, Re <lam| Y_p |psi> (= Im(i <lam|Y_p|psi>)) and
// Im <lam| Z_p |psi>, the derivatives of RotationX/Y/Z (lower.hpp:
// generator_of, weight 1, no projector); and G_RDG (position 0 only) for
// every other generator -- a Pauli string with flip mask f, sign mask zy and
// ny Y factors, a projector (pm, pv) and a weight w, all its bits in the pass:
//   w Im(i^ny sum_{j: (j & pm) == pv} conj(lam_j) (-1)^popc((j^f) & zy) psi_{j^f})
// with coefficients c[0] = (|kappa|^2 w, term index) and
// c[1] = (f | zy << 5 | pm << 10 | pv << 15 as register masks, ny).
enum KindR : int { G_RDX, G_RDY, G_RDZ, G_RDG, G_NR };

// Dense case codes for R register bits (holes where p = q are never used).
constexpr int code1(int R, int k, int p) { return k * R + p; }
constexpr int base2(int R) { return G_N1 * R; }
constexpr int code2(int R, int k, int t, int c, int cv) {
  return base2(R) + ((k * R + t) * R + c) * 2 + cv;
}
constexpr int base4(int R) { return base2(R) + G_N2 * R * R * 2; }
constexpr int code4(int R, int k, int p0, int p1) { return base4(R) + (k * R + p0) * R + p1; }
// x *= z for every register (the stage's kappa)
constexpr int code_scale(int R) { return base4(R) + G_N4 * R * R; }
constexpr int code_red(int R, int k, int p) { return code_scale(R) + 1 + k * R + p; }
constexpr int kCodeBits = 10;  // op word = code | coefficient index << kCodeBits
static_assert(code_red(5, G_NR, 0) < (1 << kCodeBits), "op codes exceed the code field");
constexpr int kMaxStageRed = 64;  // gradient terms per stage (shared-memory accumulators)

constexpr int kMaxR = 5;

// The device op word of the two-level dispatch: kind index (bits 0-4: the
// one-qubit kinds, then the controlled kinds, the two-qubit kinds and the
// scale), position index within the kind (bits 5-10) and coefficient index
// (bits 11-31).
constexpr int kKindBits = 5, kSubBits = 6, kWordCoefShift = kKindBits + kSubBits;
inline uint32_t device_word(int code, int R, uint32_t coef) {
  int kind, sub;
  if (code < base2(R)) {
    kind = code / R;
    sub = code % R;
  } else if (code < base4(R)) {
    const int r = code - base2(R);
    kind = G_N1 + (r >> 1) / (R * R);
    sub = r % (2 * R * R);
  } else if (code < code_scale(R)) {
    const int r = code - base4(R);
    kind = G_N1 + G_N2 + r / (R * R);
    sub = r % (R * R);
  } else if (code == code_scale(R)) {
    kind = G_N1 + G_N2 + G_N4;
    sub = 0;
  } else {
    const int r = code - code_red(R, 0, 0);
    kind = G_N1 + G_N2 + G_N4 + 1 + r / R;
    sub = r % R;
  }
  return (uint32_t)kind | ((uint32_t)sub << kKindBits) | (coef << kWordCoefShift);
}

// A register pass: R tile bits (local positions, ascending) and its ops
// (op words, stage-relative).
struct GxPass {
  int8_t pos[8];
  int32_t op0;
  int32_t nops;
};

struct GxStage {
  int m;
  int bits[64];
  size_t pass0, npasses, op0, nops, coef0, ncoef;
  size_t red0;  // gradient terms: red_slots[red0 .. red0 + nred)
  int nred;
};

struct GxPlan {
  int R = 4;
  std::vector<GxPass> passes;
  std::vector<uint32_t> ops;    // code | stage-relative coefficient index << kCodeBits
  std::vector<cplx> coefs;      // FP64; converted to the element type on upload
  std::vector<int32_t> red_slots;  // output row of each gradient term, by stage
  std::vector<GxStage> stages;
};

// ---- factorisation of one lowered gate --------------------------------------
struct GxOp {
  int code = 0;
  int ncoef = 0;
  cplx c[16];
};

inline bool is_real(cplx z) { return z.imag() == 0.0; }
inline bool is_imag(cplx z) { return z.real() == 0.0; }

// Coefficients are applied in the element's precision.  In float, a
// rounded coefficient would make a gate slightly non-unitary, and since the
// same gate acts on every amplitude the norm error is coherent: over
// thousands of gates it grows like a random walk (1e-6 over a 32-qubit brick
// of depth 100).  So the packer rounds first and compensates:
//   - a shear's scalar is derived from its rounded coefficient, which keeps
//     kappa [[1, t], [-t, 1]] (and the RotationX forms) exactly unitary;
//   - a phase is the float pair nearest to it with |z| closest to |z_exact|;
//   - the stage scale kappa carries its rounding error into the next stage.
inline double round_to(double x, bool f32) { return f32 ? (double)(float)x : x; }

// The float pair near z (a few ulps each way) whose modulus is closest to |z|.
inline cplx unit_round(cplx z, bool f32) {
  if (!f32) return z;
  const double target = std::abs(z);
  const float r0 = (float)z.real(), i0 = (float)z.imag();
  cplx best(r0, i0);
  double err = std::fabs(std::abs(best) - target);
  float r = r0;
  for (int a = 0; a < 8; ++a) r = std::nextafter(r, -INFINITY);
  for (int a = -8; a <= 8; ++a, r = std::nextafter(r, INFINITY)) {
    float im = i0;
    for (int b = 0; b < 8; ++b) im = std::nextafter(im, -INFINITY);
    for (int b = -8; b <= 8; ++b, im = std::nextafter(im, INFINITY)) {
      const cplx c((double)r, (double)im);
      const double e = std::fabs(std::abs(c) - target);
      if (e < err) {
        err = e;
        best = c;
      }
    }
  }
  return best;
}

// Appends the op of lowered gate L (register positions: target / first
// qubit p0, control / second qubit p1) and multiplies kappa by the scalar
// factored out.  Returns false for items the engine does not run (gradient
// reductions, misordered quads).
inline bool factor_gate(const Lowered& L, int R, int p0, int p1, std::vector<GxOp>* out,
                        cplx* kappa, bool f32 = false) {
  auto coef = [&](int i) { return cplx(L.m[2 * i], L.m[2 * i + 1]); };
  // scalar of a rotation-like shear with exact coefficient t, rounded to tr:
  // s * sqrt(1 + t^2) / sqrt(1 + tr^2) keeps s [[1, tr], [-tr, 1]] unitary
  // whenever s [[1, t], [-t, 1]] was
  auto shear_scale = [&](double s, double t, double tr) {
    return s * std::sqrt(1.0 + t * t) / std::sqrt(1.0 + tr * tr);
  };
  const cplx one(1.0, 0.0), zero(0.0, 0.0);
  GxOp op;
  switch (L.shape) {
    case SH_PAIR: {
      const cplx a = coef(0), b = coef(1), c = coef(2), d = coef(3);
      if (a == zero && d == zero && b == one && c == one) {
        op.code = code1(R, G_X, p0);
      } else if (b == zero && c == zero && a != zero) {
        if (a == one && d == -one) {
          op.code = code1(R, G_Z, p0);
        } else {
          op.code = code1(R, G_PHASE, p0);
          op.ncoef = 1;
          op.c[0] = unit_round((a == one) ? d : d / a, f32);
          *kappa *= a;
        }
      } else if (is_real(a) && is_real(b) && is_real(c) && is_real(d)) {
        const double ar = a.real(), br = b.real(), cr = c.real(), dr = d.real();
        if (ar != 0.0 && ar == br && ar == cr && ar == -dr) {
          op.code = code1(R, G_H, p0);
          *kappa *= ar;
        } else if (ar != 0.0 && ar == dr && std::fabs(ar) >= std::fabs(br) &&
                   std::fabs(ar) >= std::fabs(cr)) {
          op.code = code1(R, G_SHEAR, p0);
          op.ncoef = 1;
          const double t1 = br / ar, t2 = cr / ar;
          const double r1 = round_to(t1, f32), r2 = round_to(t2, f32);
          op.c[0] = cplx(r1, r2);
          *kappa *= (br == -cr) ? shear_scale(ar, t1, r1) : ar;
        } else if (cr != 0.0 && br == -cr && std::fabs(cr) >= std::fabs(ar) &&
                   std::fabs(cr) >= std::fabs(dr)) {
          op.code = code1(R, G_SHEARO, p0);
          op.ncoef = 1;
          const double g1 = ar / cr, g2 = dr / cr;
          const double r1 = round_to(g1, f32), r2 = round_to(g2, f32);
          op.c[0] = cplx(r1, r2);
          *kappa *= (ar == dr) ? shear_scale(cr, g1, r1) : cr;
        } else {
          op.code = code1(R, G_REAL2, p0);
          op.ncoef = 2;
          op.c[0] = cplx(ar, br);
          op.c[1] = cplx(cr, dr);
        }
      } else if (is_real(a) && is_real(d) && is_imag(b) && is_imag(c) && a.real() != 0.0 &&
                 a == d && std::fabs(a.real()) >= std::fabs(b.imag()) &&
                 std::fabs(a.real()) >= std::fabs(c.imag())) {
        op.code = code1(R, G_ISHEAR, p0);
        op.ncoef = 1;
        const double t1 = b.imag() / a.real(), t2 = c.imag() / a.real();
        const double r1 = round_to(t1, f32), r2 = round_to(t2, f32);
        op.c[0] = cplx(r1, r2);
        *kappa *= (b == c) ? shear_scale(a.real(), t1, r1) : a.real();
      } else if (is_real(a) && is_real(d) && is_imag(b) && is_imag(c) && b == c &&
                 b.imag() != 0.0 && std::fabs(b.imag()) >= std::fabs(a.real()) &&
                 std::fabs(b.imag()) >= std::fabs(d.real())) {
        const double s = -b.imag();
        op.code = code1(R, G_ISHEARO, p0);
        op.ncoef = 1;
        const double g1 = a.real() / s, g2 = d.real() / s;
        const double r1 = round_to(g1, f32), r2 = round_to(g2, f32);
        op.c[0] = cplx(r1, r2);
        *kappa *= (a == d) ? shear_scale(s, g1, r1) : s;
      } else {
        op.code = code1(R, G_GEN2, p0);
        op.ncoef = 4;
        for (int i = 0; i < 4; ++i) op.c[i] = coef(i);
      }
      break;
    }
    case SH_HALF: {
      const cplx l = coef(0);
      if (l == -one) {
        op.code = code1(R, G_Z, p0);
      } else {
        op.code = code1(R, G_PHASE, p0);
        op.ncoef = 1;
        op.c[0] = unit_round(l, f32);
      }
      break;
    }
    case SH_CPAIR: {
      const cplx a = coef(0), b = coef(1), c = coef(2), d = coef(3);
      if (a == zero && d == zero && b == one && c == one) {
        op.code = code2(R, G_CX, p0, p1, L.cval);
      } else if (a == one && b == zero && c == zero) {
        op.code = code2(R, d == -one ? G_CNEG : G_CPH, p0, p1, L.cval);
        if (d != -one) {
          op.ncoef = 1;
          op.c[0] = unit_round(d, f32);
        }
      } else {
        op.code = code2(R, G_CGEN2, p0, p1, L.cval);
        op.ncoef = 4;
        for (int i = 0; i < 4; ++i) op.c[i] = coef(i);
      }
      break;
    }
    case SH_CHALF: {
      const cplx l = coef(0);
      if (l == -one) {
        op.code = code2(R, G_CNEG, p0, p1, L.cval);
      } else {
        op.code = code2(R, G_CPH, p0, p1, L.cval);
        op.ncoef = 1;
        op.c[0] = unit_round(l, f32);
      }
      break;
    }
    case SH_SWAP: {
      if (p0 <= p1) return false;
      if (L.mul) {
        op.code = code4(R, G_ISWAP, p0, p1);
        op.ncoef = 1;
        op.c[0] = unit_round(coef(0), f32);
      } else {
        op.code = code4(R, G_SWAP, p0, p1);
      }
      break;
    }
    case SH_QUAD: {
      if (p0 <= p1) return false;
      op.code = code4(R, G_GEN4, p0, p1);
      op.ncoef = 16;
      for (int i = 0; i < 16; ++i) op.c[i] = coef(i);
      break;
    }
    default:
      return false;
  }
  out->push_back(op);
  return true;
}

// ---- host mirror of the device ops -------------------------------------------
// x: the 2^R registers of one group; c: the op's coefficients.
inline void host_apply_op(cplx* x, int R, uint32_t word, const cplx* c) {
  const int code = (int)(word & ((1u << kCodeBits) - 1u));
  const int N = 1 << R;
  const cplx I(0.0, 1.0);
  if (code < base2(R)) {
    const int k = code / R, p = code % R, mp = 1 << p;
    for (int j = 0; j < N; ++j) {
      if (j & mp) continue;
      const cplx a = x[j], b = x[j | mp];
      cplx y1 = a, y2 = b;
      switch (k) {
        case G_H: y1 = a + b; y2 = a - b; break;
        case G_SHEAR: y1 = a + c[0].real() * b; y2 = c[0].imag() * a + b; break;
        case G_SHEARO: y1 = c[0].real() * a - b; y2 = a + c[0].imag() * b; break;
        case G_ISHEAR: y1 = a + I * c[0].real() * b; y2 = I * c[0].imag() * a + b; break;
        case G_ISHEARO: y1 = c[0].real() * a - I * b; y2 = -I * a + c[0].imag() * b; break;
        case G_PHASE: y2 = c[0] * b; break;
        case G_GEN2: y1 = c[0] * a + c[1] * b; y2 = c[2] * a + c[3] * b; break;
        case G_REAL2:
          y1 = c[0].real() * a + c[0].imag() * b;
          y2 = c[1].real() * a + c[1].imag() * b;
          break;
        case G_X: y1 = b; y2 = a; break;
        case G_Z: y2 = -b; break;
      }
      x[j] = y1;
      x[j | mp] = y2;
    }
    return;
  }
  if (code < base4(R)) {
    const int r = code - base2(R);
    const int cv = r & 1, cb = (r >> 1) % R, t = ((r >> 1) / R) % R, k = (r >> 1) / (R * R);
    const int mt = 1 << t, mc = 1 << cb;
    for (int j = 0; j < N; ++j) {
      if ((j & mt) || ((j & mc) ? 1 : 0) != cv) continue;
      const cplx a = x[j], b = x[j | mt];
      switch (k) {
        case G_CX: x[j] = b; x[j | mt] = a; break;
        case G_CGEN2: x[j] = c[0] * a + c[1] * b; x[j | mt] = c[2] * a + c[3] * b; break;
        case G_CNEG: x[j | mt] = -b; break;
        case G_CPH: x[j | mt] = c[0] * b; break;
      }
    }
    return;
  }
  if (code < code_scale(R)) {
    const int r = code - base4(R);
    const int p1 = r % R, p0 = (r / R) % R, k = r / (R * R);
    const int m0 = 1 << p0, m1 = 1 << p1;
    for (int j = 0; j < N; ++j) {
      if ((j & m0) || (j & m1)) continue;
      const cplx s0 = x[j], s1 = x[j | m0], s2 = x[j | m1], s3 = x[j | m0 | m1];
      switch (k) {
        case G_SWAP: x[j | m0] = s2; x[j | m1] = s1; break;
        case G_ISWAP: x[j | m0] = c[0] * s2; x[j | m1] = c[0] * s1; break;
        case G_GEN4: {
          const cplx s[4] = {s0, s1, s2, s3};
          cplx y[4];
          for (int i = 0; i < 4; ++i)
            y[i] = c[4 * i] * s[0] + c[4 * i + 1] * s[1] + c[4 * i + 2] * s[2] +
                   c[4 * i + 3] * s[3];
          x[j] = y[0]; x[j | m0] = y[1]; x[j | m1] = y[2]; x[j | m0 | m1] = y[3];
          break;
        }
      }
    }
    return;
  }
  for (int j = 0; j < N; ++j) x[j] *= c[0];  // scale
}

// Two-vector mirror: a gradient term adds its value, times c[0].real(), to
// red[c[0].imag()]; every other op acts on both psi (x) and lambda (y).
// (c[0].real() = |kappa|^2 of the scalars factored out of the stage's
// earlier ops, which psi and lambda both still lack at that point.)
inline void host_apply_op2(cplx* x, cplx* y, int R, uint32_t word, const cplx* c, double* red) {
  const int code = (int)(word & ((1u << kCodeBits) - 1u));
  if (code <= code_scale(R)) {
    host_apply_op(x, R, word, c);
    host_apply_op(y, R, word, c);
    return;
  }
  const int r = code - code_red(R, 0, 0), k = r / R, p = r % R, mp = 1 << p;
  cplx s(0.0, 0.0);
  if (k == G_RDG) {
    const uint32_t pk = (uint32_t)c[1].real();
    const int f = pk & 31, zy = (pk >> 5) & 31, pm = (pk >> 10) & 31, pv = (pk >> 15) & 31;
    for (int j = 0; j < (1 << R); ++j)
      if ((j & pm) == pv)
        s += std::conj(y[j]) * ((__builtin_popcount((j ^ f) & zy) & 1) ? -1.0 : 1.0) * x[j ^ f];
    static const cplx ipow[4] = {cplx(1, 0), cplx(0, 1), cplx(-1, 0), cplx(0, -1)};
    red[(int)c[0].imag()] += c[0].real() * (ipow[(int)c[1].imag() & 3] * s).imag();
    return;
  }
  for (int j = 0; j < (1 << R); ++j) {
    const int f = (k == G_RDZ) ? j : (j ^ mp);
    double sg = 1.0;
    if (k == G_RDY) sg = ((f >> p) & 1) ? -1.0 : 1.0;
    if (k == G_RDZ) sg = ((j >> p) & 1) ? -1.0 : 1.0;
    s += std::conj(y[j]) * sg * x[f];
  }
  red[(int)c[0].imag()] += c[0].real() * ((k == G_RDY) ? s.real() : s.imag());
}

// ---- lane order ----------------------------------------------------------------
// The tile bits that a pass's register-group index g spreads over (all
// tile bits outside the pass), lowest g bit first, chosen so that the lanes
// of one shared-memory wavefront hit distinct banks.  With the XOR swizzle
// of stage_exec.cuh (16-byte unit u -> u ^ ((u>>3 ^ u>>6 ^ u>>9 ^ u>>12) & 7)),
// tile bit b of a 16-byte element lands on 16-byte slot bit b mod 3 of the
// 128-byte row, and of an 8-byte element (two per unit) on slot bit
// (b - 1) mod 3, bit 0 selecting the half.  A wavefront serves 8 lanes of
// 16-byte accesses (complex<double>, or complex<float> pairs when tile bit 0
// is a pass bit) or 16 lanes of 8-byte accesses: their 3 (or 4) lowest g
// bits should map to tile bits whose slot bits are distinct.
// `tma_swz` >= 0 selects the TMA layout instead (tma.cuh: u -> u ^ ((u >> 3)
// & (2^B - 1)), B = tma_swz): unit bits 0-2 are slot bits 0-2, unit bits
// 3 .. 3+B-1 fold into slot bits 0 .. B-1, the others give no distinct slot.
inline int lane_order(const int* pos, int R, int m, size_t elem_bytes, int* order,
                      int tma_swz = -1) {
  uint32_t pass = 0;
  for (int k = 0; k < R; ++k) pass |= 1u << pos[k];
  std::vector<int> rest;
  for (int b = 0; b < m; ++b)
    if (!((pass >> b) & 1u)) rest.push_back(b);
  const bool pairs = elem_bytes == 8 && (pass & 1u);
  auto slot = [&](int b) {
    const int ub = elem_bytes >= 16 ? b : b - 1;  // unit bit
    if (tma_swz < 0) return ub % 3;
    return ub < 3 ? ub : (ub - 3 < tma_swz ? ub - 3 : -1);
  };
  std::vector<int> first;
  if (elem_bytes == 8 && !pairs && !rest.empty() && rest[0] == 0) first.push_back(0);
  bool used[3] = {false, false, false};
  for (int b : rest) {
    if (b == 0 && elem_bytes == 8) continue;
    const int sl = slot(b);
    if (sl >= 0 && !used[sl]) {
      used[sl] = true;
      first.push_back(b);
    }
  }
  int k = 0;
  for (int b : first) order[k++] = b;
  for (int b : rest) {
    bool taken = false;
    for (int f : first) taken = taken || (f == b);
    if (!taken) order[k++] = b;
  }
  return k;
}

// ---- packing -----------------------------------------------------------------
// Plans `gates` (single-vector items) for an n-qubit state with tiles of 2^m
// amplitudes (`low` contiguous low bits) and register passes of R bits.
// Returns false if an item cannot run on this engine.
// With two_vector, gradient terms (SH_RED items of the adjoint's backward
// list) become RDX/RDY/RDZ ops, at most kMaxStageRed per stage.
inline bool pack_gate_plan(const std::vector<Lowered>& gates, int n, int m, int low, int R,
                           int max_gates, size_t plan_cap, size_t elem_bytes, GxPlan* out,
                           bool two_vector = false) {
  out->R = R;
  // every tile needs a bit outside its contiguous low bits unless it holds
  // the whole state
  if (m < R || R > kMaxR || (low >= m && m < n)) return false;
  for (const Lowered& L : gates)
    if (L.shape == SH_RED && !two_vector) return false;
  const std::vector<Stage> stages =
      plan_stages(gates, n, m, low, max_gates, two_vector ? kMaxStageRed : 0, plan_cap,
                  elem_bytes);
  const bool f32 = elem_bytes == 8;  // complex<float>: coefficients applied in float
  cplx carry(1.0, 0.0);  // rounding error of the stage scales so far (error feedback)
  std::vector<GxOp> ops;
  for (const Stage& stg : stages) {
    GxStage gs;
    gs.m = stg.m;
    for (int j = 0; j < 64; ++j) gs.bits[j] = (j < stg.m) ? stg.bits[j] : 0;
    gs.pass0 = out->passes.size();
    gs.op0 = out->ops.size();
    gs.coef0 = out->coefs.size();
    gs.red0 = out->red_slots.size();
    gs.nred = 0;
    int local_of[64];
    for (int j = 0; j < 64; ++j) local_of[j] = -1;
    for (int j = 0; j < stg.m; ++j) local_of[stg.bits[j]] = j;
    std::vector<uint32_t> op_bits;
    for (int gi : stg.gates) {
      const uint64_t g = gate_bits(gates[gi]);
      uint32_t lm = 0;
      for (int b = 0; b < n; ++b)
        if ((g >> b) & 1ull) lm |= 1u << local_of[b];
      op_bits.push_back(lm);
    }
    const std::vector<Pass> pl = plan_passes(op_bits, stg.m, R, true);
    cplx kappa(1.0, 0.0);
    for (size_t pi = 0; pi < pl.size(); ++pi) {
      const Pass& p = pl[pi];
      GxPass gp{};
      for (int k = 0; k < 8; ++k) gp.pos[k] = (k < p.r) ? (int8_t)p.pos[k] : 0;
      int reg_of[64];
      for (int j = 0; j < 64; ++j) reg_of[j] = -1;
      for (int k = 0; k < p.r; ++k) reg_of[p.pos[k]] = k;
      ops.clear();
      for (int oi : p.ops) {
        const Lowered& L = gates[stg.gates[oi]];
        if (L.shape == SH_RED) {
          if (gs.nred >= kMaxStageRed) return false;
          const Generator& g = L.gen;
          const uint64_t b = g.f | g.zy;
          const bool one = !g.pm && g.w == 1 && __builtin_popcountll(b) == 1;
          const bool x = one && g.f == b && g.zy == 0 && g.ny == 0;
          const bool y = one && g.f == b && g.zy == b && g.ny == 1;
          const bool z = one && g.f == 0 && g.zy == b && g.ny == 0;
          GxOp op;
          if (x || y || z) {  // coefficient: (|kappa|^2 so far, term index)
            const int r0 = reg_of[local_of[__builtin_ctzll(b)]];
            op.code = code_red(R, x ? G_RDX : (z ? G_RDZ : G_RDY), r0);
            op.ncoef = 1;
            op.c[0] = cplx(std::norm(kappa), (double)gs.nred++);
          } else {  // any other generator: its masks as register masks
            auto regmask = [&](uint64_t gm) {
              uint32_t r = 0;
              for (int q = 0; q < n; ++q)
                if ((gm >> q) & 1ull) r |= 1u << reg_of[local_of[q]];
              return r;
            };
            const uint32_t pk = regmask(g.f) | regmask(g.zy) << 5 | regmask(g.pm) << 10 |
                                regmask(g.pv) << 15;
            op.code = code_red(R, G_RDG, 0);
            op.ncoef = 2;
            op.c[0] = cplx(std::norm(kappa) * g.w, (double)gs.nred++);
            op.c[1] = cplx((double)pk, (double)(g.ny & 3));
          }
          ops.push_back(op);
          out->red_slots.push_back(L.slot);
          continue;
        }
        const bool one = L.shape == SH_PAIR || L.shape == SH_HALF;
        const int r0 = reg_of[local_of[L.t0]];
        const int r1 = one ? 0 : reg_of[local_of[L.t1]];
        if (!factor_gate(L, R, r0, r1, &ops, &kappa, f32)) return false;
      }
      if (pi + 1 == pl.size() && kappa != cplx(1.0, 0.0)) {
        GxOp sc;
        sc.code = code_scale(R);
        sc.ncoef = 1;
        const cplx want = kappa * carry;
        const cplx got(round_to(want.real(), f32), round_to(want.imag(), f32));
        sc.c[0] = got;
        if (got != cplx(0.0, 0.0)) carry = want / got;
        ops.push_back(sc);
      }
      gp.op0 = (int32_t)(out->ops.size() - gs.op0);
      gp.nops = (int32_t)ops.size();
      for (size_t i = 0; i < ops.size(); ++i) {
        const GxOp& o = ops[i];
        // ops without coefficients index entry 0 (the kernel loads every
        // op's first coefficient one op ahead)
        const size_t ci = o.ncoef ? out->coefs.size() - gs.coef0 : 0;
        if (ci >= (size_t(1) << (32 - kCodeBits))) return false;
        out->ops.push_back((uint32_t)o.code | ((uint32_t)ci << kCodeBits));
        for (int c = 0; c < o.ncoef; ++c) out->coefs.push_back(o.c[c]);
      }
      out->passes.push_back(gp);
    }
    gs.npasses = out->passes.size() - gs.pass0;
    gs.nops = out->ops.size() - gs.op0;
    if (out->coefs.size() == gs.coef0) out->coefs.push_back(cplx(0.0, 0.0));  // entry 0
    gs.ncoef = out->coefs.size() - gs.coef0;
    out->stages.push_back(gs);
  }
  return true;
}

// Host mirror of a whole plan on an n-qubit state (tests): stage by stage,
// tile by tile, pass by pass, exactly the order of the device kernel.  With
// lam (a second vector), every op acts on both and gradient terms add into
// rows[red_slots[...]].
inline void host_apply_plan(const GxPlan& P, int n, std::vector<cplx>& v,
                            std::vector<cplx>* lam = nullptr, double* rows = nullptr) {
  const int R = P.R;
  for (const GxStage& s : P.stages) {
    uint64_t S = 0;
    for (int j = 0; j < s.m; ++j) S |= 1ull << s.bits[j];
    std::vector<int> outside;
    for (int b = 0; b < n; ++b)
      if (!((S >> b) & 1ull)) outside.push_back(b);
    const uint64_t ntiles = 1ull << (n - s.m);
    std::vector<cplx> tile(size_t(1) << s.m), tile2(lam ? tile.size() : 0);
    std::vector<double> red(s.nred > 0 ? s.nred : 1, 0.0);
    for (uint64_t t = 0; t < ntiles; ++t) {
      uint64_t base = 0;
      for (size_t k = 0; k < outside.size(); ++k)
        if ((t >> k) & 1ull) base |= 1ull << outside[k];
      auto global = [&](uint32_t e) {
        uint64_t g = base;
        for (int j = 0; j < s.m; ++j)
          if ((e >> j) & 1u) g |= 1ull << s.bits[j];
        return g;
      };
      for (uint32_t e = 0; e < tile.size(); ++e) tile[e] = v[global(e)];
      if (lam)
        for (uint32_t e = 0; e < tile.size(); ++e) tile2[e] = (*lam)[global(e)];
      for (size_t pi = s.pass0; pi < s.pass0 + s.npasses; ++pi) {
        const GxPass& gp = P.passes[pi];
        uint32_t pm = 0;
        for (int k = 0; k < R; ++k) pm |= 1u << gp.pos[k];
        std::vector<int> rest;
        for (int j = 0; j < s.m; ++j)
          if (!((pm >> j) & 1u)) rest.push_back(j);
        cplx x[1 << kMaxR], y[1 << kMaxR];
        for (uint32_t g = 0; g < (1u << (s.m - R)); ++g) {
          uint32_t tb = 0;
          for (size_t k = 0; k < rest.size(); ++k)
            if ((g >> k) & 1u) tb |= 1u << rest[k];
          auto reg = [&](int j) {
            uint32_t e = tb;
            for (int k = 0; k < R; ++k)
              if ((j >> k) & 1) e |= 1u << gp.pos[k];
            return e;
          };
          for (int j = 0; j < (1 << R); ++j) x[j] = tile[reg(j)];
          if (lam)
            for (int j = 0; j < (1 << R); ++j) y[j] = tile2[reg(j)];
          for (int o = 0; o < gp.nops; ++o) {
            const uint32_t w = P.ops[s.op0 + gp.op0 + o];
            if (lam)
              host_apply_op2(x, y, R, w, P.coefs.data() + s.coef0 + (w >> kCodeBits), red.data());
            else
              host_apply_op(x, R, w, P.coefs.data() + s.coef0 + (w >> kCodeBits));
          }
          for (int j = 0; j < (1 << R); ++j) tile[reg(j)] = x[j];
          if (lam)
            for (int j = 0; j < (1 << R); ++j) tile2[reg(j)] = y[j];
        }
      }
      for (uint32_t e = 0; e < tile.size(); ++e) v[global(e)] = tile[e];
      if (lam)
        for (uint32_t e = 0; e < tile.size(); ++e) (*lam)[global(e)] = tile2[e];
    }
    if (rows)
      for (int r = 0; r < s.nred; ++r) rows[P.red_slots[s.red0 + r]] += red[r];
  }
}

}  // namespace gx
}  // namespace qsv

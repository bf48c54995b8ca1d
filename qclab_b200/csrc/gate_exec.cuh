// Device side of the gate-specialised register passes (gate_plan.hpp is
// the host side): in-place register primitives, the ops with compile-time
// register positions, the two-level op dispatch (gate_cases.inc) and the
// pass loop over a resident tile.  Used by the single-state stage kernel
// (apply_gates.cu) and the persistent batch kernel (batch.cu).
#pragma once
#include <cstdint>

#include "gate_plan.hpp"
#include "stage_exec.cuh"
#include "gate_cases.inc"

namespace qsv {
namespace gx {

using fx::align16;
using fx::copy_words;
using fx::ld_pair;
using fx::load_tile;
using fx::phys;
using fx::st_pair;
using fx::store_tile;

template <typename V> struct RealOf;
template <> struct RealOf<double2> { using T = double; };
template <> struct RealOf<float2> { using T = float; };

template <typename V, typename T>
__device__ __forceinline__ V mk(T a, T b) { return V{a, b}; }

// ---- in-place register primitives --------------------------------------------
// Each updates its "+" operands in place with one inline-PTX block (temporaries
// inside the block), so the amplitude registers keep their registers from op
// to op: written as plain C++, the switch's cases each produced new values
// that the compiler then copied back at the loop join, several moves per
// amplitude per op.
// (a + b, a - b) in two instructions and no move: b' = a - b, then
// a' = 2a - b' (= a + b up to the rounding of b', one more rounding error of
// the size of the other's)
__device__ __forceinline__ void ip_h(double& a, double& b) {
  asm("{\n .reg .f64 t;\n sub.rn.f64 %1, %0, %1;\n neg.f64 t, %1;\n"
      " fma.rn.f64 %0, %0, 0d4000000000000000, t;\n}"
      : "+d"(a), "+d"(b));
}
__device__ __forceinline__ void ip_h(float& a, float& b) {
  asm("{\n .reg .f32 t;\n sub.rn.f32 %1, %0, %1;\n neg.f32 t, %1;\n"
      " fma.rn.f32 %0, %0, 0f40000000, t;\n}"
      : "+f"(a), "+f"(b));
}
// (a + p b, q a + b)
__device__ __forceinline__ void ip_sh(double& a, double& b, double p, double q) {
  asm("{\n .reg .f64 t;\n fma.rn.f64 t, %2, %1, %0;\n fma.rn.f64 %1, %3, %0, %1;\n"
      " mov.f64 %0, t;\n}" : "+d"(a), "+d"(b) : "d"(p), "d"(q));
}
__device__ __forceinline__ void ip_sh(float& a, float& b, float p, float q) {
  asm("{\n .reg .f32 t;\n fma.rn.f32 t, %2, %1, %0;\n fma.rn.f32 %1, %3, %0, %1;\n"
      " mov.f32 %0, t;\n}" : "+f"(a), "+f"(b) : "f"(p), "f"(q));
}
// (p a - b, a + q b)
__device__ __forceinline__ void ip_sho(double& a, double& b, double p, double q) {
  asm("{\n .reg .f64 t, u;\n neg.f64 u, %1;\n fma.rn.f64 t, %2, %0, u;\n"
      " fma.rn.f64 %1, %3, %1, %0;\n mov.f64 %0, t;\n}" : "+d"(a), "+d"(b) : "d"(p), "d"(q));
}
__device__ __forceinline__ void ip_sho(float& a, float& b, float p, float q) {
  asm("{\n .reg .f32 t, u;\n neg.f32 u, %1;\n fma.rn.f32 t, %2, %0, u;\n"
      " fma.rn.f32 %1, %3, %1, %0;\n mov.f32 %0, t;\n}" : "+f"(a), "+f"(b) : "f"(p), "f"(q));
}
// (p a + b, q b - a)
__device__ __forceinline__ void ip_shop(double& a, double& b, double p, double q) {
  asm("{\n .reg .f64 t, u;\n fma.rn.f64 t, %2, %0, %1;\n neg.f64 u, %0;\n"
      " fma.rn.f64 %1, %3, %1, u;\n mov.f64 %0, t;\n}" : "+d"(a), "+d"(b) : "d"(p), "d"(q));
}
__device__ __forceinline__ void ip_shop(float& a, float& b, float p, float q) {
  asm("{\n .reg .f32 t, u;\n fma.rn.f32 t, %2, %0, %1;\n neg.f32 u, %0;\n"
      " fma.rn.f32 %1, %3, %1, u;\n mov.f32 %0, t;\n}" : "+f"(a), "+f"(b) : "f"(p), "f"(q));
}
// (re, im) *= (zr + i zi)
__device__ __forceinline__ void ip_cmul(double& re, double& im, double zr, double zi) {
  asm("{\n .reg .f64 t, u;\n mul.rn.f64 t, %3, %1;\n mul.rn.f64 u, %3, %0;\n neg.f64 t, t;\n"
      " fma.rn.f64 %0, %2, %0, t;\n fma.rn.f64 %1, %2, %1, u;\n}"
      : "+d"(re), "+d"(im) : "d"(zr), "d"(zi));
}
__device__ __forceinline__ void ip_cmul(float& re, float& im, float zr, float zi) {
  asm("{\n .reg .f32 t, u;\n mul.rn.f32 t, %3, %1;\n mul.rn.f32 u, %3, %0;\n neg.f32 t, t;\n"
      " fma.rn.f32 %0, %2, %0, t;\n fma.rn.f32 %1, %2, %1, u;\n}"
      : "+f"(re), "+f"(im) : "f"(zr), "f"(zi));
}
__device__ __forceinline__ void ip_swap(double& a, double& b) {
  asm("{\n .reg .f64 t;\n mov.f64 t, %0;\n mov.f64 %0, %1;\n mov.f64 %1, t;\n}"
      : "+d"(a), "+d"(b));
}
__device__ __forceinline__ void ip_swap(float& a, float& b) {
  asm("{\n .reg .f32 t;\n mov.f32 t, %0;\n mov.f32 %0, %1;\n mov.f32 %1, t;\n}"
      : "+f"(a), "+f"(b));
}
__device__ __forceinline__ void ip_neg(double& a) { asm("neg.f64 %0, %0;" : "+d"(a)); }
__device__ __forceinline__ void ip_neg(float& a) { asm("neg.f32 %0, %0;" : "+f"(a)); }

template <typename V>
__device__ __forceinline__ void ip_cmulv(V& x, const V& z) { ip_cmul(x.x, x.y, z.x, z.y); }
template <typename V>
__device__ __forceinline__ void ip_swapv(V& a, V& b) {
  ip_swap(a.x, b.x);
  ip_swap(a.y, b.y);
}
template <typename V>
__device__ __forceinline__ void ip_negv(V& a) {
  ip_neg(a.x);
  ip_neg(a.y);
}

// ---- ops (positions compile-time; x: the thread's N = 2^R registers) --------
template <int K, int P, typename V, int N>
__device__ __forceinline__ void op1(V (&x)[N], const V* __restrict__ c, const V cw) {
  using T = typename RealOf<V>::T;
  constexpr int M = 1 << P;
  T ca = T(0), cb = T(0);
  V c0{};
  if constexpr (K == G_SHEAR || K == G_SHEARO || K == G_ISHEAR || K == G_ISHEARO) {
    ca = cw.x;
    cb = cw.y;
  } else if constexpr (K == G_PHASE) {
    c0 = cw;
  }
#pragma unroll
  for (int j = 0; j < N; ++j) {
    if (j & M) continue;
    V& a = x[j];
    V& b = x[j | M];
    if constexpr (K == G_H) {
      ip_h(a.x, b.x);
      ip_h(a.y, b.y);
    } else if constexpr (K == G_SHEAR) {
      ip_sh(a.x, b.x, ca, cb);
      ip_sh(a.y, b.y, ca, cb);
    } else if constexpr (K == G_SHEARO) {
      ip_sho(a.x, b.x, ca, cb);
      ip_sho(a.y, b.y, ca, cb);
    } else if constexpr (K == G_ISHEAR) {
      // (a + i ca b, i cb a + b): shears of (a.re, b.im) and (a.im, b.re)
      ip_sh(a.x, b.y, -ca, cb);
      ip_sh(a.y, b.x, ca, -cb);
    } else if constexpr (K == G_ISHEARO) {
      // (ca a - i b, -i a + cb b)
      ip_shop(a.x, b.y, ca, cb);
      ip_sho(a.y, b.x, ca, cb);
    } else if constexpr (K == G_PHASE) {
      ip_cmulv(b, c0);
    } else if constexpr (K == G_GEN2) {  // coefficients read at their point of use
      const V y1 = fmac(fmul(fx::ld_use(c), a), fx::ld_use(c + 1), b);
      const V y2 = fmac(fmul(fx::ld_use(c + 2), a), fx::ld_use(c + 3), b);
      a = y1;
      b = y2;
    } else if constexpr (K == G_REAL2) {  // c[0] = (m00, m01), c[1] = (m10, m11)
      const V r0 = fx::ld_use(c), r1 = fx::ld_use(c + 1);
      const V y1 = mk<V>(fma(r0.x, a.x, r0.y * b.x), fma(r0.x, a.y, r0.y * b.y));
      const V y2 = mk<V>(fma(r1.x, a.x, r1.y * b.x), fma(r1.x, a.y, r1.y * b.y));
      a = y1;
      b = y2;
    } else if constexpr (K == G_X) {
      ip_swapv(a, b);
    } else if constexpr (K == G_Z) {
      ip_negv(b);
    }
  }
}

template <int K, int Pt, int Pc, int CV, typename V, int N>
__device__ __forceinline__ void op2(V (&x)[N], const V* __restrict__ c, const V cw) {
  constexpr int MT = 1 << Pt, MC = 1 << Pc;
  V c0{};
  if constexpr (K == G_CPH) c0 = cw;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    if ((j & MT) || (((j & MC) ? 1 : 0) != CV)) continue;
    V& a = x[j];
    V& b = x[j | MT];
    if constexpr (K == G_CX) {
      ip_swapv(a, b);
    } else if constexpr (K == G_CGEN2) {  // coefficients read at their point of use
      const V y1 = fmac(fmul(fx::ld_use(c), a), fx::ld_use(c + 1), b);
      const V y2 = fmac(fmul(fx::ld_use(c + 2), a), fx::ld_use(c + 3), b);
      a = y1;
      b = y2;
    } else if constexpr (K == G_CNEG) {
      ip_negv(b);
    } else if constexpr (K == G_CPH) {
      ip_cmulv(b, c0);
    }
  }
}

template <int K, int P0, int P1, typename V, int N>
__device__ __forceinline__ void op4(V (&x)[N], const V* __restrict__ c, const V cw) {
  constexpr int M0 = 1 << P0, M1 = 1 << P1;
  V z{};
  if constexpr (K == G_ISWAP) z = cw;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    if ((j & M0) || (j & M1)) continue;
    if constexpr (K == G_SWAP || K == G_ISWAP) {
      ip_swapv(x[j | M0], x[j | M1]);
      if constexpr (K == G_ISWAP) {
        ip_cmulv(x[j | M0], z);
        ip_cmulv(x[j | M1], z);
      }
    } else {
      // coefficients read at their point of use, so the 16 of them never
      // occupy registers together
      const V s0 = x[j], s1 = x[j | M0], s2 = x[j | M1], s3 = x[j | M0 | M1];
      V y[4];
#pragma unroll
      for (int r = 0; r < 4; ++r)
        y[r] = fmac(fmac(fmac(fmul(fx::ld_use(c + 4 * r), s0), fx::ld_use(c + 4 * r + 1), s1),
                         fx::ld_use(c + 4 * r + 2), s2),
                    fx::ld_use(c + 4 * r + 3), s3);
      x[j] = y[0]; x[j | M0] = y[1]; x[j | M1] = y[2]; x[j | M0 | M1] = y[3];
    }
  }
}

template <typename V, int N>
__device__ __forceinline__ void op_scale(V (&x)[N], const V* __restrict__ c, const V cw) {
  (void)c;
  const V z = cw;
#pragma unroll
  for (int j = 0; j < N; ++j) ip_cmulv(x[j], z);
}

// A gradient term of a two-vector sweep: c[0] = (|kappa|^2 pending in the
// stage, term index); the thread's sum over its registers of
//   RDX: conj(lam_j) psi_{j^p}             -> Im
//   RDY: conj(lam_j) (-1)^{bit p of j^p} psi_{j^p} -> Re  (= Im(i s))
//   RDZ: conj(lam_j) (-1)^{bit p of j} psi_j      -> Im
// in FP64, reduced over the warp into the term's shared-memory accumulator
// (stage_exec.cuh: red_accumulate).
// G_RDG: any generator, masks read from c[1] (gate_plan.hpp KindR).  The
// flip mask f selects one of 2^R compile-time variants (a switch), so the
// partner registers x[j ^ F] stay compile-time indices.
template <int F, typename V, int N>
__device__ __forceinline__ void red_generic_f(const V (&x)[N], const V (&y)[N], uint32_t zy,
                                              uint32_t pm, uint32_t pv, double& sr, double& si) {
#pragma unroll
  for (int j = 0; j < N; ++j) {
    if ((j & pm) != pv) continue;
    const double2 a = to_d2(y[j]), b = to_d2(x[j ^ F]);
    const double re = fma(a.x, b.x, a.y * b.y), im = fma(a.x, b.y, -a.y * b.x);
    if (__popc((j ^ F) & zy) & 1) {
      sr -= re;
      si -= im;
    } else {
      sr += re;
      si += im;
    }
  }
}

template <int F, typename V, int N>
__device__ __forceinline__ void red_generic_sel(uint32_t f, const V (&x)[N], const V (&y)[N],
                                                uint32_t zy, uint32_t pm, uint32_t pv, double& sr,
                                                double& si) {
  if constexpr (F < N) {
    if (f == F)
      red_generic_f<F>(x, y, zy, pm, pv, sr, si);
    else
      red_generic_sel<F + 1>(f, x, y, zy, pm, pv, sr, si);
  }
}

template <typename V, int N>
__device__ __forceinline__ void red_generic(const V (&x)[N], const V (&y)[N], const V* __restrict__ c,
                                            double* racc, unsigned lanes) {
  const double2 c0 = to_d2(c[0]), c1 = to_d2(c[1]);
  const uint32_t pk = (uint32_t)c1.x;
  const uint32_t f = pk & 31u, zy = (pk >> 5) & 31u, pm = (pk >> 10) & 31u, pv = (pk >> 15) & 31u;
  double sr = 0.0, si = 0.0;
  red_generic_sel<0>(f, x, y, zy, pm, pv, sr, si);
  // Im(i^ny s)
  const int ny = (int)c1.y & 3;
  const double v = ny == 0 ? si : ny == 1 ? sr : ny == 2 ? -si : -sr;
  fx::red_accumulate(c0.x * v, (int)c0.y, racc, lanes);
}

template <int K, int P, bool GEN, typename V, int N>
__device__ __forceinline__ void red_op(const V (&x)[N], const V (&y)[N], const V* __restrict__ c,
                                       const V cw, double* racc, unsigned lanes) {
  if constexpr (K == G_RDG) {  // only in the kernels built for stages that hold one
    if constexpr (GEN) red_generic(x, y, c, racc, lanes);
    else __builtin_unreachable();
    return;
  }
  constexpr int M = 1 << P;
  // only the part the term needs (RDY: Re, else Im), one independent signed
  // product per register, then a pairwise sum: a dependency chain of
  // log2(2^R) additions instead of 2^R (the sweep is latency-bound here).
  // complex<float>: products and this in-thread sum in float (the amplitudes
  // carry float rounding already; converting every operand to double cost
  // four conversions per register on the slow conversion pipe), one
  // conversion per term; the sums across lanes, tiles and the state are FP64.
  using T = typename RealOf<V>::T;
  T v[N];
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const int f = (K == G_RDZ) ? j : (j ^ M);
    const bool neg = (K == G_RDY) ? ((f & M) != 0) : (K == G_RDZ) ? ((j & M) != 0) : false;
    const V a = y[j], b = x[f];
    const T t = (K == G_RDY) ? fma(a.x, b.x, a.y * b.y) : fma(a.x, b.y, -a.y * b.x);
    v[j] = neg ? -t : t;
  }
#pragma unroll
  for (int h = 1; h < N; h <<= 1)
#pragma unroll
    for (int j = 0; j < N; j += 2 * h) v[j] += v[j + h];
  const double2 cc = to_d2(cw);
  fx::red_accumulate(cc.x * (double)v[0], (int)cc.y, racc, lanes);
}

// One op word (device_word in gate_plan.hpp): kind (bits 0-4), register
// position index (bits 5-10), coefficient index (bits 11-31); a two-level
// switch (gate_cases.inc).  cw = the op's first coefficient, loaded by the
// caller before the switch (every stage's coefficient table has at least one
// entry, and ops without coefficients index entry 0).  With NV = 2 every op acts on psi (x) and
// lambda (y) and gradient terms accumulate into racc.  GEN: the stage holds
// G_RDG terms (a separate kernel, whose extra registers the others do not pay).
template <typename V, int R, int NV, bool GEN>
__device__ __forceinline__ void apply_word(V (&x)[1 << R], V (&y)[1 << R], uint32_t w,
                                           const V cw, const V* __restrict__ cf, double* racc,
                                           unsigned lanes) {
  const V* __restrict__ c = cf + (w >> kWordCoefShift);
  const uint32_t kind = w & ((1u << kKindBits) - 1u);
  const uint32_t sub = (w >> kKindBits) & ((1u << kSubBits) - 1u);
#define GX1(f)                      \
  do {                              \
    f(x, c, cw);                        \
    if constexpr (NV == 2) f(y, c, cw); \
  } while (0)
#define GXR(K, P)                                                   \
  do {                                                              \
    if constexpr (NV == 2) red_op<K, P, GEN>(x, y, c, cw, racc, lanes); \
  } while (0)
  if constexpr (R == 3) {
    QSV_GX_NESTED_3
  } else if constexpr (R == 4) {
    QSV_GX_NESTED_4
  } else {
    static_assert(R == 5, "register passes of 3, 4 or 5 bits");
    QSV_GX_NESTED_5
  }
#undef GX1
#undef GXR
}

// ---- the stage kernel --------------------------------------------------------
// Device form of a register pass: its R tile bits, its ops, and
// boff[k] = phys(1 << pos[k]), so that the swizzled shared-memory index of
// register j is phys(tb) ^ XOR_{k in j} boff[k] (the swizzle is linear over
// GF(2) in the index bits).
// goff[k] = phys(1 << tile bit of group-index bit k) (lane_order), so the
// group's base is XOR_{k in g} goff[k].
struct GxPassDev {
  int8_t pos[8];
  int32_t op0;
  int32_t nops;
  uint32_t boff[8];
  uint32_t goff[12];
};
static_assert(sizeof(GxPassDev) == 96, "GxPassDev layout");


constexpr size_t kGxPlanCap = 16384;  // a stage's plan bytes in shared memory (bound)

// Bytes of a stage's plan staged in shared memory: passes | op words |
// coefficients, each section 16-byte aligned.
template <typename V>
inline size_t gx_plan_smem(size_t npasses, size_t nops, size_t ncoef) {
  return align16(npasses * sizeof(GxPassDev)) + align16(nops * sizeof(uint32_t)) +
         align16(ncoef * sizeof(V));
}

template <int R>
__device__ __forceinline__ uint32_t reg_off(uint32_t ptb, const uint32_t (&boff)[R], int j) {
  uint32_t o = ptb;
#pragma unroll
  for (int k = 0; k < R; ++k)
    if ((j >> k) & 1) o ^= boff[k];
  return o;
}

// The register passes of one stage on resident tiles t0 (and t1 with
// NV = 2) of 2^m amplitudes: per pass, every register group of 2^R
// amplitudes is loaded, the pass's ops are applied in order, and it is
// stored back; a block barrier ends each pass.  Threads beyond the 2^(m-R)
// groups idle in the passes (they still reach every barrier), and gradient
// terms reduce over the lanes that hold groups.
template <typename V, int R, int NV, bool GEN>
__device__ __forceinline__ void run_gate_passes(V* t0, V* t1, const GxPassDev* passes,
                                                int npasses, const uint32_t* ops,
                                                const V* coefs, double* racc, int m) {
  constexpr int N = 1 << R;
  const uint32_t ngroups = 1u << (m - R);
  const unsigned lanes = min(min(ngroups, (uint32_t)blockDim.x), 32u);
  for (int pi = 0; pi < npasses; ++pi) {
    const GxPassDev& P = passes[pi];
    uint32_t boff[R];
#pragma unroll
    for (int k = 0; k < R; ++k) boff[k] = P.boff[k];
    const int op0 = P.op0, nops = P.nops;
    // 8-byte elements with tile bit 0 in the pass: registers 2i and 2i+1 are
    // the two halves of one 16-byte unit, moved as one access
    const bool pairs = sizeof(V) == 8 && P.pos[0] == 0;
    const int gbits = m - R;
    for (uint32_t g = threadIdx.x; g < ngroups; g += blockDim.x) {
      uint32_t ptb = 0;
      for (int k = 0; k < gbits; ++k)
        if ((g >> k) & 1u) ptb ^= P.goff[k];
      V x[N], y[N];
      // register j sits at ptb ^ XOR_{k in j} boff[k]; recomputed for the
      // store rather than held across the ops
      if (pairs) {
#pragma unroll
        for (int j = 0; j < N; j += 2) {
          const uint32_t o = reg_off<R>(ptb, boff, j);
          ld_pair(t0 + o, x[j], x[j + 1]);
          if (NV == 2) ld_pair(t1 + o, y[j], y[j + 1]);
        }
      } else {
#pragma unroll
        for (int j = 0; j < N; ++j) {
          const uint32_t o = reg_off<R>(ptb, boff, j);
          x[j] = t0[o];
          if (NV == 2) y[j] = t1[o];
        }
      }
      for (int o = 0; o < nops; ++o) {
        const uint32_t w = ops[op0 + o];
        apply_word<V, R, NV, GEN>(x, y, w, coefs[w >> kWordCoefShift], coefs, racc, lanes);
      }
      // the store recomputes the offsets: without this the compiler keeps
      // all 2^R of them live across the ops for reuse, which costs registers
      // the amplitudes need
      asm volatile("" : "+r"(ptb));
#pragma unroll
      for (int k = 0; k < R; ++k) asm volatile("" : "+r"(boff[k]));
      if (pairs) {
#pragma unroll
        for (int j = 0; j < N; j += 2) {
          const uint32_t o = reg_off<R>(ptb, boff, j);
          st_pair(t0 + o, x[j], x[j + 1]);
          if (NV == 2) st_pair(t1 + o, y[j], y[j + 1]);
        }
      } else {
#pragma unroll
        for (int j = 0; j < N; ++j) {
          const uint32_t o = reg_off<R>(ptb, boff, j);
          t0[o] = x[j];
          if (NV == 2) t1[o] = y[j];
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace gx
}  // namespace qsv

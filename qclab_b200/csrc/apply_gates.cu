// Gate-specialised stage kernel for single-vector complex sweeps
// (complex<double> and complex<float> states).
//
// Same stage/tile structure as the other fused engines (plan.hpp,
// stage_exec.cuh): one 2^m-amplitude tile per CTA is copied into shared
// memory (16-byte cp.async, XOR-swizzled layout), the stage's register
// passes run on it, and it is written back.  What differs is the op
// application (gate_plan.hpp): every op is one case of a switch on a dense
// code (kind x register positions, gate_cases.inc), so its register indices
// are compile-time, and one-qubit gates are factored to two multiply-adds
// per amplitude component with their scalar folded into the stage's kappa.
// A brick layer's RotationX/RotationY/Hadamard therefore costs 2 FMAs or
// adds per component, RotationZ a complex multiply on half the amplitudes,
// CNOT register moves and CZ sign flips -- against 16 FMAs per component for
// a dense 3-bit pass of the tensor-core engine.
//
// Arithmetic is FMA-contracted in the element's precision (the fused path's
// contract: within 1e-12 of the reference-exact path for complex<double>).
#include <algorithm>
#include <cstring>
#include <vector>

#include "fused.hpp"
#include "gate_plan.hpp"
#include "stage_exec.cuh"
#include "tma.cuh"
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
  double sr = 0.0, si = 0.0;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const int f = (K == G_RDZ) ? j : (j ^ M);
    const bool neg = (K == G_RDY) ? ((f & M) != 0) : (K == G_RDZ) ? ((j & M) != 0) : false;
    const double2 a = to_d2(y[j]), b = to_d2(x[f]);
    const double re = fma(a.x, b.x, a.y * b.y), im = fma(a.x, b.y, -a.y * b.x);
    if (neg) {
      sr -= re;
      si -= im;
    } else {
      sr += re;
      si += im;
    }
  }
  const double2 cc = to_d2(cw);
  fx::red_accumulate(cc.x * ((K == G_RDY) ? sr : si), (int)cc.y, racc, lanes);
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

struct GxArgs {
  TileArgs ta;
  int npasses, nops, ncoef;
  const GxPassDev* passes;
  const uint32_t* ops;
  const void* coefs;  // V
  int vec16;
  // two-vector sweeps: the stage's gradient terms -> partial[slot][tile]
  int nred;
  const int32_t* red_slots;
  double* partial;
  // tile staging by TMA (tma.use; maps passed beside) or 16-byte cp.async
  TmaGeo tma;
  unsigned* wait_error;  // set when a bounded wait for the tile gave up
  uint32_t smem_bytes;   // dynamic shared memory of the launch
};

template <int R>
__device__ __forceinline__ uint32_t reg_off(uint32_t ptb, const uint32_t (&boff)[R], int j) {
  uint32_t o = ptb;
#pragma unroll
  for (int k = 0; k < R; ++k)
    if ((j >> k) & 1) o ^= boff[k];
  return o;
}

template <typename V, int R, int NT, int MINB, int NV, bool GEN = false>
__global__ void __launch_bounds__(NT, MINB)
    k_gates(V* __restrict__ v0, V* __restrict__ v1, GxArgs a,
            const __grid_constant__ CUtensorMap tm0, const __grid_constant__ CUtensorMap tm1) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  __shared__ uint64_t tile_bar;
  // the tiles start on a 1024-byte boundary (the TMA swizzle blocks; the
  // launch reserves the padding)
  unsigned char* smem_raw = tma::align1024(smem_dyn);
  const uint32_t size = 1u << a.ta.m;
  V* t0 = reinterpret_cast<V*>(smem_raw);
  V* t1 = t0 + size;
  // two-vector sweeps: the gradient terms' per-warp accumulators after the
  // tiles; then the stage's plan, copied once per CTA: passes | op words |
  // coefficients
  double* racc = reinterpret_cast<double*>(smem_raw + size_t(NV) * size * sizeof(V));
  unsigned char* pp = smem_raw + size_t(NV) * size * sizeof(V) + (NV == 2 ? fx::kRaccBytes : 0);
  unsigned char* po = pp + align16(size_t(a.npasses) * sizeof(GxPassDev));
  unsigned char* pc = po + align16(size_t(a.nops) * sizeof(uint32_t));
  const uint64_t base = tile_base(a.ta, blockIdx.x);
  if (a.tma.use) {  // one thread starts the tile's copies; they land while the plan is copied
    if (!tma::tile_fits<NV>(a.tma, smem_dyn, t0, size * sizeof(V), a.smem_bytes, a.wait_error))
      return;
    tma::tile_start<NV>(a.tma, &tm0, &tm1, t0, t1, base, &tile_bar);
  }
  copy_words(pp, a.passes, size_t(a.npasses) * sizeof(GxPassDev));
  copy_words(po, a.ops, size_t(a.nops) * sizeof(uint32_t));
  copy_words(pc, a.coefs, size_t(a.ncoef) * sizeof(V));
  if (NV == 2)
    for (int i = threadIdx.x; i < a.nred * fx::kRedWarps; i += blockDim.x) racc[i] = 0.0;
  const GxPassDev* passes = reinterpret_cast<const GxPassDev*>(pp);
  const uint32_t* ops = reinterpret_cast<const uint32_t*>(po);
  const V* coefs = reinterpret_cast<const V*>(pc);
  if (a.tma.use) {
    if (!tma::tile_wait(&tile_bar, a.wait_error, tma::kTileWaitLimit)) return;
  } else {
    load_tile<V, NV>(v0, v1, t0, t1, a.ta, base, a.vec16);
    __syncthreads();
  }
  constexpr int N = 1 << R;
  const uint32_t ngroups = size >> R;
  const unsigned lanes = blockDim.x < 32u ? blockDim.x : 32u;
  for (int pi = 0; pi < a.npasses; ++pi) {
    const GxPassDev& P = passes[pi];
    uint32_t boff[R];
#pragma unroll
    for (int k = 0; k < R; ++k) boff[k] = P.boff[k];
    const int op0 = P.op0, nops = P.nops;
    // 8-byte elements with tile bit 0 in the pass: registers 2i and 2i+1 are
    // the two halves of one 16-byte unit, moved as one access
    const bool pairs = sizeof(V) == 8 && P.pos[0] == 0;
    const int gbits = a.ta.m - R;
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
  if (a.tma.use) {
    tma::tile_store<NV>(a.tma, &tm0, &tm1, t0, t1, base);
  } else {
    store_tile<V, NV>(v0, v1, t0, t1, a.ta, base, a.vec16);
  }
  if (NV == 2) {  // the last pass ended with a barrier: racc is complete
    const int warps = fx::red_warps();
    for (int r = threadIdx.x; r < a.nred; r += blockDim.x) {
      double t = 0.0;
      for (int w = 0; w < warps; ++w) t += racc[r * fx::kRedWarps + w];
      a.partial[(size_t)a.red_slots[r] * gridDim.x + blockIdx.x] = t;
    }
  }
}

// Launch shapes.  A thread holds 2^R amplitudes per vector (64 registers
// for complex<double> with R = 4, whose op switch needs ~186 registers in
// all), so single-vector complex<double> runs CTAs of 128 threads, three per
// SM by default at 168 registers (two with qsv_fuse_opts.ctas_per_sm = 2:
// measured 26 % slower on a 30-qubit brick of depth 40, 1186 against
// 881 ms); complex<float> with R = 4 runs 256-thread CTAs, three per SM
// (two on request), with R = 5 two 128-thread CTAs (three on request:
// measured even).  Two-vector sweeps hold
// 2 x 2^R amplitudes: R = 3 for complex<double>, 4 for complex<float>, in
// 128-thread CTAs, three per SM (166 registers).  Each thread takes ngroups / threads
// register groups per pass.
template <typename V> struct GxKernels;
template <> struct GxKernels<double2> {
  static void* get(int R, int ctas, int nv, bool gen = false) {
    if (nv == 2)
      return gen ? (void*)k_gates<double2, 3, 128, 3, 2, true> : (void*)k_gates<double2, 3, 128, 3, 2>;
    return ctas == 2 ? (void*)k_gates<double2, 4, 128, 2, 1>
                     : (void*)k_gates<double2, 4, 128, 3, 1>;
  }
  static int threads(int R, int nv) { (void)R; (void)nv; return 128; }
};
template <> struct GxKernels<float2> {
  static void* get(int R, int ctas, int nv, bool gen = false) {
    if (nv == 2)
      return gen ? (void*)k_gates<float2, 4, 128, 3, 2, true> : (void*)k_gates<float2, 4, 128, 3, 2>;
    if (R == 5)
      return ctas == 3 ? (void*)k_gates<float2, 5, 128, 3, 1> : (void*)k_gates<float2, 5, 128, 2, 1>;
    return ctas == 2 ? (void*)k_gates<float2, 4, 256, 2, 1> : (void*)k_gates<float2, 4, 256, 3, 1>;
  }
  static int threads(int R, int nv) { return (nv == 2 || R == 5) ? 128 : 256; }
};

template <typename V> V to_elem(cplx z);
template <> double2 to_elem<double2>(cplx z) { return make_double2(z.real(), z.imag()); }
template <> float2 to_elem<float2>(cplx z) {
  return make_float2((float)z.real(), (float)z.imag());
}

constexpr size_t kGxPlanCap = 16384;  // a stage's plan bytes in shared memory (bound)

template <typename V>
size_t gx_plan_smem(size_t npasses, size_t nops, size_t ncoef) {
  return align16(npasses * sizeof(GxPassDev)) + align16(nops * sizeof(uint32_t)) +
         align16(ncoef * sizeof(V));
}

}  // namespace gx

int gate_pass_bits(size_t elem_bytes, const qsv_fuse_opts* opts, int nv) {
  // two vectors: 3 bits (complex<double>) or 4 (complex<float>); one vector:
  // 4 bits, or 5 for complex<float> with reg_bits = 5
  if (nv == 2) return elem_bytes >= 16 ? 3 : 4;
  if (elem_bytes >= 16) return 4;
  return (opts && opts->reg_bits == 4) ? 4 : 5;
}

namespace {

qsv_status pack_gates_for(const std::vector<Lowered>& items, int n, int m, int low, int R,
                          int max_gates, size_t elem_bytes, gx::GxPlan* plan, int nv) {
  if (!gx::pack_gate_plan(items, n, m, low, R, max_gates, gx::kGxPlanCap, elem_bytes, plan,
                          nv == 2))
    return QSV_ERROR_NOT_SUPPORTED;
  return QSV_SUCCESS;
}

}  // namespace

template <typename V>
qsv_status execute_gates(const ExecArgs& x, int m, int low, int max_gates, bool vec16) {
  using namespace gx;
  qsv_state_s* s = x.s;
  const int n = s->n;
  const int nv = x.nv;
  const int R = gate_pass_bits(sizeof(V), x.opts, nv);
  if (m < R + 1) return QSV_ERROR_NOT_SUPPORTED;
  GxPlan plan;
  if (qsv_status st = pack_gates_for(*x.items, n, m, low, R, max_gates, sizeof(V), &plan, nv))
    return st;
  if (nv == 2 && x.nslots > 0 && x.partial_bytes < (size_t)x.nslots * (1ull << (n - m)) * sizeof(double))
    return fail(QSV_ERROR_SIZE, "partial-sum buffer too small");
  if (plan.stages.empty()) return QSV_SUCCESS;
  // tile staging per stage: TMA maps where the tile fits one (both vectors
  // share the geometry), else cp.async; the shared-memory layout, and so the
  // passes' offsets, follow the choice
  const bool want_tma = !(x.opts && x.opts->tile_copy == 1);
  std::vector<CUtensorMap> maps(plan.stages.size() * 2);
  std::vector<TmaGeo> geos(plan.stages.size());
  for (size_t si = 0; si < plan.stages.size(); ++si) {
    const GxStage& gs = plan.stages[si];
    geos[si] = TmaGeo{};
    if (!want_tma) continue;
    if (!tma_stage_map(gs.bits, gs.m, n, sizeof(V), x.v0, &maps[2 * si], &geos[si])) continue;
    if (nv == 2 && !tma_stage_map(gs.bits, gs.m, n, sizeof(V), x.v1, &maps[2 * si + 1],
                                  &geos[si]))
      geos[si] = TmaGeo{};
  }
  std::vector<GxPassDev> dpass(plan.passes.size());
  std::vector<uint64_t> runoff;
  std::vector<size_t> run0;
  for (size_t si = 0; si < plan.stages.size(); ++si) {
    const GxStage& gs = plan.stages[si];
    const bool tma = geos[si].use != 0;
    auto phys = [&](uint32_t e) {
      return tma ? phys_tma_host(e, fx::Units<V>::per, geos[si].swz)
                 : fx::phys_host(e, fx::Units<V>::per);
    };
    for (size_t pi = gs.pass0; pi < gs.pass0 + gs.npasses; ++pi) {
      const GxPass& gp = plan.passes[pi];
      GxPassDev& d = dpass[pi];
      d = GxPassDev{};
      for (int k = 0; k < 8; ++k) d.pos[k] = gp.pos[k];
      d.op0 = gp.op0;
      d.nops = gp.nops;
      for (int k = 0; k < R; ++k) d.boff[k] = phys(1u << gp.pos[k]);
      int order[32];
      int pos[8];
      for (int k = 0; k < 8; ++k) pos[k] = gp.pos[k];
      const int ng = lane_order(pos, R, gs.m, sizeof(V), order, tma ? geos[si].swz : -1);
      if (ng > 12) return fail(QSV_ERROR_SIZE, "gate stage of %d tile bits", gs.m);
      for (int k = 0; k < ng; ++k) d.goff[k] = phys(1u << order[k]);
    }
    run0.push_back(runoff.size());
    tile_runoffs(gs.bits, gs.m, low, &runoff);
  }
  auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
  const size_t pass_bytes = dpass.size() * sizeof(GxPassDev);
  const size_t op_off = align(pass_bytes);
  const size_t coef_off = align(op_off + plan.ops.size() * sizeof(uint32_t));
  const size_t run_off = align(coef_off + plan.coefs.size() * sizeof(V));
  const size_t red_off = align(run_off + runoff.size() * sizeof(uint64_t));
  const size_t total = red_off + plan.red_slots.size() * sizeof(int32_t);
  std::vector<unsigned char> host(total);
  std::memcpy(host.data(), dpass.data(), pass_bytes);
  uint32_t* hw = reinterpret_cast<uint32_t*>(host.data() + op_off);
  for (size_t i = 0; i < plan.ops.size(); ++i) {
    const uint32_t w = plan.ops[i];
    hw[i] = device_word((int)(w & ((1u << kCodeBits) - 1u)), R, w >> kCodeBits);
  }
  V* hc = reinterpret_cast<V*>(host.data() + coef_off);
  for (size_t i = 0; i < plan.coefs.size(); ++i) hc[i] = to_elem<V>(plan.coefs[i]);
  std::memcpy(host.data() + run_off, runoff.data(), runoff.size() * sizeof(uint64_t));
  if (!plan.red_slots.empty())
    std::memcpy(host.data() + red_off, plan.red_slots.data(),
                plan.red_slots.size() * sizeof(int32_t));
  if (qsv_status st = ensure_scratch(s, total)) return st;
  unsigned char* dev = static_cast<unsigned char*>(s->scratch);
  if (qsv_status st = cuda_status(cudaMemcpyAsync(dev, host.data(), total, cudaMemcpyHostToDevice,
                                                  s->stream), "gate plan upload"))
    return st;
  // two-vector stages with generic gradient terms (G_RDG) run the kernel
  // built with them
  const int ctas = x.opts ? x.opts->ctas_per_sm : 0;
  const uint32_t rdg = (uint32_t)code_red(R, G_RDG, 0);
  std::vector<char> stage_gen(plan.stages.size(), 0);
  for (size_t si = 0; si < plan.stages.size(); ++si) {
    const GxStage& gs = plan.stages[si];
    for (size_t o = gs.op0; o < gs.op0 + gs.nops; ++o)
      if ((plan.ops[o] & ((1u << kCodeBits) - 1u)) == rdg) stage_gen[si] = 1;
  }
  for (bool gen : {false, true}) {
    if (gen && nv != 2) break;
    if (qsv_status st = cuda_status(cudaFuncSetAttribute(GxKernels<V>::get(R, ctas, nv, gen),
                                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                         200 * 1024),
                                    "gate stage shared-memory attribute"))
      return st;
  }
  const uint64_t ntiles = 1ull << (n - m);
  if (x.ntiles_out) *x.ntiles_out = ntiles;
  const unsigned threads =
      (unsigned)std::min<uint64_t>((uint64_t)GxKernels<V>::threads(R, nv), 1ull << (m - R));
  unsigned* wait_error = sweep_wait_flag();
  if (!wait_error) return fail(QSV_ERROR_CUDA, "sweep wait flag unavailable");
  StageTimer timer(x.opts && x.opts->profile, plan.stages.size(), s->stream);
  if (qsv_status st = timer.start()) return st;
  V* p0 = static_cast<V*>(x.v0);
  V* p1 = static_cast<V*>(x.v1);
  for (size_t si = 0; si < plan.stages.size(); ++si) {
    const GxStage& gs = plan.stages[si];
    GxArgs a;
    a.nred = gs.nred;
    a.red_slots = reinterpret_cast<const int32_t*>(dev + red_off) + gs.red0;
    a.partial = x.partial;
    a.ta.n = n;
    a.ta.m = gs.m;
    a.ta.low = low;
    for (int j = 0; j < 64; ++j) a.ta.bits[j] = (int8_t)gs.bits[j];
    a.ta.runoff = reinterpret_cast<const uint64_t*>(dev + run_off) + run0[si];
    a.npasses = (int)gs.npasses;
    a.nops = (int)gs.nops;
    a.ncoef = (int)gs.ncoef;
    a.passes = reinterpret_cast<const GxPassDev*>(dev) + gs.pass0;
    a.ops = reinterpret_cast<const uint32_t*>(dev + op_off) + gs.op0;
    a.coefs = dev + coef_off + gs.coef0 * sizeof(V);
    a.vec16 = vec16 ? 1 : 0;
    a.tma = geos[si];
    a.wait_error = wait_error;
    // + 1024: the tiles are placed on a 1024-byte boundary
    const size_t smem = (size_t(1) << gs.m) * sizeof(V) * nv + (nv == 2 ? fx::kRaccBytes : 0) +
                        gx_plan_smem<V>(gs.npasses, gs.nops, gs.ncoef) + 1024;
    if (smem > 200 * 1024)
      return fail(QSV_ERROR_SIZE, "gate stage needs %zu bytes of shared memory", smem);
    a.smem_bytes = (uint32_t)smem;
    void* args[] = {&p0, &p1, &a, &maps[2 * si], &maps[2 * si + (nv == 2 ? 1 : 0)]};
    void* kern = GxKernels<V>::get(R, ctas, nv, nv == 2 && stage_gen[si]);
    if (qsv_status st = cuda_status(cudaLaunchKernel(kern, dim3((unsigned)ntiles), dim3(threads),
                                                     args, smem, s->stream),
                                    "gate stage launch"))
      return st;
    count_launch();
    if (a.tma.use) count_tma_launch();
    if (qsv_status st = timer.mark(si)) return st;
  }
  if (qsv_status st = timer.finish()) return st;
  return nv == 2 && x.nslots > 0 ? reduce_rows(x, ntiles) : QSV_SUCCESS;
}

template qsv_status execute_gates<double2>(const ExecArgs&, int, int, int, bool);
template qsv_status execute_gates<float2>(const ExecArgs&, int, int, int, bool);

qsv_status gate_plan_counts(const std::vector<Lowered>& items, int n, int m, int low,
                            const qsv_fuse_opts* opts, int max_gates, size_t elem_bytes,
                            std::vector<int>* ops, std::vector<int>* passes) {
  gx::GxPlan plan;
  if (qsv_status st = pack_gates_for(items, n, m, low, gate_pass_bits(elem_bytes, opts, 1),
                                     max_gates, elem_bytes, &plan, 1))
    return st;
  for (const gx::GxStage& gs : plan.stages) {
    ops->push_back((int)gs.nops);
    passes->push_back((int)gs.npasses);
  }
  return QSV_SUCCESS;
}

}  // namespace qsv

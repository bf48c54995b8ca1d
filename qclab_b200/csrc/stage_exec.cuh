// Device and host building blocks of the fused stage executor, shared by the
// per-state sweep (apply_fused.cu) and the batched persistent kernel
// (batch.cu).
//
// A stage (plan.hpp) is executed tile by tile: the 2^m amplitudes of a tile
// are copied into shared memory (16-byte cp.async into an XOR-swizzled
// layout), the stage's register passes run on them -- each thread gathers
// the 2^R amplitudes of one assignment of the other tile bits into
// registers, applies the pass's ops, scatters them back -- and the tile is
// written back.  Ops are specialised by the structure of their coefficients
// (permutation, diagonal, real, RotationX-like) and use FMA contraction.
#pragma once

#include <cstdint>
#include <cstring>
#include <vector>
#include "common.cuh"
#include "internal.hpp"
#include "plan.hpp"
#include "tile.cuh"

// Build-time choices of the stage kernel (all variants are correct; they
// differ in instruction count and register pressure).
#ifndef QSV_CTL_STATIC      // CNOT/CZ positions as template parameters
#define QSV_CTL_STATIC 0
#endif
#ifndef QSV_PRECOMP_OFF     // pass offsets precomputed on the host
#define QSV_PRECOMP_OFF 1
#endif
// Measured on a B200 (brick circuits, 30 qubits complex<double> and 32
// qubits complex<float>, plan staged in shared memory): complex<double> runs
// fastest with 16 amplitudes per thread at 2 CTAs per SM (8 per thread: 5 %
// slower at 2 CTAs, 20 % at 3, where it spills); complex<float> with 16 per
// thread at 3 CTAs per SM (32 per thread at 2 CTAs: even).
#ifndef QSV_RBITS_C128      // register bits of a complex<double> pass
#define QSV_RBITS_C128 4
#endif
#ifndef QSV_RBITS_C64       // register bits of a complex<float> (or real) pass
#define QSV_RBITS_C64 4
#endif
#ifndef QSV_MINBLOCKS_C128  // CTAs per SM the complex<double> stage kernel targets
#define QSV_MINBLOCKS_C128 2
#endif
#ifndef QSV_MINBLOCKS_C64   // the same for complex<float> and real elements
#define QSV_MINBLOCKS_C64 3
#endif
// A register pass whose ops (no gradient terms) number at least
// QSV_DENSE_MIN_OPS is multiplied out on the host into one dense 2^R x 2^R
// matrix (P_DENSE) when R <= QSV_DENSE_MAX_R: 2^R complex MACs per amplitude
// in place of the ops' dispatch and predicates.  0 disables.
#ifndef QSV_DENSE_MIN_OPS
#define QSV_DENSE_MIN_OPS 3
#endif
#ifndef QSV_DENSE_MAX_R
#define QSV_DENSE_MAX_R 3
#endif
// Tile bits per register pass of the tensor-core engine (2 or 3).
#ifndef QSV_DMMA_BITS
#define QSV_DMMA_BITS 3
#endif
// Tensor-core plans: each pass's bits chosen to absorb the most ops (1) or
// greedily in circuit order (0).
#ifndef QSV_DENSE_SEARCH
#define QSV_DENSE_SEARCH 1
#endif
// Tensor-core plans with unset low_bits: also plan one more low bit and keep
// the plan with fewer passes (1), or keep the default (0).
#ifndef QSV_DENSE_LOW_SEARCH
#define QSV_DENSE_LOW_SEARCH 1
#endif
#ifndef QSV_TURN_BITS_C128  // log2 register groups per thread and pass (complex<double>)
#define QSV_TURN_BITS_C128 0
#endif

namespace qsv {
namespace fx {

enum Form : int8_t {
  F_GENERIC = 0,  // dense complex 2x2 / 4x4
  F_PERM = 1,     // [[0,1],[1,0]] (pairs) / swap of the |10>,|01> slots (quads)
  F_DIAG = 2,     // diagonal
  F_REAL = 3,     // all entries real
  F_RXLIKE = 4,   // real diagonal, imaginary off-diagonal
  F_NEG = 5       // P_MUL by -1 on one control/target pattern (CZ)
};

enum POpShape : int8_t { P_PAIR = 1, P_CPAIR = 2, P_MUL = 3, P_QUAD = 4, P_RED = 5, P_DENSE = 6 };
// POp.form of a P_DENSE op: the structure of its matrix U (exact zeros of
// the FP64 product), which the tensor-core kernel uses to skip MMAs
constexpr int8_t kDenseGeneral = 0, kDenseReal = 1, kDenseDiagonal = 2;

// One op of a register pass; positions index the pass's register bits.
struct POp {
  int8_t shape;
  int8_t form;
  int8_t p0, p1;    // PAIR/CPAIR: p0 target, p1 control; QUAD: p0 > p1; RED: flip positions
  int8_t cval;      // CPAIR control value
  int8_t nflip;     // RED: flip bits (0, 1, 2)
  int8_t ny, w;     // RED
  int8_t mul;       // QUAD/F_PERM: multiply the swapped slots by the coefficient
  uint8_t mmask, mval;  // MUL: x *= c where (j & mmask) == mval; RED: projector
  uint8_t zy;       // RED: sign mask
  int16_t coef;     // stage-relative index of the first coefficient
  int16_t ridx;     // RED: index among the stage's reductions (< kMaxRed)
  int32_t slot;     // RED: output row
};

// Gradient reductions of a stage accumulate per warp in shared memory,
// racc[ridx * kRedWarps + warp] (a warp-shuffle sum, no block barrier), and
// are summed over the warps once per tile or stage in a fixed order.
constexpr int kMaxRed = 64;    // reductions per stage (the planner's cap)
constexpr int kRedWarps = 8;   // warps of a 256-thread block
constexpr size_t kRaccBytes = size_t(kMaxRed) * kRedWarps * sizeof(double);

// `lanes` (a power of two <= 32) threads of the warp take part: fewer than
// 32 only when the block, or its working part, is smaller than a warp.
__device__ __forceinline__ void red_accumulate(double v, int ridx, double* racc, unsigned lanes) {
  const unsigned mask = lanes >= 32 ? 0xffffffffu : ((1u << lanes) - 1u);
  for (unsigned o = 16; o > 0; o >>= 1)
    if (o < lanes) v += __shfl_xor_sync(mask, v, o);
  if ((threadIdx.x & 31) == 0) racc[ridx * kRedWarps + (threadIdx.x >> 5)] += v;
}

__device__ __forceinline__ int red_warps() { return (int)((blockDim.x + 31) >> 5); }



struct PassDev {
  int8_t pos[8];    // local tile bits of the pass, ascending
  int32_t op0;      // first op (stage-relative)
  int32_t nops;
  // shared-memory offset (swizzled element index) of register j's pattern:
  // phys(tb | pattern(j)) = phys(tb) ^ off[j] because the swizzle is linear
  // over GF(2) in the index bits
  uint16_t off[32];
};

static_assert(sizeof(PassDev) == 80, "PassDev layout");
static_assert(sizeof(POp) == 20, "POp layout");

// A stage's plan (pass descriptors, ops, coefficients) is copied into shared
// memory once per CTA: every thread reads every op and coefficient, and from
// global memory those reads were the kernel's main latency stall.  The
// planner keeps a stage's plan within kPlanSmemMax bytes.
constexpr size_t kPlanSmemMax = 16384;

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

template <typename V>
__host__ __device__ inline size_t plan_smem_bytes(int npasses, int nops, int ncoef) {
  return align16(size_t(npasses) * sizeof(PassDev)) + align16(size_t(nops) * sizeof(POp)) +
         align16(size_t(ncoef) * sizeof(V));
}

// Copies `bytes` (a multiple of 4) from global to shared memory.
__device__ __forceinline__ void copy_words(void* dst, const void* src, size_t bytes) {
  uint32_t* d = static_cast<uint32_t*>(dst);
  const uint32_t* s = static_cast<const uint32_t*>(src);
  for (size_t i = threadIdx.x; i < bytes / 4; i += blockDim.x) d[i] = __ldg(s + i);
}

// Stages the plan at `dst` (16-byte aligned); returns the three section
// pointers.  The caller synchronises the block before use.
template <typename V>
__device__ __forceinline__ void stage_plan(unsigned char* dst, const PassDev* passes, int npasses,
                                           const POp* ops, int nops, const V* coefs, int ncoef,
                                           const PassDev** sp, const POp** so, const V** sc) {
  unsigned char* pp = dst;
  unsigned char* po = pp + align16(size_t(npasses) * sizeof(PassDev));
  unsigned char* pc = po + align16(size_t(nops) * sizeof(POp));
  copy_words(pp, passes, size_t(npasses) * sizeof(PassDev));
  copy_words(po, ops, size_t(nops) * sizeof(POp));
  copy_words(pc, coefs, size_t(ncoef) * sizeof(V));
  *sp = reinterpret_cast<const PassDev*>(pp);
  *so = reinterpret_cast<const POp*>(po);
  *sc = reinterpret_cast<const V*>(pc);
}

// Host copy of the swizzle (see phys<V> below) for `epu` elements per unit.
inline uint32_t phys_host(uint32_t e, uint32_t epu) {
  const uint32_t u = e / epu;
  const uint32_t su = u ^ (((u >> 3) ^ (u >> 6) ^ (u >> 9) ^ (u >> 12)) & 7u);
  return su * epu + (e % epu);
}

__device__ __forceinline__ uint32_t ins0(uint32_t x, int p) {
  return ((x >> p) << (p + 1)) | (x & ((1u << p) - 1u));
}

// ---- 2x2 application with coefficient-structure specialisation -----------
template <int FORM>
__device__ __forceinline__ void pair2f(const double2* c, double2& x1, double2& x2) {
  if (FORM == F_PERM) { const double2 t = x1; x1 = x2; x2 = t; }
  else if (FORM == F_DIAG) { x1 = fmul(c[0], x1); x2 = fmul(c[3], x2); }
  else if (FORM == F_REAL) {
    const double a = c[0].x, b = c[1].x, d = c[2].x, e = c[3].x;
    const double2 y1 = make_double2(fma(a, x1.x, b * x2.x), fma(a, x1.y, b * x2.y));
    const double2 y2 = make_double2(fma(d, x1.x, e * x2.x), fma(d, x1.y, e * x2.y));
    x1 = y1; x2 = y2;
  } else if (FORM == F_RXLIKE) {
    // y1 = a*x1 + i*b*x2, y2 = i*d*x1 + e*x2 (a,e real; b,d imaginary parts)
    const double a = c[0].x, b = c[1].y, d = c[2].y, e = c[3].x;
    const double2 y1 = make_double2(fma(a, x1.x, -b * x2.y), fma(a, x1.y, b * x2.x));
    const double2 y2 = make_double2(fma(e, x2.x, -d * x1.y), fma(e, x2.y, d * x1.x));
    x1 = y1; x2 = y2;
  } else {
    const double2 y1 = fmac(fmul(c[0], x1), c[1], x2);
    const double2 y2 = fmac(fmul(c[2], x1), c[3], x2);
    x1 = y1; x2 = y2;
  }
}
template <int FORM>
__device__ __forceinline__ void pair2f(const float2* c, float2& x1, float2& x2) {
  if (FORM == F_PERM) { const float2 t = x1; x1 = x2; x2 = t; }
  else if (FORM == F_DIAG) { x1 = fmul(c[0], x1); x2 = fmul(c[3], x2); }
  else if (FORM == F_REAL) {
    const float a = c[0].x, b = c[1].x, d = c[2].x, e = c[3].x;
    const float2 y1 = make_float2(fmaf(a, x1.x, b * x2.x), fmaf(a, x1.y, b * x2.y));
    const float2 y2 = make_float2(fmaf(d, x1.x, e * x2.x), fmaf(d, x1.y, e * x2.y));
    x1 = y1; x2 = y2;
  } else if (FORM == F_RXLIKE) {
    const float a = c[0].x, b = c[1].y, d = c[2].y, e = c[3].x;
    const float2 y1 = make_float2(fmaf(a, x1.x, -b * x2.y), fmaf(a, x1.y, b * x2.x));
    const float2 y2 = make_float2(fmaf(e, x2.x, -d * x1.y), fmaf(e, x2.y, d * x1.x));
    x1 = y1; x2 = y2;
  } else {
    const float2 y1 = fmac(fmul(c[0], x1), c[1], x2);
    const float2 y2 = fmac(fmul(c[2], x1), c[3], x2);
    x1 = y1; x2 = y2;
  }
}
template <int FORM, typename R>
__device__ __forceinline__ void pair2f(const R* c, R& x1, R& x2) {
  if (FORM == F_PERM) { const R t = x1; x1 = x2; x2 = t; return; }
  const R y1 = fma(c[0], x1, c[1] * x2);
  const R y2 = fma(c[2], x1, c[3] * x2);
  x1 = y1; x2 = y2;
}

__device__ __forceinline__ double2 vneg(double2 x) { return make_double2(-x.x, -x.y); }
__device__ __forceinline__ float2 vneg(float2 x) { return make_float2(-x.x, -x.y); }
__device__ __forceinline__ double vneg(double x) { return -x; }
__device__ __forceinline__ float vneg(float x) { return -x; }

__device__ __forceinline__ double2 scale1(const double2 c, double2 x) { return fmul(c, x); }
__device__ __forceinline__ float2 scale1(const float2 c, float2 x) { return fmul(c, x); }
__device__ __forceinline__ double scale1(const double c, double x) { return c * x; }
__device__ __forceinline__ float scale1(const float c, float x) { return c * x; }

__device__ __forceinline__ double2 mac(double2 acc, double2 c, double2 x) { return fmac(acc, c, x); }
__device__ __forceinline__ float2 mac(float2 acc, float2 c, float2 x) { return fmac(acc, c, x); }
__device__ __forceinline__ double mac(double acc, double c, double x) { return fma(c, x, acc); }
__device__ __forceinline__ float mac(float acc, float c, float x) { return fmaf(c, x, acc); }

// ---- register-pass ops ----------------------------------------------------
// Pairs (j, j | 1<<P) of the 2^R registers whose control bits match
// (CTRL = false: every pair, no test).
template <typename V, int R, int P, int FORM, bool CTRL>
__device__ __forceinline__ void pair_reg(V (&x)[1 << R], const V* c, uint32_t cm, uint32_t cv) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (!((j >> P) & 1) && (!CTRL || ((j & cm) == cv))) pair2f<FORM>(c, x[j], x[j | (1 << P)]);
}

template <typename V, int R, int P, bool CTRL>
__device__ __forceinline__ void pair_forms(V (&x)[1 << R], int form, const V* c, uint32_t cm,
                                           uint32_t cv) {
  switch (form) {
    case F_PERM: pair_reg<V, R, P, F_PERM, CTRL>(x, c, cm, cv); break;
    case F_DIAG: pair_reg<V, R, P, F_DIAG, CTRL>(x, c, cm, cv); break;
    case F_REAL: pair_reg<V, R, P, F_REAL, CTRL>(x, c, cm, cv); break;
    case F_RXLIKE: pair_reg<V, R, P, F_RXLIKE, CTRL>(x, c, cm, cv); break;
    default: pair_reg<V, R, P, F_GENERIC, CTRL>(x, c, cm, cv); break;
  }
}

template <typename V, int R, bool CTRL, int P = 0>
__device__ __forceinline__ void pair_dispatch(V (&x)[1 << R], int p, int form, const V* c,
                                              uint32_t cm, uint32_t cv) {
  if constexpr (P < R) {
    if (p == P) pair_forms<V, R, P, CTRL>(x, form, c, cm, cv);
    else pair_dispatch<V, R, CTRL, P + 1>(x, p, form, c, cm, cv);
  }
}

// Controlled swap (CNOT) with target P, control Q, control value CV all
// compile-time: a pure renaming of registers, no instructions.
template <typename V, int R, int P, int Q, int CV>
__device__ __forceinline__ void cperm_reg(V (&x)[1 << R]) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (!((j >> P) & 1) && (((j >> Q) & 1) == CV)) {
      const V t = x[j];
      x[j] = x[j | (1 << P)];
      x[j | (1 << P)] = t;
    }
}

// x = -x where target bit P = 1 and control bit Q = CV (CZ).
template <typename V, int R, int P, int Q, int CV>
__device__ __forceinline__ void neg_reg(V (&x)[1 << R]) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (((j >> P) & 1) && (((j >> Q) & 1) == CV)) x[j] = vneg(x[j]);
}

template <typename V, bool NEG, int R, int P = 0, int Q = 0, int CV = 0>
__device__ __forceinline__ void ctl_dispatch(V (&x)[1 << R], int p, int q, int cv) {
  if constexpr (P < R) {
    if constexpr (Q < R) {
      if constexpr (CV < 2) {
        if constexpr (P != Q) {
          if (p == P && q == Q && cv == CV) {
            if constexpr (NEG) neg_reg<V, R, P, Q, CV>(x);
            else cperm_reg<V, R, P, Q, CV>(x);
            return;
          }
        }
        ctl_dispatch<V, NEG, R, P, Q, CV + 1>(x, p, q, cv);
      } else {
        ctl_dispatch<V, NEG, R, P, Q + 1, 0>(x, p, q, cv);
      }
    } else {
      ctl_dispatch<V, NEG, R, P + 1, 0, 0>(x, p, q, cv);
    }
  }
}

// Quads (j, j|1<<P0, j|1<<P1, j|both), P0 > P1, in apply4's slot order.
// Coefficient read at its point of use (not hoisted out of the quad loop, so
// the 16 coefficients of a dense 4x4 op never occupy registers together).
__device__ __forceinline__ double2 ld_use(const double2* p) {
  double2 r;
  asm volatile("ld.v2.f64 {%0, %1}, [%2];" : "=d"(r.x), "=d"(r.y) : "l"(p));
  return r;
}
__device__ __forceinline__ float2 ld_use(const float2* p) {
  float2 r;
  asm volatile("ld.v2.f32 {%0, %1}, [%2];" : "=f"(r.x), "=f"(r.y) : "l"(p));
  return r;
}
__device__ __forceinline__ double ld_use(const double* p) {
  double r;
  asm volatile("ld.f64 %0, [%1];" : "=d"(r) : "l"(p));
  return r;
}
__device__ __forceinline__ float ld_use(const float* p) {
  float r;
  asm volatile("ld.f32 %0, [%1];" : "=f"(r) : "l"(p));
  return r;
}

template <typename V, int R, int P0, int P1>
__device__ __forceinline__ void quad_reg(V (&x)[1 << R], int form, int mul, const V* __restrict__ c) {
  constexpr int m0 = 1 << P0, m1 = 1 << P1;
  if (form == F_PERM) {
    const V lam = c[0];
#pragma unroll
    for (int j = 0; j < (1 << R); ++j)
      if (!(j & m0) && !(j & m1)) {
        const V xb = x[j | m0], xc = x[j | m1];
        x[j | m0] = mul ? scale1(lam, xc) : xc;
        x[j | m1] = mul ? scale1(lam, xb) : xb;
      }
    return;
  }
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (!(j & m0) && !(j & m1)) {
      const V x0 = x[j], x1 = x[j | m0], x2 = x[j | m1], x3 = x[j | m0 | m1];
      V y[4];
#pragma unroll
      for (int r = 0; r < 4; ++r)
        y[r] = mac(mac(mac(scale1(ld_use(c + 4 * r), x0), ld_use(c + 4 * r + 1), x1),
                       ld_use(c + 4 * r + 2), x2),
                   ld_use(c + 4 * r + 3), x3);
      x[j] = y[0]; x[j | m0] = y[1]; x[j | m1] = y[2]; x[j | m0 | m1] = y[3];
    }
}

template <typename V, int R, int P0 = 1, int P1 = 0>
__device__ __forceinline__ void quad_dispatch(V (&x)[1 << R], int p0, int p1, int form, int mul,
                                              const V* c) {
  if constexpr (P0 < R) {
    if constexpr (P1 < P0) {
      if (p0 == P0 && p1 == P1) quad_reg<V, R, P0, P1>(x, form, mul, c);
      else quad_dispatch<V, R, P0, P1 + 1>(x, p0, p1, form, mul, c);
    } else {
      quad_dispatch<V, R, P0 + 1, 0>(x, p0, p1, form, mul, c);
    }
  }
}

// SWAP/iSWAP only (the lean kernel: no dense 4x4 coefficients in registers).
template <typename V, int R, int P0 = 1, int P1 = 0>
__device__ __forceinline__ void quad_dispatch_perm(V (&x)[1 << R], int p0, int p1, int mul,
                                                   const V* c) {
  if constexpr (P0 < R) {
    if constexpr (P1 < P0) {
      if (p0 == P0 && p1 == P1) quad_reg<V, R, P0, P1>(x, F_PERM, mul, c);
      else quad_dispatch_perm<V, R, P0, P1 + 1>(x, p0, p1, mul, c);
    } else {
      quad_dispatch_perm<V, R, P0 + 1, 0>(x, p0, p1, mul, c);
    }
  }
}

// FULL = false compiles out the dense 4x4 path (the host only sends stages
// without dense quads and gradient reductions to that kernel).
// x <- U x for the pass's dense matrix U, stored column by column
// (c[k * 2^R + i] = U[i][k]): 2^R independent accumulators, one column of
// coefficients live at a time.
template <typename V, int R>
__device__ __forceinline__ void dense_reg(V (&x)[1 << R], const V* __restrict__ c) {
  constexpr int N = 1 << R;
  V y[N];
#pragma unroll
  for (int i = 0; i < N; ++i) y[i] = scale1(c[i], x[0]);
#pragma unroll
  for (int k = 1; k < N; ++k)
#pragma unroll
    for (int i = 0; i < N; ++i) y[i] = mac(y[i], c[k * N + i], x[k]);
#pragma unroll
  for (int i = 0; i < N; ++i) x[i] = y[i];
}

template <typename V, int R, bool FULL>
__device__ __forceinline__ void apply_reg(V (&x)[1 << R], const POp& op, const V* __restrict__ cf) {
  switch (op.shape) {
    case P_DENSE:
      if constexpr (R <= QSV_DENSE_MAX_R) dense_reg<V, R>(x, cf + op.coef);
      break;
    case P_PAIR: {
      V c[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) c[i] = cf[op.coef + i];
      pair_dispatch<V, R, false>(x, op.p0, op.form, c, 0u, 0u);
      break;
    }
    case P_CPAIR: {
      if constexpr (R >= 2) {
        if (QSV_CTL_STATIC && op.form == F_PERM) {  // CNOT: register renaming
          ctl_dispatch<V, false, R>(x, op.p0, op.p1, op.cval);
          break;
        }
      }
      V c[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) c[i] = cf[op.coef + i];
      pair_dispatch<V, R, true>(x, op.p0, op.form, c, 1u << op.p1, (uint32_t)op.cval << op.p1);
      break;
    }
    case P_MUL: {
      if constexpr (R >= 2) {
        if (QSV_CTL_STATIC && op.form == F_NEG) {  // CZ: p0 target, p1 control, cval
          ctl_dispatch<V, true, R>(x, op.p0, op.p1, op.cval);
          break;
        }
      }
      const V c = cf[op.coef];
#pragma unroll
      for (int j = 0; j < (1 << R); ++j)
        if ((j & op.mmask) == op.mval) x[j] = scale1(c, x[j]);
      break;
    }
    case P_QUAD:
      if constexpr (R >= 2) {
        if constexpr (FULL) quad_dispatch<V, R>(x, op.p0, op.p1, op.form, op.mul, cf + op.coef);
        else quad_dispatch_perm<V, R>(x, op.p0, op.p1, op.mul, cf + op.coef);
      }
      break;
    default:
      break;
  }
}

// sum_{j: (j & pm) == pv} conj(lam_j) (-1)^{pop((j^F) & zy)} psi_{j^F} over the registers
template <typename V, int R, int F>
__device__ __forceinline__ double2 red_sum(const V (&psi)[1 << R], const V (&lam)[1 << R],
                                           const POp& op) {
  double2 s = make_double2(0.0, 0.0);
#pragma unroll
  for (int j = 0; j < (1 << R); ++j) {
    if ((j & op.mmask) != op.mval) continue;
    const double sg = (__popc((j ^ F) & op.zy) & 1) ? -1.0 : 1.0;
    const double2 l = to_d2(lam[j]), y = to_d2(psi[j ^ F]);
    s.x = fma(sg * l.x, y.x, fma(sg * l.y, y.y, s.x));
    s.y = fma(sg * l.x, y.y, fma(-sg * l.y, y.x, s.y));
  }
  return s;
}

template <typename V, int R, int P0 = 0, int P1 = -1>
__device__ __forceinline__ double2 red_dispatch(const V (&psi)[1 << R], const V (&lam)[1 << R],
                                                const POp& op) {
  // nflip 0: F = 0; nflip 1: F = 1<<p0; nflip 2: F = 1<<p0 | 1<<p1 (p0 > p1)
  if (op.nflip == 0) return red_sum<V, R, 0>(psi, lam, op);
  if constexpr (P0 < R) {
    if constexpr (P1 < 0) {
      if (op.nflip == 1 && op.p0 == P0) return red_sum<V, R, (1 << P0)>(psi, lam, op);
      return red_dispatch<V, R, P0, P1 + 1>(psi, lam, op);
    } else if constexpr (P1 < P0) {
      if (op.nflip == 2 && op.p0 == P0 && op.p1 == P1)
        return red_sum<V, R, (1 << P0) | (1 << P1)>(psi, lam, op);
      return red_dispatch<V, R, P0, P1 + 1>(psi, lam, op);
    } else {
      return red_dispatch<V, R, P0 + 1, -1>(psi, lam, op);
    }
  }
  return make_double2(0.0, 0.0);
}

// ---- tile layout and copies -------------------------------------------------
template <typename V> struct Units { static constexpr int per = 16 / (int)sizeof(V); };

template <typename V>
__device__ __forceinline__ uint32_t phys(uint32_t e) {
  constexpr uint32_t EPU = Units<V>::per;
  const uint32_t u = e / EPU;
  const uint32_t su = u ^ (((u >> 3) ^ (u >> 6) ^ (u >> 9) ^ (u >> 12)) & 7u);
  return su * EPU + (e % EPU);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Global <-> shared copies of one tile (NV vectors).  All threads of the
// block take part; the caller synchronises.
template <typename V, int NV>
__device__ __forceinline__ void load_tile(const V* __restrict__ v0, const V* __restrict__ v1,
                                          V* t0, V* t1, const TileArgs& ta, uint64_t base,
                                          bool vec16) {
  constexpr uint32_t EPU = Units<V>::per;
  const uint32_t size = 1u << ta.m, lowmask = (1u << ta.low) - 1u;
  if (vec16) {
    for (uint32_t u = threadIdx.x; u < size / EPU; u += blockDim.x) {
      const uint32_t e = u * EPU;
      const uint64_t g = base | ta.runoff[e >> ta.low] | (e & lowmask);
      cp_async16(t0 + phys<V>(e), v0 + g);
      if (NV == 2) cp_async16(t1 + phys<V>(e), v1 + g);
    }
    cp_async_wait_all();
  } else {
    for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) {
      const uint64_t g = base | ta.runoff[e >> ta.low] | (e & lowmask);
      t0[phys<V>(e)] = v0[g];
      if (NV == 2) t1[phys<V>(e)] = v1[g];
    }
  }
}

template <typename V, int NV>
__device__ __forceinline__ void store_tile(V* __restrict__ v0, V* __restrict__ v1, const V* t0,
                                           const V* t1, const TileArgs& ta, uint64_t base,
                                           bool vec16) {
  constexpr uint32_t EPU = Units<V>::per;
  const uint32_t size = 1u << ta.m, lowmask = (1u << ta.low) - 1u;
  if (vec16) {
    for (uint32_t u = threadIdx.x; u < size / EPU; u += blockDim.x) {
      const uint32_t e = u * EPU;
      const uint64_t g = base | ta.runoff[e >> ta.low] | (e & lowmask);
      *reinterpret_cast<float4*>(v0 + g) = *reinterpret_cast<const float4*>(t0 + phys<V>(e));
      if (NV == 2)
        *reinterpret_cast<float4*>(v1 + g) = *reinterpret_cast<const float4*>(t1 + phys<V>(e));
    }
  } else {
    for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) {
      const uint64_t g = base | ta.runoff[e >> ta.low] | (e & lowmask);
      v0[g] = t0[phys<V>(e)];
      if (NV == 2) v1[g] = t1[phys<V>(e)];
    }
  }
}

// Two adjacent 8-byte elements (a 16-byte aligned unit) as one access; only
// instantiated for 8-byte element types.
template <typename V>
__device__ __forceinline__ void ld_pair(const V* p, V& a, V& b) {
  if constexpr (sizeof(V) == 8) {
    struct alignas(16) U { V a, b; };
    const U u = *reinterpret_cast<const U*>(p);
    a = u.a;
    b = u.b;
  } else {
    a = p[0];
    b = p[1];
  }
}
template <typename V>
__device__ __forceinline__ void st_pair(V* p, const V& a, const V& b) {
  if constexpr (sizeof(V) == 8) {
    struct alignas(16) U { V a, b; };
    *reinterpret_cast<U*>(p) = U{a, b};
  } else {
    p[0] = a;
    p[1] = b;
  }
}

// Shared-memory offset of register j of a pass: from the host-computed
// pattern offsets (QSV_PRECOMP_OFF) or recomputed from the pass bits.  The
// pass descriptor may sit in shared or global memory (plain loads only).
template <typename V, int R>
__device__ __forceinline__ uint32_t pass_off(uint32_t ptb, uint32_t tb, const uint16_t* poff,
                                             const int8_t* pos, int j) {
#if QSV_PRECOMP_OFF
  (void)tb; (void)pos;
  return ptb ^ poff[j];
#else
  (void)ptb; (void)poff;
  uint32_t e = tb;
#pragma unroll
  for (int k = 0; k < R; ++k)
    if ((j >> k) & 1) e |= 1u << pos[k];
  return phys<V>(e);
#endif
}

// Runs the register passes of one stage on a resident tile (t0, t1).  RED
// results accumulate into racc (see red_accumulate); every thread of the
// block runs the op loop, so the warp shuffles see full warps.
// A pass has ngroups = 2^(m-R) register groups.  Normally the block has one
// thread per group; with TURN a smaller block takes them in turns (every
// thread the same number), with PART a larger block leaves threads
// >= ngroups idle (they still reach every barrier).
template <typename V, int NV, int R, bool FULL, int TURN = 0, bool PART = false>
__device__ __forceinline__ void run_passes(V* t0, V* t1, const PassDev* __restrict__ passes,
                                           int npasses, const POp* __restrict__ ops,
                                           const V* __restrict__ coefs, double* racc,
                                           uint32_t ngroups) {
  const uint32_t ng = (TURN || PART) ? ngroups : blockDim.x;
  const unsigned lanes = PART ? (ngroups < 32u ? ngroups : 32u)
                              : (blockDim.x < 32u ? blockDim.x : 32u);
  for (int pi = 0; pi < npasses; ++pi) {
    const PassDev& P = passes[pi];
   for (uint32_t g = threadIdx.x; g < ng; g += blockDim.x) {
    uint32_t tb = g;
#pragma unroll
    for (int k = 0; k < R; ++k) tb = ins0(tb, P.pos[k]);
    const uint32_t ptb = phys<V>(tb);
    const uint16_t* __restrict__ poff = P.off;
    V x[1 << R], y[1 << R];
    // 8-byte elements with element bit 0 in the pass: registers 2i and 2i+1
    // are the two halves of one 16-byte unit, moved as one access
    const bool pairs = sizeof(V) == 8 && P.pos[0] == 0;
    if (pairs) {
#pragma unroll
      for (int j = 0; j < (1 << R); j += 2) {
        const uint32_t o = pass_off<V, R>(ptb, tb, poff, P.pos, j);
        ld_pair(t0 + o, x[j], x[j + 1]);
        if (NV == 2) ld_pair(t1 + o, y[j], y[j + 1]);
      }
    } else {
#pragma unroll
      for (int j = 0; j < (1 << R); ++j) {
        const uint32_t o = pass_off<V, R>(ptb, tb, poff, P.pos, j);
        x[j] = t0[o];
        if (NV == 2) y[j] = t1[o];
      }
    }
    for (int o = 0; o < P.nops; ++o) {
      const POp op = ops[P.op0 + o];
      if (op.shape == P_RED) {
        if constexpr (NV == 2 && FULL) {
          const double2 s = red_dispatch<V, R>(x, y, op);
          double im;
          switch (op.ny & 3) {  // Im(i^ny s)
            case 0: im = s.y; break;
            case 1: im = s.x; break;
            case 2: im = -s.y; break;
            default: im = -s.x; break;
          }
          red_accumulate(op.w * im, op.ridx, racc, lanes);
        }
      } else {
        apply_reg<V, R, FULL>(x, op, coefs);
        if (NV == 2) apply_reg<V, R, FULL>(y, op, coefs);
      }
    }
    if (pairs) {
#pragma unroll
      for (int j = 0; j < (1 << R); j += 2) {
        const uint32_t o = pass_off<V, R>(ptb, tb, poff, P.pos, j);
        st_pair(t0 + o, x[j], x[j + 1]);
        if (NV == 2) st_pair(t1 + o, y[j], y[j + 1]);
      }
    } else {
#pragma unroll
      for (int j = 0; j < (1 << R); ++j) {
        const uint32_t o = pass_off<V, R>(ptb, tb, poff, P.pos, j);
        t0[o] = x[j];
        if (NV == 2) t1[o] = y[j];
      }
    }
   }
    __syncthreads();
  }
}

// register bits per pass: 2^R amplitudes (x NV vectors) per thread
template <typename V> __host__ __device__ constexpr int reg_bits(int nv) {
  return sizeof(V) >= 16 ? (nv == 2 ? 3 : QSV_RBITS_C128) : (nv == 2 ? 4 : QSV_RBITS_C64);
}
// Two-vector (adjoint) sweeps keep 2 CTAs per SM: their passes hold twice the
// amplitudes and spill at the complex<double> single-vector target.
// log2 of the register groups each thread takes per pass (single-vector sweeps)
template <typename V> __host__ __device__ constexpr int turn_bits(int nv) {
  return (nv == 1 && sizeof(V) >= 16) ? QSV_TURN_BITS_C128 : 0;
}
template <typename V, int NV> __host__ __device__ constexpr int min_blocks() {
  return NV == 2 ? 2 : (sizeof(V) >= 16 ? QSV_MINBLOCKS_C128 : QSV_MINBLOCKS_C64);
}

// ---- host: packing a plan ---------------------------------------------------
int8_t classify(const Lowered& L, bool cplx);

template <typename V> V host_coef(const double* m, int i);
template <> inline double2 host_coef<double2>(const double* m, int i) { return make_double2(m[2 * i], m[2 * i + 1]); }
template <> inline float2 host_coef<float2>(const double* m, int i) { return make_float2((float)m[2 * i], (float)m[2 * i + 1]); }
template <> inline double host_coef<double>(const double* m, int i) { return m[2 * i]; }
template <> inline float host_coef<float>(const double* m, int i) { return (float)m[2 * i]; }

struct PackedStage {
  int m;
  int full;  // has dense 4x4 ops or gradient reductions (needs the full kernel)
  int bits[64];
  size_t pass0, npasses, op0, run0, coef0;
  size_t red0;  // the stage's reductions: red_slots[red0 .. red0 + nred)
  int nred;
  int nops, ncoef;  // the stage's ops and coefficients
};

template <typename V>
struct PackedPlan {
  std::vector<PassDev> passes;
  std::vector<POp> ops;
  std::vector<V> coefs;
  std::vector<uint64_t> runoff;
  std::vector<int32_t> red_slots;  // output row of each reduction, by stage
  std::vector<PackedStage> stages;
};

// Plans `gates` for an n-qubit state (tiles of 2^m, `low` contiguous bits,
// register passes of r bits) and appends the packed stages to `out`.
// dense_min: passes with at least this many ops (and no gradient terms) are
// multiplied out into one dense op; -1 = QSV_DENSE_MIN_OPS, 0 = never.
// plan_cap bounds a stage's plan bytes in shared memory.
template <typename V>
qsv_status pack_plan(const std::vector<Lowered>& gates, int n, int m, int low, int r,
                     int max_gates, PackedPlan<V>* out, int dense_min = -1,
                     size_t plan_cap = kPlanSmemMax, bool search_passes = false);

}  // namespace fx
}  // namespace qsv

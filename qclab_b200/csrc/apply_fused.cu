// Fused sweeps: each stage of a plan (plan.hpp) streams the state through
// shared memory once, one 2^m-amplitude tile per CTA, and applies all of the
// stage's gates to the tile before writing it back.
//
// Inside a tile the stage's gates are grouped into register passes
// (plan_passes): a pass owns r tile bits, every thread gathers the 2^r
// amplitudes of one assignment of the other bits into registers, applies all
// of the pass's gates there, and scatters them back -- one shared-memory
// round trip per pass instead of one per gate.  Tiles move with 16-byte
// cp.async copies into an XOR-swizzled layout (16-byte units, the unit index
// XOR-folded into its low 3 bits) so the strided gathers of a pass spread
// over the shared-memory banks.
//
// The same executor runs the adjoint's backward sweep: it then carries two
// vectors (psi and lambda) through every tile, applies each inverse gate to
// both, and evaluates the gradient terms w * Im(i^ny <lam| Pi P |psi>) of
// the parametric gates in registers (one partial sum per tile, reduced in a
// fixed order afterwards).
//
// Arithmetic here is FMA-contracted (within 1e-12 of the reference-exact
// path for complex<double>, not bitwise: the planner reorders commuting
// gates, which changes rounding).  Gates are specialised by the structure of
// their coefficients (permutation, diagonal, real, RotationX-like) because
// complex<double> sweeps with many gates per stage are bounded by the FP64
// pipe and shared memory, not by HBM.
#include <algorithm>
#include <cstring>
#include <vector>
#include "common.cuh"
#include "fused.hpp"
#include "internal.hpp"
#include "plan.hpp"
#include "tile.cuh"

namespace qsv {

static thread_local std::vector<float> g_stage_ms;

namespace {

enum Form : int8_t {
  F_GENERIC = 0,  // dense complex 2x2 / 4x4
  F_PERM = 1,     // [[0,1],[1,0]] (pairs) / swap of the |10>,|01> slots (quads)
  F_DIAG = 2,     // diagonal
  F_REAL = 3,     // all entries real
  F_RXLIKE = 4    // real diagonal, imaginary off-diagonal
};

enum POpShape : int8_t { P_PAIR = 1, P_CPAIR = 2, P_MUL = 3, P_QUAD = 4, P_RED = 5 };

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
  int16_t pad;
  int32_t slot;     // RED: partial-sum row
};

struct PassDev {
  int8_t pos[8];    // local tile bits of the pass, ascending
  int32_t op0;      // first op (stage-relative)
  int32_t nops;
};

struct Stage2Args {
  TileArgs ta;
  int npasses;
  const PassDev* passes;
  const POp* ops;
  const void* coefs;
  double* partial;  // [slot][tile] partial sums of the RED ops
  int vec16;        // 16-byte cp.async copies allowed (alignment and run length)
};

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

__device__ __forceinline__ double2 scale1(const double2 c, double2 x) { return fmul(c, x); }
__device__ __forceinline__ float2 scale1(const float2 c, float2 x) { return fmul(c, x); }
__device__ __forceinline__ double scale1(const double c, double x) { return c * x; }
__device__ __forceinline__ float scale1(const float c, float x) { return c * x; }

__device__ __forceinline__ double2 mac(double2 acc, double2 c, double2 x) { return fmac(acc, c, x); }
__device__ __forceinline__ float2 mac(float2 acc, float2 c, float2 x) { return fmac(acc, c, x); }
__device__ __forceinline__ double mac(double acc, double c, double x) { return fma(c, x, acc); }
__device__ __forceinline__ float mac(float acc, float c, float x) { return fmaf(c, x, acc); }

// ---- register-pass ops ----------------------------------------------------
// Pairs (j, j | 1<<P) of the 2^R registers whose control bits match.
template <typename V, int R, int P, int FORM>
__device__ __forceinline__ void pair_reg(V (&x)[1 << R], const V* c, uint32_t cm, uint32_t cv) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (!((j >> P) & 1) && ((j & cm) == cv)) pair2f<FORM>(c, x[j], x[j | (1 << P)]);
}

template <typename V, int R, int P>
__device__ __forceinline__ void pair_forms(V (&x)[1 << R], int form, const V* c, uint32_t cm,
                                           uint32_t cv) {
  switch (form) {
    case F_PERM: pair_reg<V, R, P, F_PERM>(x, c, cm, cv); break;
    case F_DIAG: pair_reg<V, R, P, F_DIAG>(x, c, cm, cv); break;
    case F_REAL: pair_reg<V, R, P, F_REAL>(x, c, cm, cv); break;
    case F_RXLIKE: pair_reg<V, R, P, F_RXLIKE>(x, c, cm, cv); break;
    default: pair_reg<V, R, P, F_GENERIC>(x, c, cm, cv); break;
  }
}

template <typename V, int R, int P = 0>
__device__ __forceinline__ void pair_dispatch(V (&x)[1 << R], int p, int form, const V* c,
                                              uint32_t cm, uint32_t cv) {
  if constexpr (P < R) {
    if (p == P) pair_forms<V, R, P>(x, form, c, cm, cv);
    else pair_dispatch<V, R, P + 1>(x, p, form, c, cm, cv);
  }
}

// Quads (j, j|1<<P0, j|1<<P1, j|both), P0 > P1, in apply4's slot order.
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
        y[r] = mac(mac(mac(scale1(c[4 * r], x0), c[4 * r + 1], x1), c[4 * r + 2], x2),
                   c[4 * r + 3], x3);
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

template <typename V, int R>
__device__ __forceinline__ void apply_reg(V (&x)[1 << R], const POp& op, const V* __restrict__ cf) {
  switch (op.shape) {
    case P_PAIR:
    case P_CPAIR: {
      V c[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) c[i] = cf[op.coef + i];
      const uint32_t cm = (op.shape == P_CPAIR) ? (1u << op.p1) : 0u;
      const uint32_t cv = (op.shape == P_CPAIR) ? ((uint32_t)op.cval << op.p1) : 0u;
      pair_dispatch<V, R>(x, op.p0, op.form, c, cm, cv);
      break;
    }
    case P_MUL: {
      const V c = cf[op.coef];
#pragma unroll
      for (int j = 0; j < (1 << R); ++j)
        if ((j & op.mmask) == op.mval) x[j] = scale1(c, x[j]);
      break;
    }
    case P_QUAD:
      if constexpr (R >= 2) quad_dispatch<V, R>(x, op.p0, op.p1, op.form, op.mul, cf + op.coef);
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

template <typename V, int NV, int R>
__global__ void __launch_bounds__(256, 2)
k_stage2(V* __restrict__ v0, V* __restrict__ v1, Stage2Args a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double2 red[32];
  constexpr uint32_t EPU = Units<V>::per;
  const int m = a.ta.m, low = a.ta.low;
  const uint32_t size = 1u << m, lowmask = (1u << low) - 1u;
  V* t0 = reinterpret_cast<V*>(smem_raw);
  V* t1 = t0 + size;
  const uint64_t* __restrict__ runoff = a.ta.runoff;
  const V* __restrict__ coefs = static_cast<const V*>(a.coefs);
  const uint64_t base = tile_base(a.ta, blockIdx.x);

  // ---- load the tile(s) ----
  if (a.vec16) {
    for (uint32_t u = threadIdx.x; u < size / EPU; u += blockDim.x) {
      const uint32_t e = u * EPU;
      const uint64_t g = base | runoff[e >> low] | (e & lowmask);
      cp_async16(t0 + phys<V>(e), v0 + g);
      if (NV == 2) cp_async16(t1 + phys<V>(e), v1 + g);
    }
    cp_async_wait_all();
  } else {
    for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) {
      const uint64_t g = base | runoff[e >> low] | (e & lowmask);
      t0[phys<V>(e)] = v0[g];
      if (NV == 2) t1[phys<V>(e)] = v1[g];
    }
  }
  __syncthreads();

  // ---- register passes ----
  for (int pi = 0; pi < a.npasses; ++pi) {
    const PassDev P = a.passes[pi];
    uint32_t bit[R];
    uint32_t tb = threadIdx.x;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      bit[k] = 1u << P.pos[k];
      tb = ins0(tb, P.pos[k]);
    }
    V x[1 << R], y[1 << R];
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      uint32_t e = tb;
#pragma unroll
      for (int k = 0; k < R; ++k)
        if ((j >> k) & 1) e |= bit[k];
      x[j] = t0[phys<V>(e)];
      if (NV == 2) y[j] = t1[phys<V>(e)];
    }
    for (int o = 0; o < P.nops; ++o) {
      const POp op = a.ops[P.op0 + o];
      if (op.shape == P_RED) {
        if constexpr (NV == 2) {
          const double2 s = red_dispatch<V, R>(x, y, op);
          double im;
          switch (op.ny & 3) {  // Im(i^ny s)
            case 0: im = s.y; break;
            case 1: im = s.x; break;
            case 2: im = -s.y; break;
            default: im = -s.x; break;
          }
          const double2 tot = block_sum(make_double2(op.w * im, 0.0), red);
          if (threadIdx.x == 0) a.partial[(size_t)op.slot * gridDim.x + blockIdx.x] = tot.x;
        }
      } else {
        apply_reg<V, R>(x, op, coefs);
        if (NV == 2) apply_reg<V, R>(y, op, coefs);
      }
    }
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      uint32_t e = tb;
#pragma unroll
      for (int k = 0; k < R; ++k)
        if ((j >> k) & 1) e |= bit[k];
      t0[phys<V>(e)] = x[j];
      if (NV == 2) t1[phys<V>(e)] = y[j];
    }
    __syncthreads();
  }

  // ---- store the tile(s) ----
  if (a.vec16) {
    for (uint32_t u = threadIdx.x; u < size / EPU; u += blockDim.x) {
      const uint32_t e = u * EPU;
      const uint64_t g = base | runoff[e >> low] | (e & lowmask);
      *reinterpret_cast<float4*>(v0 + g) = *reinterpret_cast<const float4*>(t0 + phys<V>(e));
      if (NV == 2)
        *reinterpret_cast<float4*>(v1 + g) = *reinterpret_cast<const float4*>(t1 + phys<V>(e));
    }
  } else {
    for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) {
      const uint64_t g = base | runoff[e >> low] | (e & lowmask);
      v0[g] = t0[phys<V>(e)];
      if (NV == 2) v1[g] = t1[phys<V>(e)];
    }
  }
}

// Fixed-order sum of each row of partial[rows][cols] (one block per row).
__global__ void __launch_bounds__(256)
k_rows(const double* __restrict__ partial, int cols, double* __restrict__ out) {
  __shared__ double2 red[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < cols; i += blockDim.x) acc += partial[(size_t)blockIdx.x * cols + i];
  const double2 s = block_sum(make_double2(acc, 0.0), red);
  if (threadIdx.x == 0) out[blockIdx.x] = s.x;
}

int8_t classify(const Lowered& L, bool cplx) {
  if (L.shape != SH_PAIR && L.shape != SH_CPAIR) return F_GENERIC;
  const double* m = L.m;  // a00 a01 a10 a11 as (re,im)
  auto z = [&](int i) { return m[2 * i] == 0.0 && m[2 * i + 1] == 0.0; };
  auto isone = [&](int i) { return m[2 * i] == 1.0 && m[2 * i + 1] == 0.0; };
  if (z(0) && z(3) && isone(1) && isone(2)) return F_PERM;
  if (z(1) && z(2)) return F_DIAG;
  if (!cplx || L.real) return F_REAL;
  if (m[1] == 0.0 && m[7] == 0.0 && m[2] == 0.0 && m[4] == 0.0) return F_RXLIKE;
  return F_GENERIC;
}

template <typename V> V host_coef(const double* m, int i);
template <> double2 host_coef<double2>(const double* m, int i) { return make_double2(m[2 * i], m[2 * i + 1]); }
template <> float2 host_coef<float2>(const double* m, int i) { return make_float2((float)m[2 * i], (float)m[2 * i + 1]); }
template <> double host_coef<double>(const double* m, int i) { return m[2 * i]; }
template <> float host_coef<float>(const double* m, int i) { return (float)m[2 * i]; }

// register bits per pass: 2^R amplitudes (x NV vectors) per thread
template <typename V> constexpr int reg_bits(int nv) {
  return sizeof(V) >= 16 ? (nv == 2 ? 3 : 4) : (nv == 2 ? 4 : 5);
}

template <typename V, int NV, int R>
void* stage_kernel() { return (void*)k_stage2<V, NV, R>; }

template <typename V, int NV>
void* pick_kernel(int r) {
  constexpr int RD = reg_bits<V>(NV);
  if (r == RD) return stage_kernel<V, NV, RD>();
  if (r == 2) return stage_kernel<V, NV, 2>();
  return stage_kernel<V, NV, 1>();
}

template <typename V>
qsv_status execute_typed(const ExecArgs& x) {
  constexpr bool cplx = Elem<V>::cplx;
  constexpr int EPU = Units<V>::per;
  qsv_state_s* s = x.s;
  const int n = s->n;
  const qsv_fuse_opts* opts = x.opts;
  int m = (opts && opts->tile_bits > 0) ? opts->tile_bits : default_tile_bits(sizeof(V), x.nv);
  int low = (opts && opts->low_bits > 0) ? opts->low_bits : default_low_bits(sizeof(V));
  const int max_gates = (opts && opts->max_stage_gates > 0) ? opts->max_stage_gates : 256;
  if (m > 14) m = 14;
  if (m > n) m = n;
  const int rdef = (x.nv == 2) ? reg_bits<V>(2) : reg_bits<V>(1);
  const int r = (m >= rdef) ? rdef : (m >= 2 ? 2 : 1);
  if (m - r > 8) m = r + 8;  // at most 256 threads per CTA
  if (low > m) low = m;
  const size_t smem = (size_t(1) << m) * sizeof(V) * x.nv;
  if (smem > 200 * 1024)
    return fail(QSV_ERROR_SIZE, "tile of %d x 2^%d elements exceeds shared memory", x.nv, m);
  // 16-byte copies need 16-byte aligned vectors and runs of >= 16 bytes
  int log_epu = 0;
  while ((1 << log_epu) < EPU) ++log_epu;
  const bool vec16 = (low >= log_epu) && (m >= log_epu) &&
                     (reinterpret_cast<uintptr_t>(x.v0) % 16 == 0) &&
                     (x.nv == 1 || reinterpret_cast<uintptr_t>(x.v1) % 16 == 0);

  const std::vector<Lowered>& gates = *x.items;
  std::vector<Stage> stages = plan_stages(gates, n, m, low, max_gates);
  if (stages.empty()) return QSV_SUCCESS;

  // pack passes, ops, coefficients and run offsets of every stage
  std::vector<PassDev> passes;
  std::vector<POp> ops;
  std::vector<V> coefs;
  std::vector<uint64_t> runoff;
  struct Meta { size_t pass0, npasses, op0, run0, coef0; };
  std::vector<Meta> meta;
  for (const Stage& stg : stages) {
    Meta mt{passes.size(), 0, ops.size(), runoff.size(), coefs.size()};
    int local_of[64];
    for (int j = 0; j < 64; ++j) local_of[j] = -1;
    for (int j = 0; j < stg.m; ++j) local_of[stg.bits[j]] = j;
    auto local_mask = [&](uint64_t g) {
      uint32_t r2 = 0;
      for (int b = 0; b < n; ++b)
        if ((g >> b) & 1ull) r2 |= 1u << local_of[b];
      return r2;
    };
    std::vector<uint32_t> op_bits;
    for (int gi : stg.gates) op_bits.push_back(local_mask(gate_bits(gates[gi])));
    std::vector<Pass> pl = plan_passes(op_bits, stg.m, r);
    for (const Pass& p : pl) {
      PassDev pd{};
      for (int k = 0; k < 8; ++k) pd.pos[k] = (k < p.r) ? (int8_t)p.pos[k] : 0;
      pd.op0 = (int32_t)(ops.size() - mt.op0);
      pd.nops = (int32_t)p.ops.size();
      int reg_of[32];
      for (int j = 0; j < 32; ++j) reg_of[j] = -1;
      for (int k = 0; k < p.r; ++k) reg_of[p.pos[k]] = k;
      auto reg_mask = [&](uint64_t g) {
        const uint32_t lm = local_mask(g);
        uint32_t rm = 0;
        for (int j = 0; j < stg.m; ++j)
          if ((lm >> j) & 1u) rm |= 1u << reg_of[j];
        return (uint8_t)rm;
      };
      auto reg_pos = [&](int gbit) { return (int8_t)reg_of[local_of[gbit]]; };
      for (int oi : p.ops) {
        const Lowered& L = gates[stg.gates[oi]];
        POp op{};
        if (coefs.size() - mt.coef0 > 30000) return fail(QSV_ERROR_SIZE, "fused stage too large");
        op.coef = (int16_t)(coefs.size() - mt.coef0);
        int nc = 0;
        switch (L.shape) {
          case SH_PAIR:
            op.shape = P_PAIR; op.p0 = reg_pos(L.t0); op.form = classify(L, cplx); nc = 4;
            break;
          case SH_CPAIR:
            op.shape = P_CPAIR; op.p0 = reg_pos(L.t0); op.p1 = reg_pos(L.t1);
            op.cval = (int8_t)L.cval; op.form = classify(L, cplx); nc = 4;
            break;
          case SH_HALF:
            op.shape = P_MUL; op.mmask = op.mval = (uint8_t)(1u << reg_pos(L.t0)); nc = 1;
            break;
          case SH_CHALF:
            op.shape = P_MUL;
            op.mmask = (uint8_t)((1u << reg_pos(L.t0)) | (1u << reg_pos(L.t1)));
            op.mval = (uint8_t)((1u << reg_pos(L.t0)) | ((uint32_t)L.cval << reg_pos(L.t1)));
            nc = 1;
            break;
          case SH_QUAD:
            op.shape = P_QUAD; op.p0 = reg_pos(L.t0); op.p1 = reg_pos(L.t1); op.form = F_GENERIC;
            nc = 16;
            break;
          case SH_SWAP:
            op.shape = P_QUAD; op.p0 = reg_pos(L.t0); op.p1 = reg_pos(L.t1); op.form = F_PERM;
            op.mul = (int8_t)L.mul; nc = 1;
            break;
          case SH_RED: {
            op.shape = P_RED;
            const uint8_t fm = reg_mask(L.gen.f);
            op.nflip = (int8_t)__builtin_popcount(fm);
            int hi = -1, lo = -1;
            for (int k = 0; k < 8; ++k)
              if ((fm >> k) & 1u) { lo = (lo < 0) ? k : lo; hi = k; }
            op.p0 = (int8_t)hi;
            op.p1 = (int8_t)(op.nflip == 2 ? lo : -1);
            op.zy = reg_mask(L.gen.zy);
            op.mmask = reg_mask(L.gen.pm);
            op.mval = reg_mask(L.gen.pv);
            op.ny = (int8_t)L.gen.ny;
            op.w = (int8_t)L.gen.w;
            op.slot = L.slot;
            break;
          }
          default:
            return fail(QSV_ERROR_INVALID_VALUE, "internal: shape %d in a fused stage", L.shape);
        }
        for (int i = 0; i < nc; ++i) coefs.push_back(host_coef<V>(L.m, i));
        ops.push_back(op);
      }
      passes.push_back(pd);
    }
    mt.npasses = passes.size() - mt.pass0;
    tile_runoffs(stg.bits, stg.m, low, &runoff);
    meta.push_back(mt);
  }
  auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
  const size_t pass_bytes = passes.size() * sizeof(PassDev);
  const size_t op_off = align(pass_bytes);
  const size_t coef_off = align(op_off + ops.size() * sizeof(POp));
  const size_t run_off = align(coef_off + coefs.size() * sizeof(V));
  const size_t total = run_off + runoff.size() * sizeof(uint64_t);
  std::vector<unsigned char> host(total);
  std::memcpy(host.data(), passes.data(), pass_bytes);
  std::memcpy(host.data() + op_off, ops.data(), ops.size() * sizeof(POp));
  std::memcpy(host.data() + coef_off, coefs.data(), coefs.size() * sizeof(V));
  std::memcpy(host.data() + run_off, runoff.data(), runoff.size() * sizeof(uint64_t));
  if (qsv_status st = ensure_scratch(s, total)) return st;
  unsigned char* dev = static_cast<unsigned char*>(s->scratch);
  if (qsv_status st = cuda_status(cudaMemcpyAsync(dev, host.data(), total, cudaMemcpyHostToDevice,
                                                  s->stream), "fused plan upload"))
    return st;

  void* kern = (x.nv == 2) ? pick_kernel<V, 2>(r) : pick_kernel<V, 1>(r);
  if (qsv_status st = cuda_status(
          cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024),
          "fused stage shared-memory attribute"))
    return st;
  const unsigned threads = 1u << (m - r);
  const uint64_t ntiles = 1ull << (n - m);
  if (x.ntiles_out) *x.ntiles_out = ntiles;
  if (x.nslots > 0 && x.partial_bytes < (size_t)x.nslots * ntiles * sizeof(double))
    return fail(QSV_ERROR_SIZE, "partial-sum buffer too small");
  const bool profile = opts && opts->profile;
  std::vector<cudaEvent_t> ev;
  if (profile) {
    ev.resize(stages.size() + 1);
    for (auto& e : ev)
      if (qsv_status st = cuda_status(cudaEventCreate(&e), "cudaEventCreate")) return st;
    cudaEventRecord(ev[0], s->stream);
  }
  V* p0 = static_cast<V*>(x.v0);
  V* p1 = static_cast<V*>(x.v1);
  for (size_t si = 0; si < stages.size(); ++si) {
    Stage2Args a;
    a.ta.n = n;
    a.ta.m = stages[si].m;
    a.ta.low = low;
    for (int j = 0; j < 64; ++j) a.ta.bits[j] = (j < stages[si].m) ? (int8_t)stages[si].bits[j] : 0;
    a.ta.runoff = reinterpret_cast<const uint64_t*>(dev + run_off) + meta[si].run0;
    a.npasses = (int)meta[si].npasses;
    a.passes = reinterpret_cast<const PassDev*>(dev) + meta[si].pass0;
    a.ops = reinterpret_cast<const POp*>(dev + op_off) + meta[si].op0;
    a.coefs = dev + coef_off + meta[si].coef0 * sizeof(V);
    a.partial = x.partial;
    a.vec16 = vec16 ? 1 : 0;
    void* args[] = {&p0, &p1, &a};
    if (qsv_status st = cuda_status(cudaLaunchKernel(kern, dim3((unsigned)ntiles), dim3(threads),
                                                     args, smem, s->stream),
                                    "fused stage launch"))
      return st;
    count_launch();
    if (profile) cudaEventRecord(ev[si + 1], s->stream);
  }
  if (profile) {
    qsv_status st = cuda_status(cudaEventSynchronize(ev.back()), "stage timing synchronize");
    g_stage_ms.clear();
    for (size_t si = 0; si < stages.size() && !st; ++si) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[si], ev[si + 1]);
      g_stage_ms.push_back(ms);
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (st) return st;
  }
  if (x.nslots > 0) {
    k_rows<<<x.nslots, 256, 0, s->stream>>>(x.partial, (int)ntiles, x.rows_out);
    count_launch();
    if (qsv_status st = cuda_status(cudaGetLastError(), "row reduction launch")) return st;
  }
  return QSV_SUCCESS;
}

}  // namespace

int default_tile_bits(size_t eb, int nv) { return (eb >= 16 ? 12 : 13) - (nv == 2 ? 1 : 0); }
int default_low_bits(size_t eb) { return eb >= 16 ? 2 : 3; }

qsv_status execute_fused(const ExecArgs& x) {
  switch (x.s->dtype) {
    case QSV_C128: return execute_typed<double2>(x);
    case QSV_C64:  return execute_typed<float2>(x);
    case QSV_F64:  return execute_typed<double>(x);
    case QSV_F32:  return execute_typed<float>(x);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

qsv_status run_fused(qsv_state_s* s, const std::vector<Lowered>& gates, const qsv_fuse_opts* opts) {
  ExecArgs x;
  x.s = s;
  x.items = &gates;
  x.v0 = s->d;
  x.opts = opts;
  return execute_fused(x);
}

}  // namespace qsv

extern "C" qsv_status qsv_last_stage_times(float* ms, int capacity, int* count) {
  using namespace qsv;
  if (!count) return fail(QSV_ERROR_INVALID_VALUE, "null count");
  *count = (int)g_stage_ms.size();
  if (ms)
    for (int i = 0; i < capacity && i < (int)g_stage_ms.size(); ++i) ms[i] = g_stage_ms[i];
  return QSV_SUCCESS;
}

extern "C" qsv_status qsv_plan_stats(int nbQubits, qsv_dtype dtype, const qsv_gate* gates,
                                     size_t nGates, char op, int offset,
                                     const qsv_fuse_opts* opts, int* nStages, int* stage_gates,
                                     int capacity) {
  using namespace qsv;
  if (!nStages) return fail(QSV_ERROR_INVALID_VALUE, "null nStages");
  if (!dtype_valid(dtype)) return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
  if (nbQubits < 1 || nbQubits > kMaxQubits) return fail(QSV_ERROR_SIZE, "bad nbQubits");
  qsv_state_s fake;
  fake.n = nbQubits;
  fake.dtype = dtype;
  std::vector<Lowered> low;
  if (qsv_status st = lower_for_state(&fake, gates, nGates, op, offset, &low)) return st;
  const size_t eb = elem_bytes(dtype);
  int m = (opts && opts->tile_bits > 0) ? opts->tile_bits : default_tile_bits(eb, 1);
  int lowb = (opts && opts->low_bits > 0) ? opts->low_bits : default_low_bits(eb);
  const int max_gates = (opts && opts->max_stage_gates > 0) ? opts->max_stage_gates : 256;
  std::vector<Stage> stages = plan_stages(low, nbQubits, std::min(m, 14), lowb, max_gates);
  *nStages = (int)stages.size();
  if (stage_gates)
    for (int i = 0; i < capacity && i < (int)stages.size(); ++i)
      stage_gates[i] = (int)stages[i].gates.size();
  return QSV_SUCCESS;
}

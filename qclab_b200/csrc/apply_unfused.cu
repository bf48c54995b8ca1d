// Reference-exact, one-kernel-per-gate amplitude kernels.
//
// These are the sm_100a replacements of QCLAB++'s index loops apply2,
// apply2b, apply4 (dense and controlled), apply4b and apply4bc
// (src/qgates/apply.hpp:259-371) and of their OpenMP-offload twins
// (apply.hpp:375-531).  They keep each reference lambda's arithmetic
// (same products, same summation order, no FMA) so results are bitwise
// equal to the CPU reference.
//
// Work decomposition ("warp tiles"): the 32 lanes of a warp always cover
// index bits 0..4, so every load and store of a warp is one contiguous run
// of 32 amplitudes (512 B for complex<double>).  Target bits >= 5 are held
// in registers (each lane owns the 2 or 4 amplitudes of its pair/quad);
// target bits < 5 live across lanes and partners are exchanged with warp
// shuffles.  Bits fixed by the gate (the control state, the |1> half of a
// diagonal gate) are either folded into the tile base (bits >= 5, so the
// untouched half is never read) or mask lanes (bits < 5).  Remaining bits
// enumerate warp tiles.
#include <cstdio>
#include "common.cuh"
#include "internal.hpp"

namespace qsv {
namespace {

constexpr int kLaneBits = 5;
constexpr int kThreads = 256;

struct Geo {
  uint64_t ntiles;    // number of 32-lane tiles
  int nspec;          // zero bits inserted into the tile index (ascending)
  int spec[2];
  uint64_t fixed_or;  // fixed bits >= 5 that are one
  uint32_t lane_mask; // lane active iff (lane & lane_mask) == lane_val
  uint32_t lane_val;
  uint32_t lane_lim;  // lanes >= lane_lim do not exist (n < 5)
};

template <typename V> struct M2 { V a00, a01, a10, a11; };
template <typename V> struct M4 { V a[16]; };

// Row r (0: a, 1: b) of a 2x2 gate on the pair (x1, x2), evaluated with the
// operations of its reference lambda (lower.hpp ExactForm, apply.hpp:9-128):
// signed zeros come out as the reference's do.  `form` is uniform per launch.
template <typename V>
__device__ __forceinline__ V pair_row(int form, const M2<V>& M, V x1, V x2, int r) {
  switch (form) {
    case EF_HADAMARD: {
      const auto s = ere(M.a00);
      return r ? esub(smul(s, x1), smul(s, x2)) : eadd(smul(s, x1), smul(s, x2));
    }
    case EF_ROTX: {
      const auto c = ere(M.a00);
      return r ? eadd(emul(M.a10, x1), smul(c, x2)) : eadd(smul(c, x1), emul(M.a01, x2));
    }
    case EF_ROTY:
      return r ? eadd(smul(ere(M.a10), x1), smul(ere(M.a11), x2))
               : eadd(smul(ere(M.a00), x1), smul(ere(M.a01), x2));
    case EF_DIAG:
      return r ? emul(M.a11, x2) : emul(M.a00, x1);
    case EF_SWAP:
      return r ? x1 : x2;
    case EF_SWAP_MUL:
      return r ? emul(M.a10, x1) : emul(M.a01, x2);
    default:
      return r ? eadd(emul(M.a10, x1), emul(M.a11, x2)) : eadd(emul(M.a00, x1), emul(M.a01, x2));
  }
}

__device__ __forceinline__ uint64_t tile_base(const Geo& g, uint64_t w, int n) {
  uint64_t x = (n >= kLaneBits) ? (w << kLaneBits) : 0ull;
  if (g.nspec > 0) x = insert_zero(x, g.spec[0]);
  if (g.nspec > 1) x = insert_zero(x, g.spec[1]);
  return x | g.fixed_or;
}

__device__ __forceinline__ uint64_t warp_id() {
  return ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> kLaneBits;
}

__device__ __forceinline__ bool lane_active(const Geo& g, int lane) {
  return ((lane & g.lane_mask) == g.lane_val) && ((uint32_t)lane < g.lane_lim);
}

// ---- 2x2 on a pair whose target bit is held in registers (bit >= 5) ------
// apply2 (apply.hpp:259-272) / apply4 controlled (apply.hpp:311-332).
template <typename V, int ITEMS>
__global__ void __launch_bounds__(kThreads)
k_pair_reg(V* __restrict__ st, Geo g, int n, uint64_t tmask, M2<V> M, int form) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = warp_id() * ITEMS;
  const bool lok = lane_active(g, lane);
  V x1[ITEMS], x2[ITEMS];
  uint64_t idx[ITEMS];
  bool ok[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    ok[i] = lok && (w0 + i < g.ntiles);
    idx[i] = tile_base(g, w0 + i, n) | (uint64_t)lane;
    if (ok[i]) { x1[i] = st[idx[i]]; x2[i] = st[idx[i] | tmask]; }
  }
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    if (!ok[i]) continue;
    st[idx[i]]         = pair_row(form, M, x1[i], x2[i], 0);
    st[idx[i] | tmask] = pair_row(form, M, x1[i], x2[i], 1);
  }
}

// ---- 2x2 on a pair whose target bit is a lane bit (bit < 5) --------------
template <typename V, int ITEMS>
__global__ void __launch_bounds__(kThreads)
k_pair_lane(V* __restrict__ st, Geo g, int n, int tbit, M2<V> M, int form) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = warp_id() * ITEMS;
  const bool lok = lane_active(g, lane);
  const bool upper = (lane >> tbit) & 1;
  V v[ITEMS];
  uint64_t idx[ITEMS];
  bool ok[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    ok[i] = lok && (w0 + i < g.ntiles);
    idx[i] = tile_base(g, w0 + i, n) | (uint64_t)lane;
    v[i] = ok[i] ? st[idx[i]] : vzero<V>();
  }
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const V p = shfl_xor(v[i], 1 << tbit);
    // lower lane: a = m11*x1 + m12*x2 with x1 = own, x2 = partner;
    // upper lane: b = m21*x1 + m22*x2 with x1 = partner, x2 = own.
    const V out = upper ? pair_row(form, M, p, v[i], 1) : pair_row(form, M, v[i], p, 0);
    if (ok[i]) st[idx[i]] = out;
  }
}

// ---- x *= lambda on the amplitudes selected by the fixed bits ------------
// apply2b (apply.hpp:275-287), apply4b (apply.hpp:335-352).
template <typename V, int ITEMS>
__global__ void __launch_bounds__(kThreads)
k_scale(V* __restrict__ st, Geo g, int n, V lam, int form) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = warp_id() * ITEMS;
  const bool lok = lane_active(g, lane);
  V v[ITEMS];
  uint64_t idx[ITEMS];
  bool ok[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    ok[i] = lok && (w0 + i < g.ntiles);
    idx[i] = tile_base(g, w0 + i, n) | (uint64_t)lane;
    if (ok[i]) v[i] = st[idx[i]];
  }
#pragma unroll
  for (int i = 0; i < ITEMS; ++i)
    if (ok[i]) st[idx[i]] = (form == EF_NEG) ? eneg(v[i]) : emul(lam, v[i]);
}

template <typename V>
__device__ __forceinline__ V row4(const V* a, int r, V x0, V x1, V x2, V x3) {
  // ((m_r1*x1 + m_r2*x2) + m_r3*x3) + m_r4*x4  (lambda_QGate2, apply.hpp:186-196)
  return eadd(eadd(eadd(emul(a[4 * r], x0), emul(a[4 * r + 1], x1)),
                   emul(a[4 * r + 2], x2)),
              emul(a[4 * r + 3], x3));
}

template <typename V>
__device__ __forceinline__ V row4c(V c0, V c1, V c2, V c3, V x0, V x1, V x2, V x3) {
  return eadd(eadd(eadd(emul(c0, x0), emul(c1, x1)), emul(c2, x2)), emul(c3, x3));
}

// ---- dense 4x4, both target bits in registers ----------------------------
// apply4 (apply.hpp:290-308): slots a, a|b1, a|c1, a|b1|c1.
template <typename V, int ITEMS>
__global__ void __launch_bounds__(kThreads)
k_quad_reg2(V* __restrict__ st, Geo g, int n, uint64_t m0, uint64_t m1, M4<V> M) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = warp_id() * ITEMS;
  const bool lok = lane_active(g, lane);
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    if (!(lok && (w0 + i < g.ntiles))) continue;
    const uint64_t a = tile_base(g, w0 + i, n) | (uint64_t)lane;
    const V x0 = st[a], x1 = st[a | m0], x2 = st[a | m1], x3 = st[a | m0 | m1];
    st[a]           = row4(M.a, 0, x0, x1, x2, x3);
    st[a | m0]      = row4(M.a, 1, x0, x1, x2, x3);
    st[a | m1]      = row4(M.a, 2, x0, x1, x2, x3);
    st[a | m0 | m1] = row4(M.a, 3, x0, x1, x2, x3);
  }
}

// ---- dense 4x4, high bit in registers, low bit across lanes --------------
template <typename V, int ITEMS>
__global__ void __launch_bounds__(kThreads)
k_quad_reg1(V* __restrict__ st, Geo g, int n, uint64_t m0, int t1, M4<V> M) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = warp_id() * ITEMS;
  const bool lok = lane_active(g, lane);
  const int lb = (lane >> t1) & 1;
  // rows of this lane's two slots: (bq0=0, bq1=lb) -> row 2*lb and
  // (bq0=1, bq1=lb) -> row 1+2*lb
  V c0[4], c1[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    c0[j] = lb ? M.a[4 * 2 + j] : M.a[4 * 0 + j];
    c1[j] = lb ? M.a[4 * 3 + j] : M.a[4 * 1 + j];
  }
  V v0[ITEMS], v1[ITEMS];
  uint64_t idx[ITEMS];
  bool ok[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    ok[i] = lok && (w0 + i < g.ntiles);
    idx[i] = tile_base(g, w0 + i, n) | (uint64_t)lane;
    v0[i] = ok[i] ? st[idx[i]] : vzero<V>();
    v1[i] = ok[i] ? st[idx[i] | m0] : vzero<V>();
  }
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const V p0 = shfl_xor(v0[i], 1 << t1), p1 = shfl_xor(v1[i], 1 << t1);
    const V x0 = lb ? p0 : v0[i];
    const V x1 = lb ? p1 : v1[i];
    const V x2 = lb ? v0[i] : p0;
    const V x3 = lb ? v1[i] : p1;
    if (ok[i]) {
      st[idx[i]]      = row4c(c0[0], c0[1], c0[2], c0[3], x0, x1, x2, x3);
      st[idx[i] | m0] = row4c(c1[0], c1[1], c1[2], c1[3], x0, x1, x2, x3);
    }
  }
}

// ---- dense 4x4, both target bits across lanes -----------------------------
template <typename V, int ITEMS>
__global__ void __launch_bounds__(kThreads)
k_quad_lane(V* __restrict__ st, Geo g, int n, int t0, int t1, M4<V> M) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = warp_id() * ITEMS;
  const bool lok = lane_active(g, lane);
  const int l0 = 1 << t0, l1 = 1 << t1;
  const int s = ((lane >> t0) & 1) | (((lane >> t1) & 1) << 1);
  const int base_lane = lane & ~(l0 | l1);
  V c[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const V r0 = M.a[j], r1 = M.a[4 + j], r2 = M.a[8 + j], r3 = M.a[12 + j];
    c[j] = (s == 0) ? r0 : (s == 1) ? r1 : (s == 2) ? r2 : r3;
  }
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const bool ok = lok && (w0 + i < g.ntiles);
    const uint64_t idx = tile_base(g, w0 + i, n) | (uint64_t)lane;
    const V v = ok ? st[idx] : vzero<V>();
    const V x0 = shfl_idx(v, base_lane);
    const V x1 = shfl_idx(v, base_lane | l0);
    const V x2 = shfl_idx(v, base_lane | l1);
    const V x3 = shfl_idx(v, base_lane | l0 | l1);
    if (ok) st[idx] = row4c(c[0], c[1], c[2], c[3], x0, x1, x2, x3);
  }
}

// ---- swap of the |10>,|01> slots of each quad (apply4bc, apply.hpp:355-371)
template <typename V, bool MUL, int ITEMS>
__global__ void __launch_bounds__(kThreads)
k_swap_reg2(V* __restrict__ st, Geo g, int n, uint64_t m0, uint64_t m1, V lam) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = warp_id() * ITEMS;
  const bool lok = lane_active(g, lane);
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    if (!(lok && (w0 + i < g.ntiles))) continue;
    const uint64_t a = tile_base(g, w0 + i, n) | (uint64_t)lane;
    const V xb = st[a | m0], xc = st[a | m1];
    st[a | m0] = MUL ? emul(lam, xc) : xc;
    st[a | m1] = MUL ? emul(lam, xb) : xb;
  }
}

template <typename V, bool MUL, int ITEMS>
__global__ void __launch_bounds__(kThreads)
k_swap_reg1(V* __restrict__ st, Geo g, int n, uint64_t m0, int t1, V lam) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = warp_id() * ITEMS;
  const bool lok = lane_active(g, lane);
  const int lb = (lane >> t1) & 1;
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const bool ok = lok && (w0 + i < g.ntiles);
    // lane with t1 clear owns slot |10> (t0 set); lane with t1 set owns |01>.
    const uint64_t idx = (tile_base(g, w0 + i, n) | (uint64_t)lane) | (lb ? 0ull : m0);
    const V v = ok ? st[idx] : vzero<V>();
    const V p = shfl_xor(v, 1 << t1);
    if (ok) st[idx] = MUL ? emul(lam, p) : p;
  }
}

template <typename V, bool MUL, int ITEMS>
__global__ void __launch_bounds__(kThreads)
k_swap_lane(V* __restrict__ st, Geo g, int n, int t0, int t1, V lam) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = warp_id() * ITEMS;
  const bool lok = lane_active(g, lane) && ((((lane >> t0) ^ (lane >> t1)) & 1) != 0);
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const bool ok = lok && (w0 + i < g.ntiles);
    const uint64_t idx = tile_base(g, w0 + i, n) | (uint64_t)lane;
    const V v = ok ? st[idx] : vzero<V>();
    const V p = shfl_xor(v, (1 << t0) | (1 << t1));
    if (ok) st[idx] = MUL ? emul(lam, p) : p;
  }
}

// ---- host side -------------------------------------------------------------

struct GeoBuilder {
  int n;
  int nspec = 0;
  int spec[2] = {0, 0};
  uint64_t fixed_or = 0;
  uint32_t lane_mask = 0, lane_val = 0;

  explicit GeoBuilder(int n_) : n(n_) {}
  void reg(int b) {  // target bit held in registers (caller ensures b >= 5)
    spec[nspec++] = b;
  }
  void fix(int b, int v) {
    if (b >= kLaneBits) {
      spec[nspec++] = b;
      if (v) fixed_or |= 1ull << b;
    } else {
      lane_mask |= 1u << b;
      if (v) lane_val |= 1u << b;
    }
  }
  Geo build() const {
    Geo g;
    g.nspec = nspec;
    g.spec[0] = spec[0];
    g.spec[1] = spec[1];
    if (nspec == 2 && g.spec[0] > g.spec[1]) std::swap(g.spec[0], g.spec[1]);
    g.fixed_or = fixed_or;
    g.lane_mask = lane_mask;
    g.lane_val = lane_val;
    g.lane_lim = (n >= kLaneBits) ? 32u : (1u << n);
    g.ntiles = (n >= kLaneBits) ? (1ull << (n - kLaneBits - nspec)) : 1ull;
    return g;
  }
};

inline unsigned blocks_for(uint64_t ntiles, int items) {
  const uint64_t warps = (ntiles + items - 1) / items;
  const uint64_t threads = warps * 32;
  return (unsigned)((threads + kThreads - 1) / kThreads);
}

}  // namespace

// host-side coefficient conversion (the values are already rounded to R)
template <typename V> static V hcoef(const double* m, int i);
template <> double2 hcoef<double2>(const double* m, int i) { return make_double2(m[2 * i], m[2 * i + 1]); }
template <> float2  hcoef<float2>(const double* m, int i)  { return make_float2((float)m[2 * i], (float)m[2 * i + 1]); }
template <> double  hcoef<double>(const double* m, int i)  { return m[2 * i]; }
template <> float   hcoef<float>(const double* m, int i)   { return (float)m[2 * i]; }

template <typename V>
static qsv_status launch_typed(qsv_state_s* s, const Lowered& L) {
  V* st = static_cast<V*>(s->d);
  const int n = s->n;
  cudaStream_t str = s->stream;
  GeoBuilder gb(n);
  switch (L.shape) {
    case SH_NONE:
      return QSV_SUCCESS;
    case SH_PAIR:
    case SH_CPAIR: {
      M2<V> M{hcoef<V>(L.m, 0), hcoef<V>(L.m, 1), hcoef<V>(L.m, 2), hcoef<V>(L.m, 3)};
      if (L.shape == SH_CPAIR) gb.fix(L.t1, L.cval);
      if (L.t0 >= kLaneBits) {
        gb.reg(L.t0);
        Geo g = gb.build();
        constexpr int I = 2;
        k_pair_reg<V, I><<<blocks_for(g.ntiles, I), kThreads, 0, str>>>(st, g, n, 1ull << L.t0, M,
                                                                        L.form);
      } else {
        Geo g = gb.build();
        constexpr int I = 4;
        k_pair_lane<V, I><<<blocks_for(g.ntiles, I), kThreads, 0, str>>>(st, g, n, L.t0, M,
                                                                         L.form);
      }
      break;
    }
    case SH_HALF:
    case SH_CHALF: {
      gb.fix(L.t0, 1);
      if (L.shape == SH_CHALF) gb.fix(L.t1, L.cval);
      Geo g = gb.build();
      constexpr int I = 4;
      k_scale<V, I><<<blocks_for(g.ntiles, I), kThreads, 0, str>>>(st, g, n, hcoef<V>(L.m, 0),
                                                                   L.form);
      break;
    }
    case SH_QUAD: {
      M4<V> M;
      for (int i = 0; i < 16; ++i) M.a[i] = hcoef<V>(L.m, i);
      if (L.t1 >= kLaneBits) {
        gb.reg(L.t0);
        gb.reg(L.t1);
        Geo g = gb.build();
        constexpr int I = 1;
        k_quad_reg2<V, I><<<blocks_for(g.ntiles, I), kThreads, 0, str>>>(
            st, g, n, 1ull << L.t0, 1ull << L.t1, M);
      } else if (L.t0 >= kLaneBits) {
        gb.reg(L.t0);
        Geo g = gb.build();
        constexpr int I = 2;
        k_quad_reg1<V, I><<<blocks_for(g.ntiles, I), kThreads, 0, str>>>(
            st, g, n, 1ull << L.t0, L.t1, M);
      } else {
        Geo g = gb.build();
        constexpr int I = 4;
        k_quad_lane<V, I><<<blocks_for(g.ntiles, I), kThreads, 0, str>>>(st, g, n, L.t0, L.t1, M);
      }
      break;
    }
    case SH_SWAP: {
      const V lam = hcoef<V>(L.m, 0);
      if (L.t1 >= kLaneBits) {
        gb.reg(L.t0);
        gb.reg(L.t1);
        Geo g = gb.build();
        constexpr int I = 2;
        if (L.mul)
          k_swap_reg2<V, true, I><<<blocks_for(g.ntiles, I), kThreads, 0, str>>>(st, g, n, 1ull << L.t0, 1ull << L.t1, lam);
        else
          k_swap_reg2<V, false, I><<<blocks_for(g.ntiles, I), kThreads, 0, str>>>(st, g, n, 1ull << L.t0, 1ull << L.t1, lam);
      } else if (L.t0 >= kLaneBits) {
        gb.reg(L.t0);
        Geo g = gb.build();
        constexpr int I = 4;
        if (L.mul)
          k_swap_reg1<V, true, I><<<blocks_for(g.ntiles, I), kThreads, 0, str>>>(st, g, n, 1ull << L.t0, L.t1, lam);
        else
          k_swap_reg1<V, false, I><<<blocks_for(g.ntiles, I), kThreads, 0, str>>>(st, g, n, 1ull << L.t0, L.t1, lam);
      } else {
        Geo g = gb.build();
        constexpr int I = 4;
        if (L.mul)
          k_swap_lane<V, true, I><<<blocks_for(g.ntiles, I), kThreads, 0, str>>>(st, g, n, L.t0, L.t1, lam);
        else
          k_swap_lane<V, false, I><<<blocks_for(g.ntiles, I), kThreads, 0, str>>>(st, g, n, L.t0, L.t1, lam);
      }
      break;
    }
    default:
      return fail(QSV_ERROR_INVALID_VALUE, "unknown lowered shape %d", L.shape);
  }
  count_launch();
  return cuda_status(cudaGetLastError(), "unfused gate kernel launch");
}

qsv_status launch_unfused(qsv_state_s* s, const Lowered& L) {
  switch (s->dtype) {
    case QSV_C128: return launch_typed<double2>(s, L);
    case QSV_C64:  return launch_typed<float2>(s, L);
    case QSV_F64:  return launch_typed<double>(s, L);
    case QSV_F32:  return launch_typed<float>(s, L);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

}  // namespace qsv

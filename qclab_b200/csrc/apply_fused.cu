// Fused sweeps: each stage of a plan (plan.hpp) streams the state through
// shared memory once, one 2^m-amplitude tile per CTA, and applies all of the
// stage's gates to the tile in shared memory.
//
// The same executor runs the adjoint's backward sweep: it then carries two
// vectors (psi and lambda) through every tile, applies each inverse gate to
// both, and evaluates the gradient terms w * Im(i^ny <lam| Pi P |psi>) of
// the parametric gates inside the tile (one partial sum per tile, reduced
// in a fixed order afterwards).
//
// Arithmetic here is FMA-contracted (within 1e-12 of the reference-exact
// path for complex<double>, not bitwise: the planner reorders commuting
// gates, which changes rounding).  Gates are specialised by the structure of
// their coefficients (permutation, diagonal, real, RotationX-like) because
// complex<double> sweeps with many gates per stage are bounded by the FP64
// pipe, not by HBM.
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
  F_GENERIC = 0,  // dense complex 2x2
  F_PERM = 1,     // [[0,1],[1,0]]
  F_DIAG = 2,     // diagonal
  F_REAL = 3,     // all entries real
  F_RXLIKE = 4    // real diagonal, imaginary off-diagonal
};

struct FOp {
  int8_t shape;
  int8_t form;
  int8_t j0, j1;   // local bits (PAIR/HALF/CPAIR/CHALF: j0 = target, j1 = control)
  int8_t cval;
  int8_t mul;
  int8_t ny;       // SH_RED: number of Y factors
  int8_t w;        // SH_RED: weight
  int16_t coef;    // stage-relative index of the first coefficient
  uint16_t f, zy, pm, pv;  // SH_RED: local masks
  int32_t slot;    // SH_RED: row of the partial-sum matrix
};

struct StageArgs {
  TileArgs ta;
  int nops;
  const FOp* ops;
  const void* coefs;
  double* partial;  // [slot][tile] partial sums of the SH_RED ops
};

__device__ __forceinline__ uint32_t ins0(uint32_t x, int p) {
  return ((x >> p) << (p + 1)) | (x & ((1u << p) - 1u));
}

// ---- 2x2 application with coefficient-structure specialisation -----------
__device__ __forceinline__ void pair2(int form, const double2* c, double2& x1, double2& x2) {
  switch (form) {
    case F_PERM: { const double2 t = x1; x1 = x2; x2 = t; return; }
    case F_DIAG: { x1 = fmul(c[0], x1); x2 = fmul(c[3], x2); return; }
    case F_REAL: {
      const double a = c[0].x, b = c[1].x, d = c[2].x, e = c[3].x;
      const double2 y1 = make_double2(fma(a, x1.x, b * x2.x), fma(a, x1.y, b * x2.y));
      const double2 y2 = make_double2(fma(d, x1.x, e * x2.x), fma(d, x1.y, e * x2.y));
      x1 = y1; x2 = y2; return;
    }
    case F_RXLIKE: {
      // y1 = a*x1 + i*b*x2, y2 = i*d*x1 + e*x2 (a,e real; b,d imaginary parts)
      const double a = c[0].x, b = c[1].y, d = c[2].y, e = c[3].x;
      const double2 y1 = make_double2(fma(a, x1.x, -b * x2.y), fma(a, x1.y, b * x2.x));
      const double2 y2 = make_double2(fma(e, x2.x, -d * x1.y), fma(e, x2.y, d * x1.x));
      x1 = y1; x2 = y2; return;
    }
    default: {
      const double2 y1 = fmac(fmul(c[0], x1), c[1], x2);
      const double2 y2 = fmac(fmul(c[2], x1), c[3], x2);
      x1 = y1; x2 = y2; return;
    }
  }
}
__device__ __forceinline__ void pair2(int form, const float2* c, float2& x1, float2& x2) {
  switch (form) {
    case F_PERM: { const float2 t = x1; x1 = x2; x2 = t; return; }
    case F_DIAG: { x1 = fmul(c[0], x1); x2 = fmul(c[3], x2); return; }
    case F_REAL: {
      const float a = c[0].x, b = c[1].x, d = c[2].x, e = c[3].x;
      const float2 y1 = make_float2(fmaf(a, x1.x, b * x2.x), fmaf(a, x1.y, b * x2.y));
      const float2 y2 = make_float2(fmaf(d, x1.x, e * x2.x), fmaf(d, x1.y, e * x2.y));
      x1 = y1; x2 = y2; return;
    }
    case F_RXLIKE: {
      const float a = c[0].x, b = c[1].y, d = c[2].y, e = c[3].x;
      const float2 y1 = make_float2(fmaf(a, x1.x, -b * x2.y), fmaf(a, x1.y, b * x2.x));
      const float2 y2 = make_float2(fmaf(e, x2.x, -d * x1.y), fmaf(e, x2.y, d * x1.x));
      x1 = y1; x2 = y2; return;
    }
    default: {
      const float2 y1 = fmac(fmul(c[0], x1), c[1], x2);
      const float2 y2 = fmac(fmul(c[2], x1), c[3], x2);
      x1 = y1; x2 = y2; return;
    }
  }
}
template <typename R>
__device__ __forceinline__ void pair2(int form, const R* c, R& x1, R& x2) {
  if (form == F_PERM) { const R t = x1; x1 = x2; x2 = t; return; }
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

template <typename V>
__device__ __forceinline__ void apply_op(V* __restrict__ tile, int m, const FOp& op,
                                         const V* __restrict__ cf) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  switch (op.shape) {
    case SH_PAIR: {
      const uint32_t cnt = 1u << (m - 1), tb = 1u << op.j0;
      V c[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) c[i] = cf[op.coef + i];
      for (uint32_t k = tid; k < cnt; k += nthr) {
        const uint32_t a = ins0(k, op.j0), b = a | tb;
        V x1 = tile[a], x2 = tile[b];
        pair2(op.form, c, x1, x2);
        tile[a] = x1; tile[b] = x2;
      }
      break;
    }
    case SH_HALF: {
      const uint32_t cnt = 1u << (m - 1), tb = 1u << op.j0;
      const V c = cf[op.coef];
      for (uint32_t k = tid; k < cnt; k += nthr) {
        const uint32_t b = ins0(k, op.j0) | tb;
        tile[b] = scale1(c, tile[b]);
      }
      break;
    }
    case SH_CPAIR: {
      const uint32_t cnt = 1u << (m - 2), tb = 1u << op.j0;
      const int lo = min(op.j0, op.j1), hi = max(op.j0, op.j1);
      const uint32_t cb = (uint32_t)op.cval << op.j1;
      V c[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) c[i] = cf[op.coef + i];
      for (uint32_t k = tid; k < cnt; k += nthr) {
        const uint32_t a = ins0(ins0(k, lo), hi) | cb, b = a | tb;
        V x1 = tile[a], x2 = tile[b];
        pair2(op.form, c, x1, x2);
        tile[a] = x1; tile[b] = x2;
      }
      break;
    }
    case SH_CHALF: {
      const uint32_t cnt = 1u << (m - 2);
      const int lo = min(op.j0, op.j1), hi = max(op.j0, op.j1);
      const uint32_t fix = (1u << op.j0) | ((uint32_t)op.cval << op.j1);
      const V c = cf[op.coef];
      for (uint32_t k = tid; k < cnt; k += nthr) {
        const uint32_t b = ins0(ins0(k, lo), hi) | fix;
        tile[b] = scale1(c, tile[b]);
      }
      break;
    }
    case SH_QUAD: {
      // j0 = local bit of qubits[0] (higher), j1 = of qubits[1]
      const uint32_t cnt = 1u << (m - 2), m0 = 1u << op.j0, m1 = 1u << op.j1;
      const V* c = cf + op.coef;
      for (uint32_t k = tid; k < cnt; k += nthr) {
        const uint32_t a = ins0(ins0(k, op.j1), op.j0);
        const V x0 = tile[a], x1 = tile[a | m0], x2 = tile[a | m1], x3 = tile[a | m0 | m1];
        V y[4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
          y[r] = mac(mac(mac(scale1(c[4 * r], x0), c[4 * r + 1], x1), c[4 * r + 2], x2),
                     c[4 * r + 3], x3);
        tile[a] = y[0]; tile[a | m0] = y[1]; tile[a | m1] = y[2]; tile[a | m0 | m1] = y[3];
      }
      break;
    }
    case SH_SWAP: {
      const uint32_t cnt = 1u << (m - 2), m0 = 1u << op.j0, m1 = 1u << op.j1;
      const V c = cf[op.coef];
      for (uint32_t k = tid; k < cnt; k += nthr) {
        const uint32_t a = ins0(ins0(k, op.j1), op.j0);
        const V xb = tile[a | m0], xc = tile[a | m1];
        tile[a | m0] = op.mul ? scale1(c, xc) : xc;
        tile[a | m1] = op.mul ? scale1(c, xb) : xb;
      }
      break;
    }
    default:
      break;
  }
}

// w * Im(i^ny * sum_{e in tile, (e & pm) == pv} conj(lam_e) (-1)^{pop((e^f)&zy)} psi_{e^f})
template <typename V>
__device__ __forceinline__ double red_op(const V* __restrict__ psi, const V* __restrict__ lam,
                                         int m, const FOp& op) {
  const uint32_t size = 1u << m;
  double2 s = make_double2(0.0, 0.0);
  for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) {
    if ((e & op.pm) != op.pv) continue;
    const uint32_t p = e ^ op.f;
    const double sg = (__popc(p & op.zy) & 1) ? -1.0 : 1.0;
    const double2 l = to_d2(lam[e]), x = to_d2(psi[p]);
    s.x = fma(sg * l.x, x.x, fma(sg * l.y, x.y, s.x));
    s.y = fma(sg * l.x, x.y, fma(-sg * l.y, x.x, s.y));
  }
  // Im(i^ny s)
  double im;
  switch (op.ny & 3) {
    case 0: im = s.y; break;
    case 1: im = s.x; break;
    case 2: im = -s.y; break;
    default: im = -s.x; break;
  }
  return op.w * im;
}

template <typename V, int NV>
__global__ void __launch_bounds__(512)
k_stage(V* __restrict__ v0, V* __restrict__ v1, StageArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double2 red[32];
  const int m = a.ta.m, low = a.ta.low;
  const uint32_t size = 1u << m, lowmask = (1u << low) - 1u;
  V* t0 = reinterpret_cast<V*>(smem_raw);
  V* t1 = t0 + size;
  const uint64_t* __restrict__ runoff = a.ta.runoff;
  const V* __restrict__ coefs = static_cast<const V*>(a.coefs);
  const uint64_t base = tile_base(a.ta, blockIdx.x);

#pragma unroll 4
  for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) {
    const uint64_t g = base | runoff[e >> low] | (e & lowmask);
    t0[e] = v0[g];
    if (NV == 2) t1[e] = v1[g];
  }
  __syncthreads();
  for (int i = 0; i < a.nops; ++i) {
    const FOp op = a.ops[i];
    if (op.shape == SH_RED) {
      if (NV == 2) {
        const double r = red_op<V>(t0, t1, m, op);
        const double2 tot = block_sum(make_double2(r, 0.0), red);
        if (threadIdx.x == 0) a.partial[(size_t)op.slot * gridDim.x + blockIdx.x] = tot.x;
      }
    } else {
      apply_op<V>(t0, m, op, coefs);
      if (NV == 2) apply_op<V>(t1, m, op, coefs);
    }
    __syncthreads();
  }
#pragma unroll 4
  for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) {
    const uint64_t g = base | runoff[e >> low] | (e & lowmask);
    v0[g] = t0[e];
    if (NV == 2) v1[g] = t1[e];
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

template <typename V>
qsv_status execute_typed(const ExecArgs& x) {
  constexpr bool cplx = Elem<V>::cplx;
  qsv_state_s* s = x.s;
  const int n = s->n;
  const qsv_fuse_opts* opts = x.opts;
  int m = (opts && opts->tile_bits > 0) ? opts->tile_bits : default_tile_bits(sizeof(V), x.nv);
  int low = (opts && opts->low_bits > 0) ? opts->low_bits : default_low_bits(sizeof(V));
  const int max_gates = (opts && opts->max_stage_gates > 0) ? opts->max_stage_gates : 256;
  if (m > 14) m = 14;
  if (m > n) m = n;
  if (low > m) low = m;
  const size_t smem = (size_t(1) << m) * sizeof(V) * x.nv;
  if (smem > 200 * 1024)
    return fail(QSV_ERROR_SIZE, "tile of %d x 2^%d elements exceeds shared memory", x.nv, m);

  const std::vector<Lowered>& gates = *x.items;
  std::vector<Stage> stages = plan_stages(gates, n, m, low, max_gates);
  if (stages.empty()) return QSV_SUCCESS;

  // pack ops, coefficients and run offsets of every stage into one buffer
  std::vector<FOp> ops;
  std::vector<V> coefs;
  std::vector<uint64_t> runoff;
  struct Meta { size_t op0, nops, run0, coef0; };
  std::vector<Meta> meta;
  for (const Stage& stg : stages) {
    Meta mt{ops.size(), stg.gates.size(), runoff.size(), coefs.size()};
    int local_of[64];
    for (int j = 0; j < 64; ++j) local_of[j] = -1;
    for (int j = 0; j < stg.m; ++j) local_of[stg.bits[j]] = j;
    auto local_mask = [&](uint64_t g) {
      uint32_t r = 0;
      for (int b = 0; b < n; ++b)
        if ((g >> b) & 1ull) r |= 1u << local_of[b];
      return (uint16_t)r;
    };
    for (int gi : stg.gates) {
      const Lowered& L = gates[gi];
      FOp op{};
      op.shape = (int8_t)L.shape;
      if (L.shape == SH_RED) {
        op.f = local_mask(L.gen.f);
        op.zy = local_mask(L.gen.zy);
        op.pm = local_mask(L.gen.pm);
        op.pv = local_mask(L.gen.pv);
        op.ny = (int8_t)L.gen.ny;
        op.w = (int8_t)L.gen.w;
        op.slot = L.slot;
        ops.push_back(op);
        continue;
      }
      op.form = classify(L, cplx);
      op.j0 = (int8_t)local_of[L.t0];
      op.j1 = (L.shape == SH_PAIR || L.shape == SH_HALF) ? 0 : (int8_t)local_of[L.t1];
      op.cval = (int8_t)L.cval;
      op.mul = (int8_t)L.mul;
      // coefficient index relative to the stage's first coefficient
      if (coefs.size() - mt.coef0 > 30000) return fail(QSV_ERROR_SIZE, "fused stage too large");
      op.coef = (int16_t)(coefs.size() - mt.coef0);
      const int nc = (L.shape == SH_QUAD) ? 16 : (L.shape == SH_PAIR || L.shape == SH_CPAIR) ? 4 : 1;
      for (int i = 0; i < nc; ++i) coefs.push_back(host_coef<V>(L.m, i));
      ops.push_back(op);
    }
    tile_runoffs(stg.bits, stg.m, low, &runoff);
    meta.push_back(mt);
  }
  const size_t ops_bytes = ops.size() * sizeof(FOp);
  const size_t coef_off = (ops_bytes + 255) & ~size_t(255);
  const size_t coef_bytes = coefs.size() * sizeof(V);
  const size_t run_off = (coef_off + coef_bytes + 255) & ~size_t(255);
  const size_t total = run_off + runoff.size() * sizeof(uint64_t);
  std::vector<unsigned char> host(total);
  std::memcpy(host.data(), ops.data(), ops_bytes);
  std::memcpy(host.data() + coef_off, coefs.data(), coef_bytes);
  std::memcpy(host.data() + run_off, runoff.data(), runoff.size() * sizeof(uint64_t));
  if (qsv_status st = ensure_scratch(s, total)) return st;
  unsigned char* dev = static_cast<unsigned char*>(s->scratch);
  if (qsv_status st = cuda_status(cudaMemcpyAsync(dev, host.data(), total, cudaMemcpyHostToDevice,
                                                  s->stream), "fused plan upload"))
    return st;

  auto kern = (x.nv == 2) ? k_stage<V, 2> : k_stage<V, 1>;
  if (qsv_status st = cuda_status(
          cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024),
          "fused stage shared-memory attribute"))
    return st;
  const int threads = std::min<int>(512, std::max<int>(32, (1 << m) / 8));
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
  for (size_t si = 0; si < stages.size(); ++si) {
    StageArgs a;
    a.ta.n = n;
    a.ta.m = stages[si].m;
    a.ta.low = low;
    for (int j = 0; j < 64; ++j) a.ta.bits[j] = (j < stages[si].m) ? (int8_t)stages[si].bits[j] : 0;
    a.ta.runoff = reinterpret_cast<const uint64_t*>(dev + run_off) + meta[si].run0;
    a.nops = (int)meta[si].nops;
    a.ops = reinterpret_cast<const FOp*>(dev) + meta[si].op0;
    a.coefs = dev + coef_off + meta[si].coef0 * sizeof(V);
    a.partial = x.partial;
    kern<<<(unsigned)ntiles, threads, smem, s->stream>>>(static_cast<V*>(x.v0),
                                                         static_cast<V*>(x.v1), a);
    count_launch();
    if (qsv_status st = cuda_status(cudaGetLastError(), "fused stage launch")) return st;
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
int default_low_bits(size_t eb) { return eb >= 16 ? 4 : 5; }

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

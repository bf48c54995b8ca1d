// Fused sweeps: each stage of a plan (plan.hpp) streams the state through
// shared memory once, one 2^m-amplitude tile per CTA, and applies all of the
// stage's gates to the tile before writing it back.  The gates of a stage
// run as register passes (stage_exec.cuh): one shared-memory round trip per
// pass instead of one per gate.
//
// The same executor runs the adjoint's backward sweep: it then carries two
// vectors (psi and lambda) through every tile, applies each inverse gate to
// both, and evaluates the gradient terms w * Im(i^ny <lam| Pi P |psi>) of
// the parametric gates in registers (one partial sum per tile, reduced in a
// fixed order afterwards).
//
// Arithmetic here is FMA-contracted (within 1e-12 of the reference-exact
// path for complex<double>, not bitwise: the planner reorders commuting
// gates, which changes rounding).
#include <algorithm>
#include <atomic>
#include <mutex>
#include <array>
#include <complex>
#include <initializer_list>
#include <thread>
#include <type_traits>
#include <cstring>
#include <unordered_map>
#include <vector>
#include "fused.hpp"
#include "stage_exec.cuh"
#include "tcgen05.cuh"
#include "tma.cuh"

namespace qsv {

static thread_local std::vector<float> g_stage_ms;

StageTimer::StageTimer(bool on, size_t nstages, cudaStream_t stream)
    : on_(on), stream_(stream), ev_(on ? nstages + 1 : 0, nullptr) {}

StageTimer::~StageTimer() {
  for (cudaEvent_t e : ev_)
    if (e) cudaEventDestroy(e);
}

qsv_status StageTimer::start() {
  if (!on_) return QSV_SUCCESS;
  for (auto& e : ev_)
    if (qsv_status st = cuda_status(cudaEventCreate(&e), "cudaEventCreate")) return st;
  return cuda_status(cudaEventRecord(ev_[0], stream_), "cudaEventRecord");
}

qsv_status StageTimer::mark(size_t stage) {
  if (!on_) return QSV_SUCCESS;
  return cuda_status(cudaEventRecord(ev_[stage + 1], stream_), "cudaEventRecord");
}

qsv_status StageTimer::finish() {
  if (!on_) return QSV_SUCCESS;
  if (qsv_status st = cuda_status(cudaEventSynchronize(ev_.back()), "stage timing synchronize"))
    return st;
  g_stage_ms.clear();
  for (size_t i = 0; i + 1 < ev_.size(); ++i) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev_[i], ev_[i + 1]);
    g_stage_ms.push_back(ms);
  }
  return QSV_SUCCESS;
}
static std::atomic<bool> g_tc_used{false};  // a tcgen05 sweep was launched

namespace fx {

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

using cplxd = std::complex<double>;

// Host mirror of apply_reg: op on the 2^R amplitudes of one register group,
// with FP64 coefficients c (the same semantics as pair2f / quad_reg /
// the P_MUL loop).
void host_apply_pop(std::vector<cplxd>& x, int R, const POp& op, const cplxd* c) {
  const int N = 1 << R;
  switch (op.shape) {
    case P_PAIR:
    case P_CPAIR: {
      const int mt = 1 << op.p0;
      const int cm = op.shape == P_CPAIR ? (1 << op.p1) : 0;
      const int cv = op.shape == P_CPAIR ? (op.cval << op.p1) : 0;
      for (int j = 0; j < N; ++j) {
        if ((j & mt) || (j & cm) != cv) continue;
        const cplxd x1 = x[j], x2 = x[j | mt];
        if (op.form == F_PERM) {
          x[j] = x2;
          x[j | mt] = x1;
        } else {
          x[j] = c[0] * x1 + c[1] * x2;
          x[j | mt] = c[2] * x1 + c[3] * x2;
        }
      }
      break;
    }
    case P_MUL:
      for (int j = 0; j < N; ++j)
        if ((j & op.mmask) == op.mval) x[j] *= c[0];
      break;
    case P_QUAD: {
      const int m0 = 1 << op.p0, m1 = 1 << op.p1;
      for (int j = 0; j < N; ++j) {
        if ((j & m0) || (j & m1)) continue;
        if (op.form == F_PERM) {
          const cplxd xb = x[j | m0], xc = x[j | m1];
          x[j | m0] = op.mul ? c[0] * xc : xc;
          x[j | m1] = op.mul ? c[0] * xb : xb;
        } else {
          const cplxd in[4] = {x[j], x[j | m0], x[j | m1], x[j | m0 | m1]};
          cplxd y[4];
          for (int rr = 0; rr < 4; ++rr)
            y[rr] = c[4 * rr] * in[0] + c[4 * rr + 1] * in[1] + c[4 * rr + 2] * in[2] +
                    c[4 * rr + 3] * in[3];
          x[j] = y[0];
          x[j | m0] = y[1];
          x[j | m1] = y[2];
          x[j | m0 | m1] = y[3];
        }
      }
      break;
    }
    default:
      break;
  }
}

template <typename V> V dense_coef(cplxd z);
template <> double2 dense_coef<double2>(cplxd z) { return make_double2(z.real(), z.imag()); }
template <> float2 dense_coef<float2>(cplxd z) {
  return make_float2((float)z.real(), (float)z.imag());
}
template <> double dense_coef<double>(cplxd z) { return z.real(); }
template <> float dense_coef<float>(cplxd z) { return (float)z.real(); }

template <typename V>
qsv_status pack_plan(const std::vector<Lowered>& gates, int n, int m, int low, int r,
                     int max_gates, PackedPlan<V>* out, int dense_min, size_t plan_cap,
                     bool search_passes) {
  const int min_ops = dense_min >= 0 ? dense_min : QSV_DENSE_MIN_OPS;
  constexpr bool cplx = Elem<V>::cplx;
  std::vector<Stage> stages =
      plan_stages(gates, n, m, low, max_gates, kMaxRed, kPlanSmemMax, sizeof(V));
  for (const Stage& stg : stages) {
    PackedStage ps;
    ps.m = stg.m;
    ps.full = 0;
    ps.red0 = out->red_slots.size();
    ps.nred = 0;
    for (int gi : stg.gates)
      if (gates[gi].shape == SH_QUAD || gates[gi].shape == SH_RED) ps.full = 1;
    for (int j = 0; j < 64; ++j) ps.bits[j] = (j < stg.m) ? stg.bits[j] : 0;
    ps.pass0 = out->passes.size();
    ps.op0 = out->ops.size();
    ps.run0 = out->runoff.size();
    ps.coef0 = out->coefs.size();
    int local_of[64];
    for (int j = 0; j < 64; ++j) local_of[j] = -1;
    for (int j = 0; j < stg.m; ++j) local_of[stg.bits[j]] = j;
    auto local_mask = [&](uint64_t g) {
      uint32_t lm = 0;
      for (int b = 0; b < n; ++b)
        if ((g >> b) & 1ull) lm |= 1u << local_of[b];
      return lm;
    };
    std::vector<uint32_t> op_bits;
    for (int gi : stg.gates) op_bits.push_back(local_mask(gate_bits(gates[gi])));
    std::vector<Pass> pl = plan_passes(op_bits, stg.m, r, search_passes);
    // Phase 1: every pass packed sparse into its own buffers (op.coef
    // relative to the pass), with its coefficients also kept in FP64.
    struct PassBuf {
      PassDev pd;
      int r;
      std::vector<POp> ops;
      std::vector<V> coefs;
      std::vector<cplxd> c64;
      bool red = false;
    };
    std::vector<PassBuf> bufs(pl.size());
    for (size_t pi = 0; pi < pl.size(); ++pi) {
      const Pass& p = pl[pi];
      PassBuf& B = bufs[pi];
      B.r = p.r;
      PassDev& pd = B.pd;
      pd = PassDev{};
      for (int k = 0; k < 8; ++k) pd.pos[k] = (k < p.r) ? (int8_t)p.pos[k] : 0;
      for (int j = 0; j < (1 << p.r) && j < 32; ++j) {
        uint32_t pat = 0;
        for (int k = 0; k < p.r; ++k)
          if ((j >> k) & 1) pat |= 1u << p.pos[k];
        pd.off[j] = (uint16_t)phys_host(pat, Units<V>::per);
      }
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
        op.coef = (int16_t)B.coefs.size();
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
            if (L.m[0] == -1.0 && L.m[1] == 0.0) {  // CZ: negation, positions compile-time
              op.form = F_NEG;
              op.p0 = reg_pos(L.t0);
              op.p1 = reg_pos(L.t1);
              op.cval = (int8_t)L.cval;
            }
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
            if (ps.nred >= kMaxRed) return fail(QSV_ERROR_INVALID_VALUE, "internal: stage reductions");
            op.ridx = (int16_t)ps.nred++;
            out->red_slots.push_back(L.slot);
            B.red = true;
            break;
          }
          default:
            return fail(QSV_ERROR_INVALID_VALUE, "internal: shape %d in a fused stage", L.shape);
        }
        for (int i = 0; i < nc; ++i) {
          B.coefs.push_back(host_coef<V>(L.m, i));
          B.c64.push_back(cplx ? cplxd(L.m[2 * i], L.m[2 * i + 1]) : cplxd(L.m[2 * i], 0.0));
        }
        B.ops.push_back(op);
      }
    }
    // Phase 2: multiply passes out into one dense 2^r x 2^r op (no gradient
    // terms, enough ops) while the stage's plan stays within its budget.
    size_t nops_total = 0, ncoef_total = 0;
    for (const PassBuf& B : bufs) {
      nops_total += B.ops.size();
      ncoef_total += B.coefs.size();
    }
    for (PassBuf& B : bufs) {
      const int N = 1 << B.r;
      if (min_ops <= 0 || B.r != r || r > QSV_DENSE_MAX_R || B.red || (int)B.ops.size() < min_ops)
        continue;
      const size_t nops_after = nops_total - B.ops.size() + 1;
      const size_t ncoef_after = ncoef_total - B.coefs.size() + size_t(N) * N;
      if (plan_smem_bytes<V>((int)bufs.size(), (int)nops_after, (int)ncoef_after) > plan_cap)
        continue;
      std::vector<cplxd> U(size_t(N) * N);  // column-major: U[k * N + i]
      std::vector<cplxd> x(N);
      for (int k = 0; k < N; ++k) {
        std::fill(x.begin(), x.end(), cplxd(0.0, 0.0));
        x[k] = 1.0;
        for (const POp& q : B.ops) host_apply_pop(x, B.r, q, B.c64.data() + q.coef);
        for (int i = 0; i < N; ++i) U[size_t(k) * N + i] = x[i];
      }
      bool real = true, diagonal = true;
      for (int k = 0; k < N; ++k)
        for (int i = 0; i < N; ++i) {
          const cplxd z = U[size_t(k) * N + i];
          if (z.imag() != 0.0) real = false;
          if (i != k && z != cplxd(0.0, 0.0)) diagonal = false;
        }
      POp d{};
      d.shape = P_DENSE;
      d.form = diagonal ? kDenseDiagonal : (real ? kDenseReal : kDenseGeneral);
      d.coef = 0;
      B.ops.assign(1, d);
      B.coefs.clear();
      for (const cplxd& z : U) B.coefs.push_back(dense_coef<V>(z));
      nops_total = nops_after;
      ncoef_total = ncoef_after;
    }
    // Phase 3: append (op.coef and PassDev.op0 relative to the stage).
    for (PassBuf& B : bufs) {
      if (out->coefs.size() - ps.coef0 + B.coefs.size() > 30000)
        return fail(QSV_ERROR_SIZE, "fused stage too large");
      B.pd.op0 = (int32_t)(out->ops.size() - ps.op0);
      B.pd.nops = (int32_t)B.ops.size();
      const int16_t cbase = (int16_t)(out->coefs.size() - ps.coef0);
      for (POp q : B.ops) {
        q.coef = (int16_t)(q.coef + cbase);
        out->ops.push_back(q);
      }
      out->coefs.insert(out->coefs.end(), B.coefs.begin(), B.coefs.end());
      out->passes.push_back(B.pd);
    }
    ps.npasses = out->passes.size() - ps.pass0;
    ps.nops = (int)(out->ops.size() - ps.op0);
    ps.ncoef = (int)(out->coefs.size() - ps.coef0);
    if (plan_smem_bytes<V>((int)ps.npasses, ps.nops, ps.ncoef) > plan_cap)
      return fail(QSV_ERROR_INVALID_VALUE, "internal: stage plan exceeds its shared-memory budget");
    tile_runoffs(stg.bits, stg.m, low, &out->runoff);
    out->stages.push_back(ps);
  }
  return QSV_SUCCESS;
}

template qsv_status pack_plan<double2>(const std::vector<Lowered>&, int, int, int, int, int, PackedPlan<double2>*, int, size_t, bool);
template qsv_status pack_plan<float2>(const std::vector<Lowered>&, int, int, int, int, int, PackedPlan<float2>*, int, size_t, bool);
template qsv_status pack_plan<double>(const std::vector<Lowered>&, int, int, int, int, int, PackedPlan<double>*, int, size_t, bool);
template qsv_status pack_plan<float>(const std::vector<Lowered>&, int, int, int, int, int, PackedPlan<float>*, int, size_t, bool);

}  // namespace fx

// Register bits of a pass for a tile of m bits (fewer for tiny tiles).
int pass_bits(size_t eb, int nv, int m) {
  const int rdef = (eb >= 16) ? fx::reg_bits<double2>(nv) : fx::reg_bits<float2>(nv);
  return (m >= rdef) ? rdef : (m >= 2 ? 2 : 1);
}

namespace {

using namespace fx;

struct Stage2Args {
  TileArgs ta;
  int npasses;
  const PassDev* passes;
  const POp* ops;
  const void* coefs;
  double* partial;           // [slot][tile] partial sums of the RED ops
  const int32_t* red_slots;  // slot of each of the stage's nred reductions
  int nred;
  int nops, ncoef;           // the stage's ops and coefficients (staged in shared memory)
  int vec16;                 // 16-byte cp.async copies allowed (alignment and run length)
};

template <typename V, int NV, int R, bool FULL>
__global__ void __launch_bounds__(256, min_blocks<V, NV>())
k_stage2(V* __restrict__ v0, V* __restrict__ v1, Stage2Args a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t size = 1u << a.ta.m;
  V* t0 = reinterpret_cast<V*>(smem_raw);
  V* t1 = t0 + size;
  // gradient accumulators after the tiles (allocated for two-vector sweeps),
  // then the stage's plan
  double* racc = reinterpret_cast<double*>(smem_raw + size_t(NV) * size * sizeof(V));
  unsigned char* plan = smem_raw + size_t(NV) * size * sizeof(V) + (NV == 2 ? kRaccBytes : 0);
  const PassDev* passes;
  const POp* ops;
  const V* coefs;
  stage_plan<V>(plan, a.passes, a.npasses, a.ops, a.nops, static_cast<const V*>(a.coefs),
                a.ncoef, &passes, &ops, &coefs);
  const bool red = NV == 2 && FULL && a.nred > 0;
  if (red)
    for (int i = threadIdx.x; i < a.nred * kRedWarps; i += blockDim.x) racc[i] = 0.0;
  const uint64_t base = tile_base(a.ta, blockIdx.x);
  load_tile<V, NV>(v0, v1, t0, t1, a.ta, base, a.vec16);
  __syncthreads();
  run_passes<V, NV, R, FULL, turn_bits<V>(NV)>(t0, t1, passes, a.npasses, ops, coefs, racc,
                                                size >> R);
  store_tile<V, NV>(v0, v1, t0, t1, a.ta, base, a.vec16);
  if (red) {  // run_passes ended with a barrier: racc is complete
    const int warps = red_warps();
    for (int r = threadIdx.x; r < a.nred; r += blockDim.x) {
      double t = 0.0;
      for (int w = 0; w < warps; ++w) t += racc[r * kRedWarps + w];
      a.partial[(size_t)a.red_slots[r] * gridDim.x + blockIdx.x] = t;
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

template <typename V, int NV, int R>
void* stage_kernel(bool full) {
  return full ? (void*)k_stage2<V, NV, R, true> : (void*)k_stage2<V, NV, R, false>;
}

template <typename V, int NV>
void* pick_kernel(int r, bool full) {
  constexpr int RD = reg_bits<V>(NV);
  if (r == RD) return stage_kernel<V, NV, RD>(full);
  if (r == 2) return stage_kernel<V, NV, 2>(full);
  return stage_kernel<V, NV, 1>(full);
}

// ---- dense register passes on the FP64 tensor cores ------------------------
// Every register pass of a stage acts on 2 tile bits with one 4x4 complex
// matrix U (the product of its gates, formed on the host in FP64).  A warp
// takes 32 groups of 4 amplitudes at a time (a "chunk") and applies the 8x8
// real matrix M = [[Re U, -Im U], [Im U, Re U]] to their (re; im) vectors
// with mma.sync m8n8k4 f64: per 8-group column tile, D = A0 B0 + A1 B1 with
//   A_s[r][k] = M[r][4s + k]          lane: r = lane / 4, k = lane % 4
//   B_s[k][g] = (s ? im : re) of amplitude k of group g     (g = lane / 4)
//   D[r][g]   -> lane: r = lane / 4, g = 2 (lane % 4) + {0, 1}
// (row r < 4: real part of output amplitude r, r >= 4: imaginary part of
// amplitude r - 4).  Amplitudes are read and written in shared memory in
// their storage type and computed in FP64.  The tile bit insertion and the
// shared-memory swizzle are linear over GF(2), so the address of (group,
// amplitude) is the XOR of a chunk part and per-lane parts.
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b,
                                            double c0, double c1) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%4, %5};"
               : "=d"(d0), "=d"(d1)
               : "d"(a), "d"(b), "d"(c0), "d"(c1));
}

struct DmmaArgs {
  TileArgs ta;
  int npasses, nops, ncoef;
  const PassDev* passes;
  const POp* ops;
  const double2* coefs;  // per pass: U column-major (U[i][k] at k * 4 + i)
  int vec16;
  // k_dmma3: tile staging by TMA (tma.use, map passed beside) or cp.async
  TmaGeo tma;
  unsigned* wait_error;
  uint32_t smem_bytes;
};

template <typename V>
__global__ void __launch_bounds__(256, 3) k_dmma(V* __restrict__ v0, DmmaArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t size = 1u << a.ta.m;
  V* t0 = reinterpret_cast<V*>(smem_raw);
  const PassDev* passes;
  const POp* ops;
  const double2* coefs;
  stage_plan<double2>(smem_raw + size_t(size) * sizeof(V), a.passes, a.npasses, a.ops, a.nops,
                      a.coefs, a.ncoef, &passes, &ops, &coefs);
  const uint64_t base = tile_base(a.ta, blockIdx.x);
  load_tile<V, 1>(v0, nullptr, t0, nullptr, a.ta, base, a.vec16);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int q = lane >> 2, k4 = lane & 3;
  const bool im_row = q >= 4;
  const uint32_t nchunks = size >> 7;  // 32 groups x 4 amplitudes
  for (int pi = 0; pi < a.npasses; ++pi) {
    const PassDev& P = passes[pi];
    const uint16_t* T = P.off;  // address tables (dmma_tables)
    const double2 u = coefs[ops[P.op0].coef + k4 * 4 + (q & 3)];  // U[q % 4][k4]
    const double a0 = im_row ? u.y : u.x;
    const double a1 = im_row ? u.x : -u.y;
    // input (group q, amplitude k4); output (amplitude q % 4, group 2 k4 +
    // im_row) after the real/imaginary exchange between lanes l and l ^ 16
    const uint32_t in_lane = (uint32_t)T[4 + q] ^ T[12 + k4];
    const uint32_t out_lane = (uint32_t)T[4 + 2 * k4 + (im_row ? 1 : 0)] ^ T[12 + (q & 3)];
    uint32_t col[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) col[t] = T[t];
    for (uint32_t c = warp; c < nchunks; c += nwarps) {
      uint32_t cb = 0;
      for (uint32_t cc = c, k = 0; cc; cc >>= 1, ++k)
        if (cc & 1u) cb ^= T[16 + k];
      double b0[4], b1[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const double2 xv = to_d2(t0[cb ^ col[t] ^ in_lane]);
        b0[t] = xv.x;
        b1[t] = xv.y;
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        double d0, d1;
        dmma_m8n8k4(d0, d1, a0, b0[t], 0.0, 0.0);
        dmma_m8n8k4(d0, d1, a1, b1[t], d0, d1);
        // lane l < 16 holds the real parts of amplitude q for groups 2k4 and
        // 2k4 + 1, lane l ^ 16 the imaginary parts: swap one value each
        const double recv = __shfl_xor_sync(0xffffffffu, im_row ? d0 : d1, 16);
        t0[cb ^ col[t] ^ out_lane] =
            from_d2<V>(im_row ? make_double2(recv, d1) : make_double2(d0, recv));
      }
    }
    __syncthreads();
  }
  store_tile<V, 1>(v0, nullptr, t0, nullptr, a.ta, base, a.vec16);
}

// Three-bit passes: the 8x8 complex U as the 16x16 real matrix M (rows /
// columns 0-7: real parts of amplitudes 0-7, 8-15: imaginary parts); per
// 8-group column tile and row half h, D_h = sum_s A_hs B_s over 4 k-steps
//   A_hs[r][k] = M[8h + r][4s + k],  B_s[k][g] = row 4s + k of group g,
// so one lane ends with the real (h = 0) and imaginary (h = 1) parts of the
// same output amplitude q for groups 2k4 and 2k4 + 1: 32 MMAs per chunk of
// 32 groups x 8 amplitudes, one 16-byte store per output.
template <typename V>
__global__ void __launch_bounds__(256, 2)
    k_dmma3(V* __restrict__ v0, DmmaArgs a, const __grid_constant__ CUtensorMap tm0) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  __shared__ uint64_t tile_bar;
  unsigned char* smem_raw = tma::align1024(smem_dyn);  // the launch reserves the padding
  const uint32_t size = 1u << a.ta.m;
  V* t0 = reinterpret_cast<V*>(smem_raw);
  const uint64_t base = tile_base(a.ta, blockIdx.x);
  if (a.tma.use) {  // one thread starts the tile's copies; they land while the plan is copied
    if (!tma::tile_fits<1>(a.tma, smem_dyn, t0, size * sizeof(V), a.smem_bytes, a.wait_error))
      return;
    tma::tile_start<1>(a.tma, &tm0, &tm0, t0, nullptr, base, &tile_bar);
  }
  const PassDev* passes;
  const POp* ops;
  const double2* coefs;
  stage_plan<double2>(smem_raw + size_t(size) * sizeof(V), a.passes, a.npasses, a.ops, a.nops,
                      a.coefs, a.ncoef, &passes, &ops, &coefs);
  if (a.tma.use) {
    if (!tma::tile_wait(&tile_bar, a.wait_error, tma::kTileWaitLimit)) return;
    // the passes' address tables are for the cp.async layout (fewer bank
    // conflicts in the MMA operand loads than the TMA swizzle gives)
    if (a.tma.relayout) {
      tma::relayout_rows(t0, (size * sizeof(V)) >> 7, a.tma.swz);
      __syncthreads();
    }
  } else {
    load_tile<V, 1>(v0, nullptr, t0, nullptr, a.ta, base, a.vec16);
    __syncthreads();
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int q = lane >> 2, k4 = lane & 3;
  const uint32_t nchunks = size >> 8;  // 32 groups x 8 amplitudes
  for (int pi = 0; pi < a.npasses; ++pi) {
    const PassDev& P = passes[pi];
    const uint16_t* T = P.off;
    const double2* U = coefs + ops[P.op0].coef;        // U[i][k] at k * 8 + i
    const int form = ops[P.op0].form;                   // uniform over the block
    if (form == kDenseDiagonal) {
      // out_j = U[j][j] x_j, in place: lane (q, k4) owns amplitudes k4 and
      // 4 + k4 of group q in every column tile
      const double2 d0 = U[k4 * 8 + k4], d1 = U[(4 + k4) * 8 + 4 + k4];
      const uint32_t in0 = (uint32_t)T[4 + q] ^ T[12 + k4];
      const uint32_t in1 = (uint32_t)T[4 + q] ^ T[12 + 4 + k4];
      for (uint32_t c = warp; c < nchunks; c += nwarps) {
        uint32_t cb = 0;
        for (uint32_t cc = c, k = 0; cc; cc >>= 1, ++k)
          if (cc & 1u) cb ^= T[20 + k];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const uint32_t tb = cb ^ T[t];
          const double2 x0 = to_d2(t0[tb ^ in0]), x1 = to_d2(t0[tb ^ in1]);
          t0[tb ^ in0] = from_d2<V>(make_double2(fma(d0.x, x0.x, -d0.y * x0.y),
                                                 fma(d0.x, x0.y, d0.y * x0.x)));
          t0[tb ^ in1] = from_d2<V>(make_double2(fma(d1.x, x1.x, -d1.y * x1.y),
                                                 fma(d1.x, x1.y, d1.y * x1.x)));
        }
      }
      __syncthreads();
      continue;
    }
    const double2 ulo = U[k4 * 8 + q], uhi = U[(4 + k4) * 8 + q];
    double A[2][4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const double2 uu = (s & 1) ? uhi : ulo;
      A[0][s] = (s < 2) ? uu.x : -uu.y;   // real output row
      A[1][s] = (s < 2) ? uu.y : uu.x;    // imaginary output row
    }
    const uint32_t in0 = (uint32_t)T[4 + q] ^ T[12 + k4];
    const uint32_t in1 = (uint32_t)T[4 + q] ^ T[12 + 4 + k4];
    const uint32_t out0 = (uint32_t)T[4 + 2 * k4] ^ T[12 + q];
    const uint32_t out1 = (uint32_t)T[4 + 2 * k4 + 1] ^ T[12 + q];
    for (uint32_t c = warp; c < nchunks; c += nwarps) {
      uint32_t cb = 0;
      for (uint32_t cc = c, k = 0; cc; cc >>= 1, ++k)
        if (cc & 1u) cb ^= T[20 + k];
      double B[4][4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const uint32_t tb = cb ^ T[t];
        const double2 x0 = to_d2(t0[tb ^ in0]), x1 = to_d2(t0[tb ^ in1]);
        B[t][0] = x0.x;  // real part of amplitude k4
        B[t][1] = x1.x;  // real part of amplitude 4 + k4
        B[t][2] = x0.y;
        B[t][3] = x1.y;
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        double re0 = 0.0, re1 = 0.0, im0 = 0.0, im1 = 0.0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          dmma_m8n8k4(re0, re1, A[0][s], B[t][s], re0, re1);
          dmma_m8n8k4(im0, im1, A[1][s], B[t][s], im0, im1);
        }
        const uint32_t tb = cb ^ T[t];
        t0[tb ^ out0] = from_d2<V>(make_double2(re0, im0));
        t0[tb ^ out1] = from_d2<V>(make_double2(re1, im1));
      }
    }
    __syncthreads();
  }
  if (a.tma.use) {
    if (a.tma.relayout) tma::relayout_rows(t0, (size * sizeof(V)) >> 7, a.tma.swz);  // back
    tma::tile_store<1>(a.tma, &tm0, &tm0, t0, nullptr, base);
  } else
    store_tile<V, 1>(v0, nullptr, t0, nullptr, a.ta, base, a.vec16);
}

// complex<float> passes of three tile bits on the TF32 tensor cores with the
// three-term split: each operand x = hi + lo (hi = tf32(x), lo = tf32(x - hi))
// and D += A_lo B_hi + A_hi B_lo + A_hi B_hi in FP32 (the lo*lo term, ~2^-22
// relative, is dropped), mma.sync m16n8k8 tf32: 24 MMAs per chunk of 32
// groups x 8 amplitudes.  Fragment lanes as in k_dmma3 (g = lane / 4 is the
// column group and output amplitude, t = lane % 4 the input amplitudes t and
// t + 4), so the same address tables serve.
__device__ __forceinline__ uint32_t tf32_of(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = tf32_of(x);
  lo = tf32_of(x - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
      "{%8, %9}, {%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__global__ void __launch_bounds__(256, 2) k_tf32x3(float2* __restrict__ v0, DmmaArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t size = 1u << a.ta.m;
  float2* t0 = reinterpret_cast<float2*>(smem_raw);
  const PassDev* passes;
  const POp* ops;
  const double2* coefs;
  stage_plan<double2>(smem_raw + size_t(size) * sizeof(float2), a.passes, a.npasses, a.ops,
                      a.nops, a.coefs, a.ncoef, &passes, &ops, &coefs);
  const uint64_t base = tile_base(a.ta, blockIdx.x);
  load_tile<float2, 1>(v0, nullptr, t0, nullptr, a.ta, base, a.vec16);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const uint32_t nchunks = size >> 8;  // 32 groups x 8 amplitudes
  for (int pi = 0; pi < a.npasses; ++pi) {
    const PassDev& P = passes[pi];
    const uint16_t* T = P.off;
    const double2* U = coefs + ops[P.op0].coef;  // U[i][k] at k * 8 + i
    const double2 u0 = U[t * 8 + g], u4 = U[(t + 4) * 8 + g];
    // A fragments of k-step s: rows g (real out) and g + 8 (imaginary out),
    // columns t and t + 4 of the real (s = 0) or imaginary (s = 1) inputs
    float av[2][4];
    av[0][0] = (float)u0.x;  av[0][1] = (float)u0.y;  av[0][2] = (float)u4.x;  av[0][3] = (float)u4.y;
    av[1][0] = (float)-u0.y; av[1][1] = (float)u0.x;  av[1][2] = (float)-u4.y; av[1][3] = (float)u4.x;
    uint32_t ahi[2][4], alo[2][4];
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
      for (int j = 0; j < 4; ++j) split_tf32(av[s][j], ahi[s][j], alo[s][j]);
    const uint32_t in0 = (uint32_t)T[4 + g] ^ T[12 + t];
    const uint32_t in1 = (uint32_t)T[4 + g] ^ T[12 + 4 + t];
    const uint32_t out0 = (uint32_t)T[4 + 2 * t] ^ T[12 + g];
    const uint32_t out1 = (uint32_t)T[4 + 2 * t + 1] ^ T[12 + g];
    for (uint32_t c = warp; c < nchunks; c += nwarps) {
      uint32_t cb = 0;
      for (uint32_t cc = c, k = 0; cc; cc >>= 1, ++k)
        if (cc & 1u) cb ^= T[20 + k];
      float2 x0[4], x1[4];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const uint32_t tb = cb ^ T[nt];
        x0[nt] = t0[tb ^ in0];  // amplitude t of column group g
        x1[nt] = t0[tb ^ in1];  // amplitude t + 4
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        float d[4] = {0.f, 0.f, 0.f, 0.f};
        // k-step 0: real inputs, k-step 1: imaginary inputs
        const float bv[2][2] = {{x0[nt].x, x1[nt].x}, {x0[nt].y, x1[nt].y}};
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          uint32_t bh0, bl0, bh1, bl1;
          split_tf32(bv[s][0], bh0, bl0);
          split_tf32(bv[s][1], bh1, bl1);
          mma_tf32(d, alo[s], bh0, bh1);
          mma_tf32(d, ahi[s], bl0, bl1);
          mma_tf32(d, ahi[s], bh0, bh1);
        }
        // d0, d1: real parts of amplitude g for groups 2t, 2t + 1; d2, d3: imaginary
        const uint32_t tb = cb ^ T[nt];
        t0[tb ^ out0] = make_float2(d[0], d[2]);
        t0[tb ^ out1] = make_float2(d[1], d[3]);
      }
    }
    __syncthreads();
  }
  store_tile<float2, 1>(v0, nullptr, t0, nullptr, a.ta, base, a.vec16);
}

// ---- complex<float> passes on tcgen05 (kind::tf32), state rows in TMEM -----
// A pass on three tile bits applies one 8x8 complex U to every group of 8
// amplitudes.  As a GEMM, D[g][n] = sum_k X[g][k] W[k][n] with X[g] the row
// (Re x_0..7, Im x_0..7) of group g and the real 16x16 W
//   W[j][i] = Re U[i][j], W[8+j][i] = -Im U[i][j],
//   W[j][8+i] = Im U[i][j], W[8+j][8+i] = Re U[i][j].
// 128 groups form one M = 128 tile.  Each thread gathers its group from the
// shared-memory state tile, splits the row into X_hi + X_lo (tc::tf32_split)
// and stores the two halves to tensor memory; one thread per warpgroup then
// issues
//   D[:, 0:32]  = X_hi [W_hi | W_lo]     (N = 32, two K-steps of 8)
//   D[:, 0:16] += X_lo W_hi              (N = 16, two K-steps)
// and the output row is D[:, n] + D[:, 16 + n] (the X_lo W_lo term, about
// 2^-22 relative, is dropped).  An MMA costs about the same for N = 16 and
// N = 32 (12.9 and 13.0 ns per SM in a probe), so the W_lo product rides in
// the upper half of the first pair.  Each warpgroup alternates two
// tensor-memory slots (A_hi 16 | A_lo 16 | D 32 columns).  Per slot, one
// mbarrier counts the 128 threads' stores of A (only the issuing thread
// waits on it) and one receives the MMAs' commit; so a warp gathers the next
// M tile while the tensor cores work on the previous one.  W, as tf32 hi/lo
// halves, sits in shared memory in the K-major no-swizzle layout (8-row x
// 16-byte core matrices; 512 bytes between K chunks, 128 bytes between
// 8-row groups of N), double-buffered across passes; each thread builds one
// entry per pass from a U element it loaded a pass earlier.
constexpr uint32_t kTcCols = 256;        // tensor-memory columns per CTA
constexpr int kTcWaitLimit = 2000;       // suspended polls (up to 1 ms each)
constexpr size_t kTcMinSmem = 80 * 1024; // at most two CTAs (2 x 256 columns) per SM
__device__ unsigned g_tc_status;         // non-zero: a tensor-core wait gave up

// Entry e = threadIdx.x (k = e / 16, n = e % 16) of W: hi at column n, lo
// at 16 + n, from u = U[n % 8][k % 8].
__device__ __forceinline__ void tc_w_entry(float* img, double2 u) {
  const int e = threadIdx.x, k = e >> 4, n = e & 15;
  const double w = ((k < 8) == (n < 8)) ? u.x : (k < 8 ? u.y : -u.y);
  const float hi = __uint_as_float(tc::tf32_round((float)w));
  const float lo = __uint_as_float(tc::tf32_round((float)(w - (double)hi)));
  const int kb = (k >> 2) * 128 + (k & 3) + (n & 7) * 4;
  img[kb + (n >> 3) * 32] = hi;
  img[kb + ((n + 16) >> 3) * 32] = lo;
}
__device__ __forceinline__ int tc_u_index() {  // U[i][j] at j * 8 + i
  return ((threadIdx.x >> 4) & 7) * 8 + (threadIdx.x & 7);
}

__global__ void __launch_bounds__(256, 2) k_tc32(float2* __restrict__ v0, DmmaArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t size = 1u << a.ta.m;  // 2^10 .. 2^13 amplitudes
  float2* t0 = reinterpret_cast<float2*>(smem_raw);
  float* wimg = reinterpret_cast<float*>(smem_raw + size_t(size) * sizeof(float2));  // 2 x 2 KB
  // bars[wg * 2 + s]: MMAs of slot s done; bars[4 + wg * 2 + s]: A of slot s stored
  uint64_t* bars = reinterpret_cast<uint64_t*>(wimg + 1024);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 8);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
  unsigned char* plan = reinterpret_cast<unsigned char*>(bars) + 128;
  const PassDev* passes;
  const POp* ops;
  const double2* coefs_unused;
  // tables and ops in shared memory; W is built from U in global memory
  stage_plan<double2>(plan, a.passes, a.npasses, a.ops, a.nops, a.coefs, 0, &passes, &ops,
                      &coefs_unused);
  const int tid = threadIdx.x, warp = tid >> 5, wg = tid >> 7, r = tid & 127;
  if (tid == 0) {
    for (int b = 0; b < 4; ++b) tc::bar_init(bars + b, 1);
    for (int b = 4; b < 8; ++b) tc::bar_init(bars + b, 128);
    tc::bar_init_fence();
    *abort_flag = 0;
  }
  if (warp == 0) tc::alloc(tslot, kTcCols);
  const uint64_t base = tile_base(a.ta, blockIdx.x);
  load_tile<float2, 1>(v0, nullptr, t0, nullptr, a.ta, base, a.vec16);
  const int uix = tc_u_index();
  double2 unext = make_double2(0.0, 0.0);
  if (a.npasses > 0) tc_w_entry(wimg, a.coefs[a.ops[a.passes[0].op0].coef + uix]);
  if (a.npasses > 1) unext = a.coefs[a.ops[a.passes[1].op0].coef + uix];
  tc::fence_proxy_async();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tbase = *tslot;
  const uint32_t lane_off = (uint32_t)((warp & 3) * 32) << 16;
  const uint32_t nm = size >> 10;           // M tiles of 128 groups
  const uint32_t jn = (nm + 1 - wg) / 2;    // this warpgroup's: i = 2 j + wg < nm
  const uint32_t id32 = tc::idesc_tf32(128, 32), id16 = tc::idesc_tf32(128, 16);
  uint64_t* done = bars + wg * 2;
  uint64_t* stored = bars + 4 + wg * 2;
  uint32_t uses = 0;  // bit s: parity of the next completion of slot s's barriers
  for (int pi = 0; pi < a.npasses; ++pi) {
    const uint16_t* T = passes[pi].off;
    if (pi + 1 < a.npasses) tc_w_entry(wimg + ((pi + 1) & 1) * 512, unext);
    if (pi + 2 < a.npasses) unext = a.coefs[ops[passes[pi + 2].op0].coef + uix];
    const uint32_t wsm = tc::smem_addr(wimg + (pi & 1) * 512);
    uint32_t ao[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) ao[j] = T[j];
    uint32_t gr = 0;
#pragma unroll
    for (int b = 0; b < 7; ++b)
      if ((r >> b) & 1) gr ^= T[8 + b];
    uint32_t prev = 0;
    for (uint32_t j = 0; j <= jn; ++j) {
      uint32_t gb = 0;
      if (j < jn) {
        const uint32_t s = j & 1, i = 2 * j + wg;
        gb = gr;
        for (int b = 0; (i >> b) != 0u; ++b)
          if ((i >> b) & 1u) gb ^= T[15 + b];
        const uint32_t col = wg * 128 + s * 64;
        uint32_t hi[16], lo[16];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float2 x = t0[gb ^ ao[k]];
          tc::tf32_split(x.x, hi[k], lo[k]);
          tc::tf32_split(x.y, hi[8 + k], lo[8 + k]);
        }
        tc::st_32x32b_x16(tbase + lane_off + col, hi);
        tc::st_32x32b_x16(tbase + lane_off + col + 16, lo);
        tc::wait_st();
        tc::fence_before();
        tc::bar_arrive(stored + s);
        if (r == 0) {
          if (tc::bar_wait(stored + s, (uses >> s) & 1u, abort_flag, kTcWaitLimit)) {
            tc::fence_after();
            const uint32_t ta = tbase + col, td = tbase + col + 32;
            const uint64_t b0 = tc::sdesc_kmajor(wsm, 512, 128);
            const uint64_t b1 = tc::sdesc_kmajor(wsm + 1024, 512, 128);
            tc::mma_tf32_ts(td, ta, b0, id32, 0);
            tc::mma_tf32_ts(td, ta + 8, b1, id32, 1);
            tc::mma_tf32_ts(td, ta + 16, b0, id16, 1);
            tc::mma_tf32_ts(td, ta + 24, b1, id16, 1);
            tc::commit(done + s);
          } else {
            *abort_flag = 1;
            atomicOr(&g_tc_status, 1u);
          }
        }
      }
      if (j > 0) {  // finish M tile j - 1: wait for its MMAs, read D, scatter
        const uint32_t s = (j - 1) & 1;
        if (!tc::bar_wait(done + s, (uses >> s) & 1u, abort_flag, kTcWaitLimit)) {
          *abort_flag = 1;
          atomicOr(&g_tc_status, 1u);
        }
        uses ^= 1u << s;
        __syncwarp();
        tc::fence_after();
        float d[32];
        tc::ld_32x32b_x32(tbase + lane_off + wg * 128 + s * 64 + 32, d);
#pragma unroll
        for (int k = 0; k < 8; ++k)
          t0[prev ^ ao[k]] = make_float2(d[k] + d[16 + k], d[8 + k] + d[24 + k]);
      }
      prev = gb;
    }
    tc::fence_proxy_async();  // the next pass's W
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
  }
  store_tile<float2, 1>(v0, nullptr, t0, nullptr, a.ta, base, a.vec16);
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::dealloc(tbase, kTcCols);
}

// Rank over GF(2) of up to four 4-bit vectors.
int gf2_rank(std::initializer_list<uint32_t> in) {
  uint32_t v[4];
  int k = 0;
  for (uint32_t x : in) v[k++] = x;
  int r = 0;
  for (int bit = 3; bit >= 0; --bit) {
    int piv = -1;
    for (int i = r; i < k; ++i)
      if ((v[i] >> bit) & 1u) { piv = i; break; }
    if (piv < 0) continue;
    std::swap(v[r], v[piv]);
    for (int i = 0; i < k; ++i)
      if (i != r && ((v[i] >> bit) & 1u)) v[i] ^= v[r];
    ++r;
  }
  return r;
}

// Address tables of one tensor-core pass on R = 2 or 3 tile bits p0 < p1
// (< p2) of an m-bit tile (epu elements per 16-byte unit), in PassDev.off:
//   off[t]          t < 4     group part of column tile t   (group bits 3, 4)
//   off[4 + g]      g < 8     group part of column g         (group bits 0..2)
//   off[12 + j]     j < 2^R   amplitude part of amplitude j  (pass bits)
//   off[12+2^R + k] k         chunk part of chunk bit k      (group bits 5..)
// all as swizzled shared-memory element offsets (phys is linear, so the
// address of (chunk, tile, column, amplitude) is the XOR of its parts).
// Group index bits map to the tile's other bits; the three lowest are chosen
// so that the shared-memory banks a quarter-warp (16-byte elements) or
// half-warp (8-byte elements) touches on load and on store are independent
// of the banks of the pass bits p0, p1 that vary within it.
// swz < 0: the cp.async layout (phys_host); swz >= 0: a TMA-staged tile
// whose swizzle has XOR width swz (phys_tma_host).
void dmma_tables_compute(PassDev* P, int R, int m, int epu, int swz);

// The tables depend only on (pass bits, tile bits, element size, layout);
// passes of a circuit repeat a few patterns, so they are cached per host
// thread.
void dmma_tables(PassDev* P, int R, int m, int epu, int swz) {
  thread_local std::unordered_map<uint64_t, std::array<uint16_t, 32>> cache;
  const uint64_t key = (uint64_t)(uint8_t)P->pos[0] | ((uint64_t)(uint8_t)P->pos[1] << 8) |
                       ((uint64_t)(uint8_t)(R == 3 ? P->pos[2] : 0xff) << 16) |
                       ((uint64_t)m << 24) | ((uint64_t)epu << 32) | ((uint64_t)R << 40) |
                       ((uint64_t)(swz + 1) << 44);
  auto it = cache.find(key);
  if (it == cache.end()) {
    if (cache.size() > 4096) cache.clear();
    PassDev tmp = *P;
    dmma_tables_compute(&tmp, R, m, epu, swz);
    std::array<uint16_t, 32> t;
    std::memcpy(t.data(), tmp.off, sizeof(tmp.off));
    it = cache.emplace(key, t).first;
  }
  std::memcpy(P->off, it->second.data(), sizeof(P->off));
}

void dmma_tables_compute(PassDev* P, int R, int m, int epu, int swz) {
  const int nb = R;
  int pos[3] = {P->pos[0], P->pos[1], R == 3 ? P->pos[2] : -1};
  const uint32_t bank_mask = epu == 1 ? 7u : 15u;
  auto phys = [&](uint32_t e) {
    return swz < 0 ? phys_host(e, (uint32_t)epu) : phys_tma_host(e, (uint32_t)epu, swz);
  };
  auto dir = [&](int b) { return phys(1u << b) & bank_mask; };
  std::vector<int> rest;
  for (int b = 0; b < m; ++b)
    if (b != pos[0] && b != pos[1] && b != pos[2]) rest.push_back(b);
  const uint32_t u = dir(pos[0]), v = dir(pos[1]);
  const int top = epu == 1 ? 6 : 8;
  int best = -1, s0 = rest[0], s1 = rest[1], s2 = rest[2];
  for (size_t i0 = 0; i0 < rest.size() && best < top; ++i0)
    for (size_t i1 = 0; i1 < rest.size() && best < top; ++i1)
      for (size_t i2 = 0; i2 < rest.size() && best < top; ++i2) {
        const int b0 = rest[i0], b1 = rest[i1], b2 = rest[i2];
        if (b0 == b1 || b0 == b2 || b1 == b2) continue;
        const int score = epu == 1
            ? gf2_rank({dir(b0), u, v}) + gf2_rank({u, dir(b1), dir(b2)})
            : gf2_rank({dir(b0), dir(b1), u, v}) + gf2_rank({u, v, dir(b1), dir(b2)});
        if (score > best) { best = score; s0 = b0; s1 = b1; s2 = b2; }
      }
  std::vector<int> sel = {s0, s1, s2};
  for (int b : rest)
    if (b != s0 && b != s1 && b != s2) sel.push_back(b);
  auto map = [&](uint32_t g) {
    uint32_t e = 0;
    for (size_t i = 0; i < sel.size(); ++i)
      if ((g >> i) & 1u) e |= 1u << sel[i];
    return e;
  };
  auto ph = [&](uint32_t e) { return (uint16_t)phys(e); };
  for (int t = 0; t < 4; ++t) P->off[t] = ph(map(8u * t));
  for (int g = 0; g < 8; ++g) P->off[4 + g] = ph(map((uint32_t)g));
  const int na = 1 << nb;
  for (int j = 0; j < na; ++j) {
    uint32_t e = 0;
    for (int k = 0; k < nb; ++k)
      if ((j >> k) & 1) e |= 1u << pos[k];
    P->off[12 + j] = ph(e);
  }
  for (int k = 0; k + 5 + nb < m && 12 + na + k < 32; ++k) P->off[12 + na + k] = ph(map(32u << k));
}

// Address tables of one tcgen05 pass (k_tc32) on tile bits p0 < p1 < p2 of
// an m-bit complex<float> tile, in PassDev.off:
//   off[j]      j < 8       amplitude part of amplitude j (pass bits)
//   off[8 + k]  k < m - 3   group part of group bit k
// Group bits 0..6 are the row of the M = 128 tile (bits 0..4 the lane), the
// rest the M tile.  The four lowest are chosen, where the pass bits allow,
// so that the banks a half-warp touches (8-byte elements: element index mod
// 16) are all different.
void tc_tables(PassDev* P, int m) {
  const int pos[3] = {P->pos[0], P->pos[1], P->pos[2]};
  std::vector<int> rest, sel;
  for (int b = 0; b < m; ++b)
    if (b != pos[0] && b != pos[1] && b != pos[2]) rest.push_back(b);
  uint32_t basis[4] = {0, 0, 0, 0};  // reduced bank directions, by leading bit
  auto independent_add = [&](uint32_t v) {
    for (int bit = 3; bit >= 0; --bit) {
      if (!((v >> bit) & 1u)) continue;
      if (!basis[bit]) { basis[bit] = v; return true; }
      v ^= basis[bit];
    }
    return false;
  };
  std::vector<bool> used(rest.size(), false);
  for (size_t i = 0; i < rest.size() && sel.size() < 4; ++i)
    if (independent_add((uint32_t)phys_host(1u << rest[i], 2) & 15u)) {
      sel.push_back(rest[i]);
      used[i] = true;
    }
  for (size_t i = 0; i < rest.size(); ++i)
    if (!used[i]) sel.push_back(rest[i]);
  for (int j = 0; j < 8; ++j) {
    uint32_t e = 0;
    for (int k = 0; k < 3; ++k)
      if ((j >> k) & 1) e |= 1u << pos[k];
    P->off[j] = (uint16_t)phys_host(e, 2);
  }
  for (int k = 0; k < m - 3; ++k) P->off[8 + k] = (uint16_t)phys_host(1u << sel[k], 2);
}

constexpr size_t kDmmaPlanMax = 96 * 1024;  // a tensor-core stage's plan bytes, at most

// Tile bits of the tensor-core engine for an n-qubit complex sweep, or -1
// when it does not apply (real elements, engine 1, tiles under 2^(5+R)).
// Its tiles have no per-thread register limit: the requested or default
// size, at most 14 bits, n and the shared memory.
template <typename V>
int dmma_tile_bits(int n, const qsv_fuse_opts* opts) {
  if (!Elem<V>::cplx || (opts && opts->engine == 1)) return -1;
  int md = (opts && opts->tile_bits > 0) ? opts->tile_bits : default_tile_bits(sizeof(V), 1);
  md = std::min(std::min(md, 14), n);
  while (md > 7 && (size_t(1) << md) * sizeof(V) + kDmmaPlanMax > 200 * 1024) --md;
  return md >= 7 ? md : -1;
}

// The gate engine runs when asked for (engine 5), and by default for
// complex<float> single-vector sweeps (measured on a B200: 32-qubit brick of
// depth 100 in 7.0 s against 8.4 s on the FP64 tensor cores, with
// 1 - |<psi32|psi64>|^2 = 1.6e-7 against 1.2e-7); complex<double> sweeps
// default to the FP64 tensor-core passes (28-qubit brick: 220 ms against
// 288 ms on the gate engine).
template <typename V>
bool use_gate_engine(const qsv_fuse_opts* opts) {
  if (opts && opts->engine == 5) return true;
  return sizeof(V) == 8 && Elem<V>::cplx && (!opts || opts->engine == 0);
}

// Tile bits of the gate engine: the requested (or default) size, at most 14
// and n, with the tile and a plan in shared memory; -1 if too small.
template <typename V>
int gate_tile_bits(int n, const qsv_fuse_opts* opts) {
  int m = (opts && opts->tile_bits > 0) ? opts->tile_bits : default_tile_bits(sizeof(V), 1);
  m = std::min(std::min(m, 14), n);
  while (m > 1 && (size_t(1) << m) * sizeof(V) + 16384 > 200 * 1024) --m;
  return m >= gate_pass_bits(sizeof(V), opts) + 1 ? m : -1;
}

int dmma_pass_bits(int m) { return (QSV_DMMA_BITS == 3 && m >= 8) ? 3 : 2; }

// The tensor-core engine's plan.  A dense pass costs the same whatever it
// holds, and the pass count depends strongly on which low bits every tile
// keeps (brick circuits: 1982 passes with 2 low bits, 1782 with 3, for 30
// qubits and 12 tile bits).  So when the caller leaves low_bits unset, the
// default and more contiguous low bits are planned (in parallel host
// threads) and the plan with the least passes + kappa * stages is kept: a
// stage's tile load and store cost about one pass for 16-byte amplitudes
// and a quarter of one for 8-byte amplitudes (fitted from 29-qubit brick
// sweeps on a B200: complex<double> 862 passes/154 stages 1100 ms against
// 837/193 1121 ms; complex<float> 853/150 962 ms against 826/182 940 ms).
// States of fewer than 27 qubits, or of a single tile, keep the default.
qsv_status pack_dense_plan(const std::vector<Lowered>& items, int n, int m, int low,
                           bool low_fixed, int R, int max_gates, size_t elem_bytes,
                           PackedPlan<double2>* plan, int* low_used) {
  // The low-bit candidates only where they can pay: an extra plan costs a
  // few ms of host time for a thousand gates, which ~10 % fewer passes win
  // back only from about 2^27 amplitudes on (a 26-qubit pass takes ~0.14 ms);
  // with one tile every low-bit choice gives the same plan.  (The rollout
  // choice of pass bits pays at every size: an adjoint loop over 8..18-qubit
  // circuits ran 14.5 s with it, 16.5 s without.)
  const bool search = QSV_DENSE_SEARCH != 0;
  std::vector<int> lows = {low};
  if (!low_fixed && QSV_DENSE_LOW_SEARCH && n > m && n >= 27) {
    const int extra = elem_bytes >= 16 ? 1 : 3;
    for (int d = 1; d <= extra && low + d < m; ++d) lows.push_back(low + d);
  }
  std::vector<PackedPlan<double2>> plans(lows.size());
  std::vector<qsv_status> status(lows.size(), QSV_SUCCESS);
  std::vector<std::thread> workers;
  for (size_t i = 1; i < lows.size(); ++i)
    workers.emplace_back([&, i] {
      status[i] = pack_plan<double2>(items, n, m, lows[i], R, max_gates, &plans[i], 1,
                                     kDmmaPlanMax, search);
    });
  status[0] = pack_plan<double2>(items, n, m, lows[0], R, max_gates, &plans[0], 1, kDmmaPlanMax,
                                 search);
  for (std::thread& t : workers) t.join();
  if (status[0] != QSV_SUCCESS) return status[0];
  const double kappa = elem_bytes >= 16 ? 1.0 : 0.25;
  size_t best = 0;
  double best_cost = 0.0;
  for (size_t i = 0; i < lows.size(); ++i) {
    if (status[i] != QSV_SUCCESS) continue;
    const double cost = (double)plans[i].passes.size() + kappa * (double)plans[i].stages.size();
    if (i == 0 || cost < best_cost) { best = i; best_cost = cost; }
  }
  *plan = std::move(plans[best]);
  *low_used = lows[best];
  return QSV_SUCCESS;
}

// Single-vector sweep of a complex state on the tensor-core engine; returns
// QSV_ERROR_NOT_SUPPORTED (nothing launched) when the plan does not fit it.
template <typename V>
qsv_status execute_dmma(const ExecArgs& x, int m, int low, int max_gates, bool vec16) {
  qsv_state_s* s = x.s;
  const int n = s->n;
  const int R = dmma_pass_bits(m);
  PackedPlan<double2> plan;
  // plans sized per launch: a few KB typically, at most kDmmaPlanMax
  // (+ 1024: k_dmma3 aligns its tile to 1024 bytes)
  if ((size_t(1) << m) * sizeof(V) + kDmmaPlanMax + 1024 > 200 * 1024)
    return QSV_ERROR_NOT_SUPPORTED;
  const bool low_fixed = x.opts && x.opts->low_bits > 0;
  if (qsv_status st = pack_dense_plan(*x.items, n, m, low, low_fixed, R, max_gates, sizeof(V), &plan,
                                      &low))
    return st;
  if (plan.stages.empty()) return QSV_SUCCESS;
  // complex<float> three-bit passes run on FP64 MMA like complex<double>
  // (rounded to nearest once per pass, so the norm does not drift); TF32
  // with the three-term split is opt-in: on tcgen05 with the state rows in
  // tensor memory (engine 3, tiles of 2^10 .. 2^13 amplitudes) or on
  // mma.sync (engine 4, and engine 3 for smaller tiles).  Its FP32
  // accumulation truncates, which shrinks the norm by ~1e-7 per pass.
  const int engine = x.opts ? x.opts->engine : 0;
  const bool f32 = std::is_same<V, float2>::value && R == 3;
  const bool tcg = f32 && engine == 3 && m >= 10 && m <= 13;
  const bool tf32 = f32 && (engine == 4 || engine == 3);
  // k_dmma3 tiles move by TMA where the stage's tile fits a tensor map
  // (qsv_fuse_opts.tile_copy = 1: cp.async)
  const bool dmma3 = !tcg && !tf32 && R == 3;
  const bool want_tma = dmma3 && !(x.opts && x.opts->tile_copy == 1);
  std::vector<CUtensorMap> maps(plan.stages.size());
  std::vector<TmaGeo> geos(plan.stages.size());
  for (size_t si = 0; si < plan.stages.size(); ++si) {
    geos[si] = TmaGeo{};
    const PackedStage& ps = plan.stages[si];
    if (want_tma && tma_stage_map(ps.bits, ps.m, n, sizeof(V), x.v0, &maps[si], &geos[si]))
      geos[si].relayout = 1;
  }
  for (size_t si = 0; si < plan.stages.size(); ++si) {
    const PackedStage& ps = plan.stages[si];
    for (size_t pi = ps.pass0; pi < ps.pass0 + ps.npasses; ++pi) {
      PassDev& P = plan.passes[pi];
      if (P.nops != 1 || plan.ops[ps.op0 + P.op0].shape != P_DENSE || ps.m < 5 + R ||
          (tcg && ps.m < 10))
        return QSV_ERROR_NOT_SUPPORTED;
      if (tcg)
        tc_tables(&P, ps.m);
      else  // k_dmma3 converts TMA-staged tiles to the cp.async layout (relayout_rows)
        dmma_tables(&P, R, ps.m, Units<V>::per, -1);
    }
  }
  unsigned* wait_error = sweep_wait_flag();
  if (dmma3 && !wait_error) return fail(QSV_ERROR_CUDA, "sweep wait flag unavailable");
  auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
  const size_t pass_bytes = plan.passes.size() * sizeof(PassDev);
  const size_t op_off = align(pass_bytes);
  const size_t coef_off = align(op_off + plan.ops.size() * sizeof(POp));
  const size_t run_off = align(coef_off + plan.coefs.size() * sizeof(double2));
  const size_t total = run_off + plan.runoff.size() * sizeof(uint64_t);
  std::vector<unsigned char> host(total);
  std::memcpy(host.data(), plan.passes.data(), pass_bytes);
  std::memcpy(host.data() + op_off, plan.ops.data(), plan.ops.size() * sizeof(POp));
  std::memcpy(host.data() + coef_off, plan.coefs.data(), plan.coefs.size() * sizeof(double2));
  std::memcpy(host.data() + run_off, plan.runoff.data(), plan.runoff.size() * sizeof(uint64_t));
  if (qsv_status st = ensure_scratch(s, total)) return st;
  unsigned char* dev = static_cast<unsigned char*>(s->scratch);
  if (qsv_status st = cuda_status(cudaMemcpyAsync(dev, host.data(), total, cudaMemcpyHostToDevice,
                                                  s->stream), "dense plan upload"))
    return st;
  void* kern = tcg ? (void*)k_tc32
                   : (tf32 ? (void*)k_tf32x3 : (R == 3 ? (void*)k_dmma3<V> : (void*)k_dmma<V>));
  if (tcg) g_tc_used = true;
  if (qsv_status st = cuda_status(cudaFuncSetAttribute(kern,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       200 * 1024), "dense stage shared-memory attribute"))
    return st;
  const uint64_t ntiles = 1ull << (n - m);
  if (x.ntiles_out) *x.ntiles_out = ntiles;
  const bool profile = x.opts && x.opts->profile;
  std::vector<cudaEvent_t> ev;
  if (profile) {
    ev.resize(plan.stages.size() + 1);
    for (auto& e : ev)
      if (qsv_status st = cuda_status(cudaEventCreate(&e), "cudaEventCreate")) return st;
    cudaEventRecord(ev[0], s->stream);
  }
  V* p0 = static_cast<V*>(x.v0);
  for (size_t si = 0; si < plan.stages.size(); ++si) {
    const PackedStage& ps = plan.stages[si];
    DmmaArgs a;
    a.ta.n = n;
    a.ta.m = ps.m;
    a.ta.low = low;
    for (int j = 0; j < 64; ++j) a.ta.bits[j] = (int8_t)ps.bits[j];
    a.ta.runoff = reinterpret_cast<const uint64_t*>(dev + run_off) + ps.run0;
    a.npasses = (int)ps.npasses;
    a.nops = ps.nops;
    a.ncoef = ps.ncoef;
    a.passes = reinterpret_cast<const PassDev*>(dev) + ps.pass0;
    a.ops = reinterpret_cast<const POp*>(dev + op_off) + ps.op0;
    a.coefs = reinterpret_cast<const double2*>(dev + coef_off) + ps.coef0;
    a.vec16 = vec16 ? 1 : 0;
    a.tma = geos[si];
    a.wait_error = wait_error;
    // k_dmma3: + 1024 for its tile's 1024-byte alignment
    const size_t smem_stage =
        tcg ? std::max(kTcMinSmem, (size_t(1) << ps.m) * sizeof(V) + 4096 + 128 +
                                       plan_smem_bytes<double2>((int)ps.npasses, ps.nops, 0))
            : (size_t(1) << ps.m) * sizeof(V) +
                  plan_smem_bytes<double2>((int)ps.npasses, ps.nops, ps.ncoef) +
                  (dmma3 ? 1024 : 0);
    a.smem_bytes = (uint32_t)smem_stage;
    void* args2[] = {&p0, &a};
    void* args3[] = {&p0, &a, &maps[si]};
    void** args = dmma3 ? args3 : args2;
    if (qsv_status st = cuda_status(cudaLaunchKernel(kern, dim3((unsigned)ntiles),
                                                     dim3(256), args, smem_stage, s->stream),
                                    "dense stage launch"))
      return st;
    count_launch();
    if (a.tma.use) count_tma_launch();
    if (profile) cudaEventRecord(ev[si + 1], s->stream);
  }
  if (profile) {
    qsv_status st = cuda_status(cudaEventSynchronize(ev.back()), "stage timing synchronize");
    g_stage_ms.clear();
    for (size_t si = 0; si < plan.stages.size() && !st; ++si) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[si], ev[si + 1]);
      g_stage_ms.push_back(ms);
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (st) return st;
  }
  return QSV_SUCCESS;
}

template <typename V>
qsv_status execute_typed(const ExecArgs& x) {
  constexpr int EPU = Units<V>::per;
  qsv_state_s* s = x.s;
  const int n = s->n;
  const qsv_fuse_opts* opts = x.opts;
  const int m = effective_tile_bits(sizeof(V), x.nv, n, opts);
  int low = (opts && opts->low_bits > 0) ? opts->low_bits : default_low_bits(sizeof(V));
  const int max_gates = (opts && opts->max_stage_gates > 0) ? opts->max_stage_gates : 256;
  const int r = pass_bits(sizeof(V), x.nv, m);
  if (low > m) low = m;
  const size_t smem_fixed = (size_t(1) << m) * sizeof(V) * x.nv + (x.nv == 2 ? kRaccBytes : 0);
  const size_t smem = smem_fixed + kPlanSmemMax;  // bound; each launch asks for its own size
  if (smem > 200 * 1024)
    return fail(QSV_ERROR_SIZE, "tile of %d x 2^%d elements exceeds shared memory", x.nv, m);
  // 16-byte copies need 16-byte aligned vectors and runs of >= 16 bytes
  int log_epu = 0;
  while ((1 << log_epu) < EPU) ++log_epu;
  const bool vec16 = (low >= log_epu) && (m >= log_epu) &&
                     (reinterpret_cast<uintptr_t>(x.v0) % 16 == 0) &&
                     (x.nv == 1 || reinterpret_cast<uintptr_t>(x.v1) % 16 == 0);

  // complex single-vector sweeps: the gate engine when selected, else the
  // tensor-core engine unless the caller asks for sparse passes; tiles need
  // at least one 128-amplitude chunk
  if constexpr (Elem<V>::cplx) {
    if (x.nv == 1 && x.nslots == 0 && use_gate_engine<V>(opts)) {
      const int mg = gate_tile_bits<V>(n, opts);
      const int lowg = (opts && opts->low_bits > 0) ? low : gate_default_low(sizeof(V));
      if (mg > 0) {
        const qsv_status st = execute_gates<V>(x, mg, std::min(lowg, mg), max_gates, vec16);
        if (st != QSV_ERROR_NOT_SUPPORTED) return st;
      }
    }
    // two-vector (adjoint) sweeps: the gate engine unless the sparse passes
    // are asked for (engine 1), with the tiles the caller sized its partial
    // sums for (fused_tiles)
    if (x.nv == 2 && (!opts || opts->engine != 1)) {
      const qsv_status st = execute_gates<V>(x, m, low, max_gates, vec16);
      if (st != QSV_ERROR_NOT_SUPPORTED) return st;
    }
  }
  if (x.nv == 1 && x.nslots == 0) {
    const int md = dmma_tile_bits<V>(n, opts);
    if (md > 0) {
      const qsv_status st = execute_dmma<V>(x, md, std::min(low, md), max_gates, vec16);
      if (st != QSV_ERROR_NOT_SUPPORTED) return st;
    }
  }

  PackedPlan<V> plan;
  if (qsv_status st = pack_plan<V>(*x.items, n, m, low, r, max_gates, &plan)) return st;
  if (plan.stages.empty()) return QSV_SUCCESS;
  auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
  const size_t pass_bytes = plan.passes.size() * sizeof(PassDev);
  const size_t op_off = align(pass_bytes);
  const size_t coef_off = align(op_off + plan.ops.size() * sizeof(POp));
  const size_t run_off = align(coef_off + plan.coefs.size() * sizeof(V));
  const size_t red_off = align(run_off + plan.runoff.size() * sizeof(uint64_t));
  const size_t total = red_off + plan.red_slots.size() * sizeof(int32_t);
  std::vector<unsigned char> host(total);
  std::memcpy(host.data(), plan.passes.data(), pass_bytes);
  std::memcpy(host.data() + op_off, plan.ops.data(), plan.ops.size() * sizeof(POp));
  std::memcpy(host.data() + coef_off, plan.coefs.data(), plan.coefs.size() * sizeof(V));
  std::memcpy(host.data() + run_off, plan.runoff.data(), plan.runoff.size() * sizeof(uint64_t));
  if (!plan.red_slots.empty())
    std::memcpy(host.data() + red_off, plan.red_slots.data(), plan.red_slots.size() * sizeof(int32_t));
  if (qsv_status st = ensure_scratch(s, total)) return st;
  unsigned char* dev = static_cast<unsigned char*>(s->scratch);
  if (qsv_status st = cuda_status(cudaMemcpyAsync(dev, host.data(), total, cudaMemcpyHostToDevice,
                                                  s->stream), "fused plan upload"))
    return st;

  void* kerns[2] = {(x.nv == 2) ? pick_kernel<V, 2>(r, false) : pick_kernel<V, 1>(r, false),
                    (x.nv == 2) ? pick_kernel<V, 2>(r, true) : pick_kernel<V, 1>(r, true)};
  for (void* k : kerns)
    if (qsv_status st = cuda_status(
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024),
            "fused stage shared-memory attribute"))
      return st;
  const unsigned threads = 1u << std::min(m - r, 8);
  const uint64_t ntiles = 1ull << (n - m);
  if (x.ntiles_out) *x.ntiles_out = ntiles;
  if (x.nslots > 0 && x.partial_bytes < (size_t)x.nslots * ntiles * sizeof(double))
    return fail(QSV_ERROR_SIZE, "partial-sum buffer too small");
  const bool profile = opts && opts->profile;
  std::vector<cudaEvent_t> ev;
  if (profile) {
    ev.resize(plan.stages.size() + 1);
    for (auto& e : ev)
      if (qsv_status st = cuda_status(cudaEventCreate(&e), "cudaEventCreate")) return st;
    cudaEventRecord(ev[0], s->stream);
  }
  V* p0 = static_cast<V*>(x.v0);
  V* p1 = static_cast<V*>(x.v1);
  for (size_t si = 0; si < plan.stages.size(); ++si) {
    const PackedStage& ps = plan.stages[si];
    Stage2Args a;
    a.ta.n = n;
    a.ta.m = ps.m;
    a.ta.low = low;
    for (int j = 0; j < 64; ++j) a.ta.bits[j] = (int8_t)ps.bits[j];
    a.ta.runoff = reinterpret_cast<const uint64_t*>(dev + run_off) + ps.run0;
    a.npasses = (int)ps.npasses;
    a.passes = reinterpret_cast<const PassDev*>(dev) + ps.pass0;
    a.ops = reinterpret_cast<const POp*>(dev + op_off) + ps.op0;
    a.coefs = dev + coef_off + ps.coef0 * sizeof(V);
    a.partial = x.partial;
    a.red_slots = reinterpret_cast<const int32_t*>(dev + red_off) + ps.red0;
    a.nred = ps.nred;
    a.nops = ps.nops;
    a.ncoef = ps.ncoef;
    const size_t smem_stage = smem_fixed + plan_smem_bytes<V>((int)ps.npasses, ps.nops, ps.ncoef);
    a.vec16 = vec16 ? 1 : 0;
    void* args[] = {&p0, &p1, &a};
    if (qsv_status st = cuda_status(cudaLaunchKernel(kerns[ps.full ? 1 : 0], dim3((unsigned)ntiles),
                                                     dim3(threads),
                                                     args, smem_stage, s->stream),
                                    "fused stage launch"))
      return st;
    count_launch();
    if (profile) cudaEventRecord(ev[si + 1], s->stream);
  }
  if (profile) {
    qsv_status st = cuda_status(cudaEventSynchronize(ev.back()), "stage timing synchronize");
    g_stage_ms.clear();
    for (size_t si = 0; si < plan.stages.size() && !st; ++si) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[si], ev[si + 1]);
      g_stage_ms.push_back(ms);
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (st) return st;
  }
  if (x.nslots > 0) return reduce_rows(x, ntiles);
  return QSV_SUCCESS;
}

}  // namespace

qsv_status reduce_rows(const ExecArgs& x, uint64_t ntiles) {
  k_rows<<<x.nslots, 256, 0, x.s->stream>>>(x.partial, (int)ntiles, x.rows_out);
  count_launch();
  return cuda_status(cudaGetLastError(), "row reduction launch");
}

int default_tile_bits(size_t eb, int nv) { return (eb >= 16 ? 12 : 13) - (nv == 2 ? 1 : 0); }

int effective_tile_bits(size_t eb, int nv, int n, const qsv_fuse_opts* opts) {
  int m = (opts && opts->tile_bits > 0) ? opts->tile_bits : default_tile_bits(eb, nv);
  if (m > 14) m = 14;
  if (m > n) m = n;
  const int r = pass_bits(eb, nv, m);
  const int turns = (eb >= 16) ? fx::turn_bits<double2>(nv) : fx::turn_bits<float2>(nv);
  if (m - r > 8 + turns) m = r + 8 + turns;  // at most 256 threads per CTA
  return m;
}
int default_low_bits(size_t eb) { return eb >= 16 ? 2 : 3; }

// complex<float> gate passes keep 4 low bits unless told otherwise: a
// 128-byte innermost TMA box and fewer passes (30-qubit brick, depth 40:
// 166 passes in 503 ms against 192 passes in 528 ms with 3 low bits)
int gate_default_low(size_t eb) { return eb == 8 ? 4 : default_low_bits(eb); }

unsigned* sweep_wait_flag() {
  static unsigned* addr = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_tc_status) == cudaSuccess) addr = static_cast<unsigned*>(p);
  });
  if (addr) g_tc_used = true;
  return addr;
}

qsv_status tc_check_status(cudaStream_t stream) {
  if (!g_tc_used.load(std::memory_order_relaxed)) return QSV_SUCCESS;
  unsigned v = 0;
  if (qsv_status st = cuda_status(cudaMemcpyFromSymbolAsync(&v, g_tc_status, sizeof(v), 0,
                                                            cudaMemcpyDeviceToHost, stream),
                                  "tensor-core status read"))
    return st;
  if (qsv_status st = cuda_status(cudaStreamSynchronize(stream), "tensor-core status read"))
    return st;
  if (!v) return QSV_SUCCESS;
  static const unsigned zero = 0;
  cudaMemcpyToSymbolAsync(g_tc_status, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, stream);
  cudaStreamSynchronize(stream);
  return fail(QSV_ERROR_TIMEOUT,
              "a fused sweep gave up waiting for its MMAs or tile copies, or found a tile copy "
              "outside its shared memory (results invalid)");
}

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

namespace qsv {
namespace {

// The executor's plan of a single-vector sweep: ops and passes per stage.
template <typename V>
qsv_status plan_counts(const std::vector<Lowered>& low, int n, const qsv_fuse_opts* opts,
                       std::vector<int>* ops, std::vector<int>* passes) {
  if constexpr (Elem<V>::cplx) {
    const int mg = use_gate_engine<V>(opts) ? gate_tile_bits<V>(n, opts) : -1;
    if (mg > 0) {
      const int lowb = std::min((opts && opts->low_bits > 0) ? opts->low_bits
                                                             : gate_default_low(sizeof(V)), mg);
      const int max_gates = (opts && opts->max_stage_gates > 0) ? opts->max_stage_gates : 256;
      std::vector<int> o, p;
      const qsv_status st = gate_plan_counts(low, n, mg, lowb, opts, max_gates, sizeof(V), &o, &p);
      if (st == QSV_SUCCESS) {
        *ops = o;
        *passes = p;
        return st;
      }
      if (st != QSV_ERROR_NOT_SUPPORTED) return st;
    }
  }
  const int md = dmma_tile_bits<V>(n, opts);
  if (md > 0) {  // the tensor-core engine's plan (its ops are the passes' matrices)
    const int lowb = std::min((opts && opts->low_bits > 0) ? opts->low_bits : default_low_bits(sizeof(V)), md);
    const int max_gates = (opts && opts->max_stage_gates > 0) ? opts->max_stage_gates : 256;
    fx::PackedPlan<double2> plan;
    int low_used = lowb;
    if (qsv_status st = pack_dense_plan(low, n, md, lowb, opts && opts->low_bits > 0,
                                        dmma_pass_bits(md), max_gates, sizeof(V), &plan, &low_used))
      return st;
    for (const fx::PackedStage& ps : plan.stages) {
      ops->push_back(ps.nops);
      passes->push_back((int)ps.npasses);
    }
    return QSV_SUCCESS;
  }
  const int m = effective_tile_bits(sizeof(V), 1, n, opts);
  const int lowb = (opts && opts->low_bits > 0) ? opts->low_bits : default_low_bits(sizeof(V));
  const int max_gates = (opts && opts->max_stage_gates > 0) ? opts->max_stage_gates : 256;
  fx::PackedPlan<V> plan;
  if (qsv_status st = fx::pack_plan<V>(low, n, m, lowb, pass_bits(sizeof(V), 1, m), max_gates, &plan))
    return st;
  for (const fx::PackedStage& ps : plan.stages) {
    ops->push_back(ps.nops);
    passes->push_back((int)ps.npasses);
  }
  return QSV_SUCCESS;
}

qsv_status plan_counts_any(int nbQubits, qsv_dtype dtype, const qsv_gate* gates, size_t nGates,
                           char op, int offset, const qsv_fuse_opts* opts, std::vector<int>* ops,
                           std::vector<int>* passes) {
  if (!dtype_valid(dtype)) return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
  if (nbQubits < 1 || nbQubits > kMaxQubits) return fail(QSV_ERROR_SIZE, "bad nbQubits");
  qsv_state_s fake;
  fake.n = nbQubits;
  fake.dtype = dtype;
  std::vector<Lowered> low;
  if (qsv_status st = lower_for_state(&fake, gates, nGates, op, offset, &low, true)) return st;
  switch (dtype) {
    case QSV_C128: return plan_counts<double2>(low, nbQubits, opts, ops, passes);
    case QSV_C64:  return plan_counts<float2>(low, nbQubits, opts, ops, passes);
    case QSV_F64:  return plan_counts<double>(low, nbQubits, opts, ops, passes);
    default:       return plan_counts<float>(low, nbQubits, opts, ops, passes);
  }
}

}  // namespace
}  // namespace qsv

extern "C" qsv_status qsv_plan_stats(int nbQubits, qsv_dtype dtype, const qsv_gate* gates,
                                     size_t nGates, char op, int offset,
                                     const qsv_fuse_opts* opts, int* nStages, int* stage_gates,
                                     int capacity) {
  using namespace qsv;
  if (!nStages) return fail(QSV_ERROR_INVALID_VALUE, "null nStages");
  std::vector<int> ops, passes;
  if (qsv_status st = plan_counts_any(nbQubits, dtype, gates, nGates, op, offset, opts, &ops, &passes))
    return st;
  *nStages = (int)ops.size();
  if (stage_gates)
    for (int i = 0; i < capacity && i < (int)ops.size(); ++i) stage_gates[i] = ops[i];
  return QSV_SUCCESS;
}

extern "C" qsv_status qsv_plan_passes(int nbQubits, qsv_dtype dtype, const qsv_gate* gates,
                                      size_t nGates, char op, int offset,
                                      const qsv_fuse_opts* opts, int* nStages, int* nPasses,
                                      int* nOps) {
  using namespace qsv;
  if (!nStages || !nPasses || !nOps) return fail(QSV_ERROR_INVALID_VALUE, "null output");
  std::vector<int> ops, passes;
  if (qsv_status st = plan_counts_any(nbQubits, dtype, gates, nGates, op, offset, opts, &ops, &passes))
    return st;
  *nStages = (int)ops.size();
  *nPasses = 0;
  *nOps = 0;
  for (size_t i = 0; i < ops.size(); ++i) {
    *nPasses += passes[i];
    *nOps += ops[i];
  }
  return QSV_SUCCESS;
}

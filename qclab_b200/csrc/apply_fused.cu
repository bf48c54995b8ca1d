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
#include <cstring>
#include <vector>
#include "fused.hpp"
#include "stage_exec.cuh"

namespace qsv {

static thread_local std::vector<float> g_stage_ms;

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

template <typename V>
qsv_status pack_plan(const std::vector<Lowered>& gates, int n, int m, int low, int r,
                     int max_gates, PackedPlan<V>* out) {
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
    std::vector<Pass> pl = plan_passes(op_bits, stg.m, r);
    for (const Pass& p : pl) {
      PassDev pd{};
      for (int k = 0; k < 8; ++k) pd.pos[k] = (k < p.r) ? (int8_t)p.pos[k] : 0;
      pd.op0 = (int32_t)(out->ops.size() - ps.op0);
      pd.nops = (int32_t)p.ops.size();
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
        if (out->coefs.size() - ps.coef0 > 30000)
          return fail(QSV_ERROR_SIZE, "fused stage too large");
        op.coef = (int16_t)(out->coefs.size() - ps.coef0);
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
            break;
          }
          default:
            return fail(QSV_ERROR_INVALID_VALUE, "internal: shape %d in a fused stage", L.shape);
        }
        for (int i = 0; i < nc; ++i) out->coefs.push_back(host_coef<V>(L.m, i));
        out->ops.push_back(op);
      }
      out->passes.push_back(pd);
    }
    ps.npasses = out->passes.size() - ps.pass0;
    ps.nops = (int)(out->ops.size() - ps.op0);
    ps.ncoef = (int)(out->coefs.size() - ps.coef0);
    if (plan_smem_bytes<V>((int)ps.npasses, ps.nops, ps.ncoef) > kPlanSmemMax)
      return fail(QSV_ERROR_INVALID_VALUE, "internal: stage plan exceeds its shared-memory budget");
    tile_runoffs(stg.bits, stg.m, low, &out->runoff);
    out->stages.push_back(ps);
  }
  return QSV_SUCCESS;
}

template qsv_status pack_plan<double2>(const std::vector<Lowered>&, int, int, int, int, int, PackedPlan<double2>*);
template qsv_status pack_plan<float2>(const std::vector<Lowered>&, int, int, int, int, int, PackedPlan<float2>*);
template qsv_status pack_plan<double>(const std::vector<Lowered>&, int, int, int, int, int, PackedPlan<double>*);
template qsv_status pack_plan<float>(const std::vector<Lowered>&, int, int, int, int, int, PackedPlan<float>*);

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
  if (x.nslots > 0) {
    k_rows<<<x.nslots, 256, 0, s->stream>>>(x.partial, (int)ntiles, x.rows_out);
    count_launch();
    if (qsv_status st = cuda_status(cudaGetLastError(), "row reduction launch")) return st;
  }
  return QSV_SUCCESS;
}

}  // namespace

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
  if (qsv_status st = lower_for_state(&fake, gates, nGates, op, offset, &low)) return st;
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

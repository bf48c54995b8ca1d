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
#include "gate_exec.cuh"
#include "gate_plan.hpp"
#include "stage_exec.cuh"
#include "tma.cuh"

namespace qsv {
namespace gx {

struct GxArgs {
  TileArgs ta;
  int npasses, nops;  // the stage's plan (GxStagePlan)
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

// A stage's plan (passes | op words | coefficients, the layout of
// gx_plan_smem), passed by value as a kernel parameter: the kernel reads it
// from the constant bank, where the warp-uniform op words, coefficients and
// pass descriptors load without a shared-memory copy per CTA (measured 4 %
// faster on a 32-qubit complex<float> brick than staging it in shared
// memory).
struct alignas(16) GxStagePlan {
  unsigned char bytes[kGxPlanCap];
};

template <typename V, int R, int NT, int MINB, int NV, bool GEN = false>
__global__ void __launch_bounds__(NT, MINB)
    k_gates(V* __restrict__ v0, V* __restrict__ v1, GxArgs a,
            const __grid_constant__ CUtensorMap tm0, const __grid_constant__ CUtensorMap tm1,
            const __grid_constant__ GxStagePlan sp) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  __shared__ uint64_t tile_bar;
  // the tiles start on a 1024-byte boundary (the TMA swizzle blocks; the
  // launch reserves the padding)
  unsigned char* smem_raw = tma::align1024(smem_dyn);
  const uint32_t size = 1u << a.ta.m;
  V* t0 = reinterpret_cast<V*>(smem_raw);
  V* t1 = t0 + size;
  // two-vector sweeps: the gradient terms' per-warp accumulators after the
  // tiles
  double* racc = reinterpret_cast<double*>(smem_raw + size_t(NV) * size * sizeof(V));
  const unsigned char* pp = sp.bytes;
  const unsigned char* po = pp + align16(size_t(a.npasses) * sizeof(GxPassDev));
  const unsigned char* pc = po + align16(size_t(a.nops) * sizeof(uint32_t));
  const uint64_t base = tile_base(a.ta, blockIdx.x);
  if (a.tma.use) {  // one thread starts the tile's copies
    if (!tma::tile_fits<NV>(a.tma, smem_dyn, t0, size * sizeof(V), a.smem_bytes, a.wait_error))
      return;
    tma::tile_start<NV>(a.tma, &tm0, &tm1, t0, t1, base, &tile_bar);
  }
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
  run_gate_passes<V, R, NV, GEN>(t0, t1, passes, a.npasses, ops, coefs, racc, a.ta.m);
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
  // device words and element-type coefficients (copied into each stage's
  // parameter block at its launch)
  std::vector<uint32_t> hw(plan.ops.size());
  for (size_t i = 0; i < plan.ops.size(); ++i) {
    const uint32_t w = plan.ops[i];
    hw[i] = device_word((int)(w & ((1u << kCodeBits) - 1u)), R, w >> kCodeBits);
  }
  std::vector<V> hc(plan.coefs.size());
  for (size_t i = 0; i < plan.coefs.size(); ++i) hc[i] = to_elem<V>(plan.coefs[i]);
  // device scratch: the stages' tile run offsets and gradient rows
  auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
  const size_t run_off = 0;
  const size_t red_off = align(run_off + runoff.size() * sizeof(uint64_t));
  const size_t total = red_off + plan.red_slots.size() * sizeof(int32_t);
  std::vector<unsigned char> host(total);
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
    a.vec16 = vec16 ? 1 : 0;
    a.tma = geos[si];
    a.wait_error = wait_error;
    // + 1024: the tiles are placed on a 1024-byte boundary
    const size_t smem = (size_t(1) << gs.m) * sizeof(V) * nv + (nv == 2 ? fx::kRaccBytes : 0) +
                        1024;
    if (smem > 200 * 1024)
      return fail(QSV_ERROR_SIZE, "gate stage needs %zu bytes of shared memory", smem);
    a.smem_bytes = (uint32_t)smem;
    // the stage's plan as the kernel's parameter block (the planner caps it
    // at kGxPlanCap bytes)
    GxStagePlan sp;
    {
      const size_t pb = gs.npasses * sizeof(GxPassDev), ob = gs.nops * sizeof(uint32_t);
      if (gx_plan_smem<V>(gs.npasses, gs.nops, gs.ncoef) > sizeof(sp.bytes))
        return fail(QSV_ERROR_SIZE, "gate stage plan exceeds the parameter block");
      std::memset(sp.bytes, 0, sizeof(sp.bytes));
      std::memcpy(sp.bytes, dpass.data() + gs.pass0, pb);
      std::memcpy(sp.bytes + align16(pb), hw.data() + gs.op0, ob);
      std::memcpy(sp.bytes + align16(pb) + align16(ob), hc.data() + gs.coef0, gs.ncoef * sizeof(V));
    }
    void* args[] = {&p0, &p1, &a, &maps[2 * si], &maps[2 * si + (nv == 2 ? 1 : 0)], &sp};
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

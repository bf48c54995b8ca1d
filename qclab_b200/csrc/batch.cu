// Batched variational sweep: many small circuits (each with its own qubit
// count, gate list and Pauli-sum observable) -> energy <psi|H|psi> and the
// full adjoint gradient of every circuit, in ONE persistent kernel launch
// captured in a CUDA graph.
//
// Every CTA pulls job indices from an atomic work counter (largest
// circuits first).  A circuit that fits one tile runs on one CTA; a larger
// one is split into a team of up to 16 consecutive jobs whose CTAs share its
// tiles stage by stage, meeting at a team barrier (a counter in global
// memory, bounded waits) between stages, so a few large circuits no longer
// hold single CTAs long after the rest of the batch is done.  Each circuit
// runs
//   forward fused stages on psi  ->  lambda = H psi and E = <psi|lambda>
//   ->  backward fused stages on (psi, lambda) with in-tile gradient terms.
// A circuit whose two vectors fit in the CTA's shared memory (n <= m) never
// touches global memory except for its results; larger circuits stream
// their tiles through a per-CTA slot of a global workspace.  The stage and
// pass plans come from the same planner as the single-state fused path, and
// the passes are the gate-specialised register passes (gate_plan.hpp,
// gate_exec.cuh: every gate one op with compile-time register positions,
// one-qubit gates factored to two multiply-adds per component), packed for
// all circuits into one device buffer.
// Gradient terms are summed by warp shuffles into a per-stage shared-memory
// accumulator and added to the results once per stage, all in a fixed order,
// so results are deterministic.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>
#include "fused.hpp"
#include "gate_exec.cuh"
#include "gate_plan.hpp"
#include "stage_exec.cuh"

using namespace qsv;
using namespace qsv::fx;

struct qsv_batch_s {
  qsv_dtype dtype = QSV_C64;
  int ncirc = 0;
  int tile_bits = 12;
  int blocks = 0;
  int threads = 128;
  size_t smem = 0;
  bool gen = false;           // backward stages hold generic gradient terms
  double global_bytes = 0;    // per launch: tile traffic of the circuits larger than a tile
  double amp_updates = 0;     // per launch: gate x amplitude updates (both vectors)
  void* plan = nullptr;       // packed plan (device)
  size_t plan_bytes = 0;
  void* work = nullptr;       // per-CTA workspace (device)
  size_t work_bytes = 0;
  double* results = nullptr;  // [ncirc energies][grads] (device)
  size_t nresults = 0;
  unsigned* counter = nullptr;
  unsigned* team_sync = nullptr;  // inside the results allocation
  double* team_part = nullptr;
  unsigned* error = nullptr;
  size_t zero_bytes = 0;          // results + team state, zeroed before every launch
  int njobs = 0;                  // job entries (a team counts once per member)
  int nteams = 0;
  std::vector<size_t> grad_off;  // per circuit, into the gradient part
  std::vector<int> nparams;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t captured_on = nullptr;
  // offsets of the plan sections
  size_t off_jobs = 0, off_stages = 0, off_passes = 0, off_ops = 0, off_coefs = 0,
         off_runoff = 0, off_groups = 0, off_terms = 0, off_red = 0;
};

namespace {

struct BStage {          // one fused stage of one circuit
  int8_t bits[32];       // local tile bit -> global bit
  int32_t m, pad;
  int32_t pass0, npasses, op0, coef0;  // into the plan arrays (absolute)
  int32_t run0;                        // runoff offset (absolute)
  int32_t red0, nred;                  // gradient reductions: red_slots[red0..+nred)
  int32_t nops, ncoef;                 // ops and coefficients (staged in shared memory)
};

struct BGroup {          // observable term group (terms whose flips fit a tile)
  int8_t bits[32];
  int32_t m;
  int32_t term0, nterms;
  int32_t run0;
};

struct BTerm {
  uint32_t flip_local;
  uint32_t pad;
  uint64_t flip, zy;     // global masks
  double wr, wi;         // coef * i^ny
};

struct BJob {
  int32_t n, m, low;
  int32_t fwd0, nfwd, bwd0, nbwd;   // stage ranges
  int32_t grp0, ngrp;               // term-group range
  int32_t circ;                     // circuit index (results)
  int32_t team, rank, team_id;      // team size (1: one CTA), this job's rank, team index
  int32_t nparams;
  int64_t grad_off;                 // into results (after the energies)
  int64_t part_off;                 // team: its partial sums in BArgs.team_part
};

struct BArgs {
  const BJob* jobs;
  int njobs;
  const BStage* stages;
  const gx::GxPassDev* passes;
  const uint32_t* ops;   // op words (gate_plan.hpp device_word)
  const void* coefs;
  const uint64_t* runoff;
  const BGroup* groups;
  const BTerm* terms;
  const int32_t* red_slots;
  void* work;
  size_t work_stride;    // elements per CTA slot (2 vectors)
  double* results;       // [ncirc] energies, then gradients
  unsigned* counter;
  unsigned* team_sync;   // per team: [arrivals, 1 + blockIdx of rank 0, -, -]; then the error flag
  double* team_part;     // per team: energies[team], then gradients[team][nparams]
  unsigned* error;       // set when a team barrier gave up waiting
  int vec16;
  int tile_elems;        // 2^M: the shared-memory tiles hold 2 x tile_elems elements
};

// Spins of a team barrier before it gives up (with __nanosleep(100) each,
// a few seconds): the persistent grid is resident and teams are handed out
// in order, so every member arrives; the limit only bounds a broken run.
// Once one barrier has given up (the error flag), the others stop waiting.
constexpr unsigned kTeamSpinLimit = 1u << 25;

// Team barrier: all T members arrive, then each waits for the k-th round
// (arrivals >= T (k + 1)).  Global writes before it are visible after it.
__device__ __forceinline__ void team_barrier(unsigned* arrive, unsigned target, unsigned* error) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(arrive, 1u);
    unsigned spins = 0;
    while (true) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(arrive) : "memory");
      if (v >= target) break;
      if (++spins > kTeamSpinLimit) {
        atomicOr(error, 1u);
        break;
      }
      if ((spins & 1023u) == 0) {
        unsigned e;
        asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(e) : "l"(error) : "memory");
        if (e) break;
      }
      __nanosleep(100);
    }
    __threadfence();
  }
  __syncthreads();
}

template <typename V>
__device__ __forceinline__ TileArgs stage_tile(const BStage& S, int n, int low,
                                               const uint64_t* runoff) {
  TileArgs ta;
  ta.n = n;
  ta.m = S.m;
  ta.low = low;
  for (int j = 0; j < 32; ++j) ta.bits[j] = S.bits[j];
  ta.runoff = runoff + S.run0;
  return ta;
}

// One fused stage of a job on psi (NV = 1) or psi and lambda (NV = 2): the
// stage's plan (pass descriptors | op words | coefficients) is staged in
// shared memory once, then every tile of the stage is swept (the one
// resident tile of a circuit that fits shared memory).  Threads beyond the
// stage's 2^(m-R) register groups idle in the passes.
template <typename V, int NV, int R, bool GEN>
__device__ __forceinline__ void run_stage(const BStage& S, int n, int low, bool single,
                                          const BArgs& a, V* t0, V* t1, V* psi, V* lam,
                                          double* racc, unsigned char* plan, int rank = 0,
                                          int team = 1) {
  unsigned char* po = plan + align16(size_t(S.npasses) * sizeof(gx::GxPassDev));
  unsigned char* pc = po + align16(size_t(S.nops) * sizeof(uint32_t));
  copy_words(plan, a.passes + S.pass0, size_t(S.npasses) * sizeof(gx::GxPassDev));
  copy_words(po, a.ops + S.op0, size_t(S.nops) * sizeof(uint32_t));
  copy_words(pc, static_cast<const V*>(a.coefs) + S.coef0, size_t(S.ncoef) * sizeof(V));
  __syncthreads();
  const gx::GxPassDev* passes = reinterpret_cast<const gx::GxPassDev*>(plan);
  const uint32_t* ops = reinterpret_cast<const uint32_t*>(po);
  const V* coefs = reinterpret_cast<const V*>(pc);
  if (single) {
    gx::run_gate_passes<V, R, NV, GEN>(t0, t1, passes, S.npasses, ops, coefs, racc, S.m);
    return;
  }
  const TileArgs ta = stage_tile<V>(S, n, low, a.runoff);
  const uint64_t ntiles = 1ull << (n - S.m);
  for (uint64_t t = rank; t < ntiles; t += team) {
    const uint64_t base = tile_base(ta, t);
    load_tile<V, NV>(psi, lam, t0, t1, ta, base, a.vec16);
    __syncthreads();
    gx::run_gate_passes<V, R, NV, GEN>(t0, t1, passes, S.npasses, ops, coefs, racc, S.m);
    store_tile<V, NV>(psi, lam, t0, t1, ta, base, a.vec16);
    __syncthreads();
  }
}

// lambda (+)= H_group psi on a resident tile; returns this thread's
// contribution to <psi|H_group psi>.
template <typename V>
__device__ __forceinline__ double apply_group(const V* t0, V* t1, const BGroup& G,
                                              const BTerm* __restrict__ terms, uint64_t base,
                                              const uint64_t* runoff, int low, bool accumulate) {
  const uint32_t size = 1u << G.m, lowmask = (1u << low) - 1u;
  double e = 0.0;
  for (uint32_t el = threadIdx.x; el < size; el += blockDim.x) {
    const uint64_t g = base | runoff[el >> low] | (el & lowmask);
    double2 acc = accumulate ? to_d2(t1[phys<V>(el)]) : make_double2(0.0, 0.0);
    double2 add = make_double2(0.0, 0.0);
    for (int t = 0; t < G.nterms; ++t) {
      const BTerm T = terms[G.term0 + t];
      const double2 y = to_d2(t0[phys<V>(el ^ T.flip_local)]);
      const double sg = (__popcll((g ^ T.flip) & T.zy) & 1) ? -1.0 : 1.0;
      add.x = fma(sg * T.wr, y.x, fma(-sg * T.wi, y.y, add.x));
      add.y = fma(sg * T.wr, y.y, fma(sg * T.wi, y.x, add.y));
    }
    const double2 x = to_d2(t0[phys<V>(el)]);
    e += x.x * add.x + x.y * add.y;  // Re(conj(psi) * (H_g psi))
    acc.x += add.x;
    acc.y += add.y;
    t1[phys<V>(el)] = from_d2<V>(acc);
  }
  return e;
}

// The persistent kernel runs CTAs of kBatchThreads threads, compiled for
// three per SM (168 registers a thread: the two-vector gate passes hold 2 x
// 2^RB amplitudes plus the op dispatch's temporaries; complex<float> spills
// about 70 bytes).  Shared memory admits three with 2^11-amplitude tiles
// (two with 2^12): on the 4096-circuit batch 2^11 tiles at three CTAs per SM
// took 265-270 ms against 286-289 ms with 2^12 tiles at two (compiled for
// two per SM, 236 registers, no spills: the same 288 ms).  GEN: the backward
// stages hold generic gradient terms (gate_exec.cuh red_generic).
constexpr int kBatchThreads = 128;
#ifndef QSV_BATCH_MINBLOCKS
#define QSV_BATCH_MINBLOCKS 3
#endif

template <typename V, int RF, int RB, bool GEN>
__global__ void __launch_bounds__(kBatchThreads, QSV_BATCH_MINBLOCKS)
k_batch(BArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double2 red[32];
  __shared__ int job_s;
  __shared__ unsigned slot_s;
  V* t0 = reinterpret_cast<V*>(smem_raw);
  double* racc = reinterpret_cast<double*>(smem_raw + size_t(2) * a.tile_elems * sizeof(V));
  unsigned char* plan = smem_raw + size_t(2) * a.tile_elems * sizeof(V) + kRaccBytes;
  for (;;) {
    if (threadIdx.x == 0) job_s = (int)atomicAdd(a.counter, 1u);
    __syncthreads();
    const int jb = job_s;
    __syncthreads();
    if (jb >= a.njobs) break;
    const BJob J = a.jobs[jb];
    const uint32_t tsize = 1u << J.m;
    V* t1 = t0 + tsize;
    const bool single = (J.m == J.n);
    const int team = J.team, rank = J.rank;
    unsigned* arrive = a.team_sync + 4 * (size_t)J.team_id;
    unsigned rounds = 0;
    auto barrier = [&]() {
      if (team > 1) team_barrier(arrive, (unsigned)team * ++rounds, a.error);
    };
    // a team works in the workspace slot of its rank-0 CTA
    unsigned slot = blockIdx.x;
    if (team > 1) {
      if (rank == 0 && threadIdx.x == 0) {
        asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(arrive + 1), "r"(blockIdx.x + 1u)
                     : "memory");
      }
      barrier();
      if (threadIdx.x == 0) {
        unsigned v;
        asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(arrive + 1) : "memory");
        slot_s = v ? v - 1u : blockIdx.x;
      }
      __syncthreads();
      slot = slot_s;
    }
    V* psi = static_cast<V*>(a.work) + (size_t)slot * a.work_stride;
    V* lam = psi + ((size_t)1 << J.n);
    const uint64_t N = 1ull << J.n;
    // gradients: straight into the results for one CTA, else into this
    // member's row of the team's partial sums (summed in rank order at the end)
    double* grads = team > 1 ? a.team_part + J.part_off + team + (size_t)rank * J.nparams
                             : a.results + J.grad_off;
    // (results and partial sums were zeroed before the launch)

    // ---- psi = |0...0> ----
    if (single) {
      for (uint32_t e = threadIdx.x; e < tsize; e += blockDim.x)
        t0[phys<V>(e)] = from_d2<V>(make_double2(e == 0 ? 1.0 : 0.0, 0.0));
    } else {
      for (uint64_t e = (uint64_t)rank * blockDim.x + threadIdx.x; e < N;
           e += (uint64_t)team * blockDim.x)
        psi[e] = from_d2<V>(make_double2(e == 0 ? 1.0 : 0.0, 0.0));
    }
    __syncthreads();
    barrier();

    // ---- forward ----
    for (int s = 0; s < J.nfwd; ++s) {
      run_stage<V, 1, RF, false>(a.stages[J.fwd0 + s], J.n, J.low, single, a, t0, t1, psi, lam,
                                 racc, plan, rank, team);
      barrier();
    }

    // ---- lambda = H psi, E = <psi|H|psi> ----
    double e = 0.0;
    if (J.ngrp == 0) {  // H = 0: lambda = 0
      if (single) {
        for (uint32_t el = threadIdx.x; el < tsize; el += blockDim.x) t1[el] = from_d2<V>(make_double2(0.0, 0.0));
      } else {
        for (uint64_t el = (uint64_t)rank * blockDim.x + threadIdx.x; el < N;
             el += (uint64_t)team * blockDim.x)
          lam[el] = from_d2<V>(make_double2(0.0, 0.0));
      }
      __syncthreads();
      barrier();
    }
    for (int g = 0; g < J.ngrp; ++g) {
      const BGroup G = a.groups[J.grp0 + g];
      if (single) {
        e += apply_group<V>(t0, t1, G, a.terms, 0, a.runoff + G.run0, J.low, g > 0);
        __syncthreads();
      } else {
        TileArgs ta;
        ta.n = J.n;
        ta.m = G.m;
        ta.low = J.low;
        for (int j = 0; j < 32; ++j) ta.bits[j] = G.bits[j];
        ta.runoff = a.runoff + G.run0;
        const uint64_t ntiles = 1ull << (J.n - G.m);
        for (uint64_t t = rank; t < ntiles; t += team) {
          const uint64_t base = tile_base(ta, t);
          if (g > 0) load_tile<V, 2>(psi, lam, t0, t1, ta, base, a.vec16);
          else load_tile<V, 1>(psi, nullptr, t0, nullptr, ta, base, a.vec16);
          __syncthreads();
          e += apply_group<V>(t0, t1, G, a.terms, base, ta.runoff, J.low, g > 0);
          __syncthreads();
          store_tile<V, 1>(lam, nullptr, t1, nullptr, ta, base, a.vec16);
          __syncthreads();
        }
        barrier();
      }
    }
    const double2 et = block_sum(make_double2(e, 0.0), red);
    if (threadIdx.x == 0) {
      if (team > 1) a.team_part[J.part_off + rank] = et.x;
      else a.results[J.circ] = et.x;
    }
    __syncthreads();

    // ---- backward: uncompute psi and lambda, gradient terms in-tile ----
    for (int s = 0; s < J.nbwd; ++s) {
      const BStage S = a.stages[J.bwd0 + s];
      for (int i = threadIdx.x; i < S.nred * kRedWarps; i += blockDim.x) racc[i] = 0.0;
      run_stage<V, 2, RB, GEN>(S, J.n, J.low, single, a, t0, t1, psi, lam, racc, plan, rank,
                               team);
      // the stage's gradient terms, summed over warps in a fixed order by one
      // thread (parameters may repeat within a stage)
      if (threadIdx.x == 0) {
        const int warps = red_warps();
        for (int r = 0; r < S.nred; ++r) {
          double t = 0.0;
          for (int w = 0; w < warps; ++w) t += racc[r * kRedWarps + w];
          grads[a.red_slots[S.red0 + r]] += t;
        }
      }
      __syncthreads();
      barrier();
    }
    // a team's energy and gradients: rank 0 sums the members' rows in rank order
    barrier();
    if (team > 1 && rank == 0) {
      const double* part = a.team_part + J.part_off;
      if (threadIdx.x == 0) {
        double et2 = 0.0;
        for (int r = 0; r < team; ++r) et2 += part[r];
        a.results[J.circ] = et2;
      }
      for (int q = threadIdx.x; q < J.nparams; q += blockDim.x) {
        double t = 0.0;
        for (int r = 0; r < team; ++r) t += part[team + (size_t)r * J.nparams + q];
        a.results[J.grad_off + q] = t;
      }
    }
    __syncthreads();
  }
}

template <typename V> V batch_coef(gx::cplx z);
template <> double2 batch_coef<double2>(gx::cplx z) { return make_double2(z.real(), z.imag()); }
template <> float2 batch_coef<float2>(gx::cplx z) {
  return make_float2((float)z.real(), (float)z.imag());
}

template <typename V>
constexpr int fwd_bits() { return reg_bits<V>(1); }
template <typename V>
constexpr int bwd_bits() { return reg_bits<V>(2); }

struct HTermH {
  uint64_t flip, zy;
  int ny;
  double coef;
};

qsv_status parse_obs(int n, const char* paulis, const double* coefs, size_t nt,
                     std::vector<HTermH>* out) {
  out->clear();
  for (size_t t = 0; t < nt; ++t) {
    HTermH h{0, 0, 0, coefs[t]};
    for (int q = 0; q < n; ++q) {
      const char c = paulis[t * (size_t)n + q];
      const uint64_t b = 1ull << (n - 1 - q);
      switch (c) {
        case 'I': case 'i': break;
        case 'X': case 'x': h.flip |= b; break;
        case 'Y': case 'y': h.flip |= b; h.zy |= b; ++h.ny; break;
        case 'Z': case 'z': h.zy |= b; break;
        default: return fail(QSV_ERROR_INVALID_VALUE, "term %zu: '%c' is not I, X, Y or Z", t, c);
      }
    }
    out->push_back(h);
  }
  return QSV_SUCCESS;
}

template <typename V>
qsv_status build_batch(qsv_batch_s* b, int ncirc, const int* nq, const qsv_gate* gates,
                       const size_t* gate_off, const char* paulis, const size_t* char_off,
                       const double* coefs, const size_t* term_off, const int* nparams,
                       const qsv_batch_opts* opts) {
  constexpr int RF = fwd_bits<V>(), RB = bwd_bits<V>();
  const int M = (opts && opts->tile_bits > 0) ? opts->tile_bits : 11;
  const int low = (opts && opts->low_bits > 0) ? opts->low_bits : default_low_bits(sizeof(V));
  if (M < RF || M - RB > 8 || M > 14)
    return fail(QSV_ERROR_INVALID_VALUE, "batch tile_bits %d outside [%d, %d]", M, RF, RB + 8);
  const size_t smem = (size_t(2) << M) * sizeof(V) + kRaccBytes + kPlanSmemMax;
  if (smem > 200 * 1024) return fail(QSV_ERROR_SIZE, "batch tiles exceed shared memory");

  PackedPlan<V> plan;  // run offsets of stages and term groups
  std::vector<gx::GxPassDev> gpasses;
  std::vector<uint32_t> gops;
  std::vector<V> gcoefs;
  std::vector<int32_t> gred;
  bool gen = false;
  std::vector<BStage> stages;
  std::vector<BGroup> groups;
  std::vector<BTerm> terms;
  std::vector<BJob> jobs;
  b->grad_off.assign(ncirc, 0);
  b->nparams.assign(ncirc, 0);
  size_t goff = ncirc;  // gradients follow the energies
  int nmax = 0;
  for (int c = 0; c < ncirc; ++c) {
    const int n = nq[c];
    if (n < RF || n > 30) return fail(QSV_ERROR_SIZE, "circuit %d: %d qubits outside [%d, 30]", c, n, RF);
    nmax = std::max(nmax, n);
    const int m = std::min(n, M);
    const int lo = std::min(low, m);
    const qsv_gate* g = gates + gate_off[c];
    const size_t ng = gate_off[c + 1] - gate_off[c];
    // forward
    qsv_state_s fake;
    fake.n = n;
    fake.dtype = b->dtype;
    std::vector<Lowered> fwd;
    if (qsv_status st = lower_for_state(&fake, g, ng, 'N', 0, &fwd))
      return fail(st, "circuit %d: %s", c, qsv_last_error());
    // backward: [RED(param)] U^+ in reverse order
    std::vector<Lowered> bwd;
    for (size_t i = 0; i < ng; ++i) {
      const size_t k = ng - 1 - i;
      if (g[k].param >= 0) {
        if (g[k].param >= nparams[c])
          return fail(QSV_ERROR_INVALID_VALUE, "circuit %d gate %zu: param %d >= %d", c, k,
                      g[k].param, nparams[c]);
        Lowered R;
        R.shape = SH_RED;
        if (!generator_of(g[k], 0, n, &R.gen))
          return fail(QSV_ERROR_NOT_SUPPORTED, "circuit %d gate %zu has no trainable angle", c, k);
        R.slot = g[k].param;
        bwd.push_back(R);
      }
      Lowered inv;
      qsv_status st = dtype_double(b->dtype)
          ? lower_gate<double>(g[k], 'C', 0, n, dtype_real(b->dtype), &inv)
          : lower_gate<float>(g[k], 'C', 0, n, dtype_real(b->dtype), &inv);
      if (st) return fail(st, "circuit %d gate %zu could not be inverted", c, k);
      if (inv.shape != SH_NONE) bwd.push_back(inv);
    }
    BJob J{};
    J.n = n;
    J.m = m;
    J.low = lo;
    J.circ = c;
    J.team = 1;
    J.rank = 0;
    J.team_id = 0;
    J.nparams = nparams[c];
    J.part_off = 0;
    J.grad_off = (int64_t)goff;
    b->grad_off[c] = goff - ncirc;
    b->nparams[c] = nparams[c];
    goff += nparams[c];
    // gate-specialised plan of one direction -> device stages, passes (with
    // their shared-memory offsets for the cp.async tile layout), op words,
    // coefficients and gradient rows
    auto pack = [&](const std::vector<Lowered>& items, int r, bool two, int32_t* first,
                    int32_t* count) -> qsv_status {
      gx::GxPlan gp;
      if (!gx::pack_gate_plan(items, n, m, lo, r, 256, kPlanSmemMax, sizeof(V), &gp, two))
        return fail(QSV_ERROR_NOT_SUPPORTED, "circuit %d: a gate cannot run in a batched sweep", c);
      *first = (int32_t)stages.size();
      const uint32_t rdg = (uint32_t)gx::code_red(r, gx::G_RDG, 0);
      for (const gx::GxStage& gs : gp.stages) {
        BStage S{};
        for (int j = 0; j < 32; ++j) S.bits[j] = (int8_t)(j < gs.m ? gs.bits[j] : 0);
        S.m = gs.m;
        S.pass0 = (int32_t)gpasses.size();
        S.npasses = (int32_t)gs.npasses;
        S.op0 = (int32_t)gops.size();
        S.nops = (int32_t)gs.nops;
        S.coef0 = (int32_t)gcoefs.size();
        S.ncoef = (int32_t)gs.ncoef;
        S.red0 = (int32_t)gred.size();
        S.nred = gs.nred;
        S.run0 = (int32_t)plan.runoff.size();
        tile_runoffs(gs.bits, gs.m, lo, &plan.runoff);
        if (gx::gx_plan_smem<V>(gs.npasses, gs.nops, gs.ncoef) > kPlanSmemMax)
          return fail(QSV_ERROR_SIZE, "circuit %d: a stage plan exceeds shared memory", c);
        for (size_t pi = gs.pass0; pi < gs.pass0 + gs.npasses; ++pi) {
          const gx::GxPass& q = gp.passes[pi];
          gx::GxPassDev d{};
          int pos[8];
          for (int k = 0; k < 8; ++k) {
            d.pos[k] = q.pos[k];
            pos[k] = q.pos[k];
          }
          d.op0 = q.op0;
          d.nops = q.nops;
          for (int k = 0; k < r; ++k) d.boff[k] = phys_host(1u << pos[k], Units<V>::per);
          int order[32];
          const int ng = gx::lane_order(pos, r, gs.m, sizeof(V), order, -1);
          if (ng > 12) return fail(QSV_ERROR_SIZE, "circuit %d: stage of %d tile bits", c, gs.m);
          for (int k = 0; k < ng; ++k) d.goff[k] = phys_host(1u << order[k], Units<V>::per);
          gpasses.push_back(d);
        }
        for (size_t o = gs.op0; o < gs.op0 + gs.nops; ++o) {
          const uint32_t w = gp.ops[o];
          const uint32_t code = w & ((1u << gx::kCodeBits) - 1u);
          if (two && code == rdg) gen = true;
          gops.push_back(gx::device_word((int)code, r, w >> gx::kCodeBits));
        }
        for (size_t k = gs.coef0; k < gs.coef0 + gs.ncoef; ++k)
          gcoefs.push_back(batch_coef<V>(gp.coefs[k]));
        for (int k = 0; k < gs.nred; ++k) gred.push_back(gp.red_slots[gs.red0 + k]);
        stages.push_back(S);
      }
      *count = (int32_t)(stages.size() - *first);
      return QSV_SUCCESS;
    };
    if (qsv_status st = pack(fwd, RF, false, &J.fwd0, &J.nfwd)) return st;
    if (qsv_status st = pack(bwd, RB, true, &J.bwd0, &J.nbwd)) return st;
    {  // work of this circuit: every gate updates 2^n amplitudes (forward),
       // 2 x 2^n backward (psi and lambda)
      size_t nf = 0, nb = 0;
      for (const Lowered& L : fwd) nf += L.shape != SH_NONE;
      for (const Lowered& L : bwd) nb += L.shape != SH_NONE && L.shape != SH_RED;
      const double N = (double)(1ull << n);
      b->amp_updates += N * (double)(nf + 2 * nb);
    }
    // observable term groups (flip bits within an m-bit tile)
    std::vector<HTermH> H;
    const size_t nt = term_off[c + 1] - term_off[c];
    if (qsv_status st = parse_obs(n, paulis ? paulis + char_off[c] : nullptr, coefs + term_off[c],
                                  nt, &H))
      return st;
    const uint64_t lowmask = (1ull << lo) - 1ull;
    std::vector<uint64_t> sets;
    std::vector<std::vector<int>> members;
    for (int t = 0; t < (int)H.size(); ++t) {
      if (__builtin_popcountll(lowmask | H[t].flip) > m)
        return fail(QSV_ERROR_NOT_SUPPORTED, "circuit %d term %d flips more than %d bits", c, t, m);
      bool placed = false;
      for (size_t k = 0; k < sets.size() && !placed; ++k)
        if (__builtin_popcountll(sets[k] | H[t].flip) <= m) {
          sets[k] |= H[t].flip;
          members[k].push_back(t);
          placed = true;
        }
      if (!placed) {
        sets.push_back(lowmask | H[t].flip);
        members.push_back({t});
      }
    }
    J.grp0 = (int32_t)groups.size();
    J.ngrp = (int32_t)sets.size();
    for (size_t k = 0; k < sets.size(); ++k) {
      BGroup G{};
      int bits[64];
      G.m = tile_bits_of(sets[k], n, m, bits);
      for (int j = 0; j < 32; ++j) G.bits[j] = (int8_t)(j < G.m ? bits[j] : 0);
      G.run0 = (int32_t)plan.runoff.size();
      tile_runoffs(bits, G.m, lo, &plan.runoff);
      int local_of[64];
      for (int j = 0; j < 64; ++j) local_of[j] = -1;
      for (int j = 0; j < G.m; ++j) local_of[bits[j]] = j;
      G.term0 = (int32_t)terms.size();
      G.nterms = (int32_t)members[k].size();
      static const double pr[4] = {1, 0, -1, 0}, pi[4] = {0, 1, 0, -1};
      for (int t : members[k]) {
        BTerm T{};
        for (int q = 0; q < n; ++q)
          if ((H[t].flip >> q) & 1ull) T.flip_local |= 1u << local_of[q];
        T.flip = H[t].flip;
        T.zy = H[t].zy;
        T.wr = H[t].coef * pr[H[t].ny & 3];
        T.wi = H[t].coef * pi[H[t].ny & 3];
        terms.push_back(T);
      }
      groups.push_back(G);
    }
    if (n > m) {  // streamed through the workspace: every stage reads and
                  // writes its vector(s) once, a term group reads psi (and
                  // lambda after the first) and writes lambda
      const double vb = (double)(1ull << n) * sizeof(V);
      b->global_bytes += vb * (2.0 * J.nfwd + 4.0 * J.nbwd + 2.0 + 3.0 * (J.ngrp - 1));
    }
    jobs.push_back(J);
  }
  // largest circuits first (static cost estimate: amplitudes x stages)
  std::stable_sort(jobs.begin(), jobs.end(), [](const BJob& x, const BJob& y) {
    return ((double)(1ull << x.n) * (x.nfwd + x.nbwd + 1)) > ((double)(1ull << y.n) * (y.nfwd + y.nbwd + 1));
  });
  // launch shape (every CTA resident: the team barriers rely on it)
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  void* kern = gen ? (void*)k_batch<V, RF, RB, true> : (void*)k_batch<V, RF, RB, false>;
  if (qsv_status st = cuda_status(cudaFuncSetAttribute(kern,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)smem), "batch smem attribute"))
    return st;
  int per_sm = 0;
  // one thread per register group of the widest pass, kBatchThreads at most
  const int threads = std::max(32, std::min(kBatchThreads, 1 << (M - std::min(RF, RB))));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (opts && opts->ctas_per_sm > 0) per_sm = std::min(per_sm, opts->ctas_per_sm);
  if (per_sm < 1) return fail(QSV_ERROR_NOT_SUPPORTED, "batch kernel does not fit an SM");
  int blocks = sms * per_sm;
  const size_t stride = (size_t(2) << nmax);  // elements per CTA slot (psi + lambda)
  if (nmax > M) {  // every CTA needs a slot: at most 8 GiB of workspace in all
    const size_t cap = std::max<size_t>(1, (size_t(8) << 30) / (stride * sizeof(V)));
    blocks = (int)std::min<size_t>((size_t)blocks, cap);
  }
  // circuits larger than a tile become teams: one job per member, ranks
  // consecutive, at most max_team members and about two tiles per member
  // per stage, and never more than half the grid
  const int max_team = (opts && opts->max_team > 0) ? opts->max_team : 16;
  std::vector<BJob> entries;
  size_t part = 0;
  int nteams = 0;
  for (const BJob& J0 : jobs) {
    int T = 1;
    if (J0.n > J0.m) {
      const uint64_t ntiles = 1ull << (J0.n - J0.m);
      T = (int)std::min<uint64_t>((uint64_t)max_team, std::max<uint64_t>(1, ntiles / 2));
      T = std::max(1, std::min(T, blocks / 2));
    }
    if (T == 1) {
      entries.push_back(J0);
      continue;
    }
    for (int r = 0; r < T; ++r) {
      BJob J = J0;
      J.team = T;
      J.rank = r;
      J.team_id = nteams;
      J.part_off = (int64_t)part;
      entries.push_back(J);
    }
    part += (size_t)T * (1 + (size_t)J0.nparams);
    ++nteams;
  }
  jobs.swap(entries);
  b->njobs = (int)jobs.size();
  b->nteams = nteams;

  auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
  size_t off = 0;
  b->off_jobs = off;   off = align(off + jobs.size() * sizeof(BJob));
  b->off_stages = off; off = align(off + stages.size() * sizeof(BStage));
  b->off_passes = off; off = align(off + gpasses.size() * sizeof(gx::GxPassDev));
  b->off_ops = off;    off = align(off + gops.size() * sizeof(uint32_t));
  b->off_coefs = off;  off = align(off + gcoefs.size() * sizeof(V));
  b->off_runoff = off; off = align(off + plan.runoff.size() * sizeof(uint64_t));
  b->off_groups = off; off = align(off + groups.size() * sizeof(BGroup));
  b->off_terms = off;  off = align(off + terms.size() * sizeof(BTerm));
  b->off_red = off;    off = align(off + gred.size() * sizeof(int32_t));
  std::vector<unsigned char> host(off, 0);
  auto put = [&](size_t o, const void* p, size_t bytes) { if (bytes) std::memcpy(host.data() + o, p, bytes); };
  put(b->off_jobs, jobs.data(), jobs.size() * sizeof(BJob));
  put(b->off_stages, stages.data(), stages.size() * sizeof(BStage));
  put(b->off_passes, gpasses.data(), gpasses.size() * sizeof(gx::GxPassDev));
  put(b->off_ops, gops.data(), gops.size() * sizeof(uint32_t));
  put(b->off_coefs, gcoefs.data(), gcoefs.size() * sizeof(V));
  put(b->off_runoff, plan.runoff.data(), plan.runoff.size() * sizeof(uint64_t));
  put(b->off_groups, groups.data(), groups.size() * sizeof(BGroup));
  put(b->off_terms, terms.data(), terms.size() * sizeof(BTerm));
  put(b->off_red, gred.data(), gred.size() * sizeof(int32_t));

  // every CTA can hold a team member, but a grid smaller than the jobs is enough
  b->blocks = std::min<int>(blocks, b->njobs);
  b->threads = threads;
  b->gen = gen;
  b->smem = smem;
  b->tile_bits = M;
  b->work_bytes = (nmax > M) ? (size_t)b->blocks * stride * sizeof(V) : 256;
  b->nresults = goff;
  b->plan_bytes = off;
  // results | counter | team sync words | error flag | team partial sums
  const size_t res_bytes = (goff * sizeof(double) + 127) & ~size_t(127);
  const size_t sync_off = res_bytes + 128;
  const size_t err_off = sync_off + (((size_t)nteams * 4 * sizeof(unsigned) + 127) & ~size_t(127));
  const size_t part_off = err_off + 128;
  const size_t total = part_off + part * sizeof(double) + 128;
  if (qsv_status st = cuda_status(cudaMalloc(&b->plan, off), "batch plan")) return st;
  if (qsv_status st = cuda_status(cudaMalloc(&b->work, b->work_bytes), "batch workspace")) return st;
  if (qsv_status st = cuda_status(cudaMalloc(&b->results, total), "batch results")) return st;
  unsigned char* rb = reinterpret_cast<unsigned char*>(b->results);
  b->counter = reinterpret_cast<unsigned*>(rb + res_bytes);
  b->team_sync = reinterpret_cast<unsigned*>(rb + sync_off);
  b->error = reinterpret_cast<unsigned*>(rb + err_off);
  b->team_part = reinterpret_cast<double*>(rb + part_off);
  b->zero_bytes = total;
  return cuda_status(cudaMemcpy(b->plan, host.data(), off, cudaMemcpyHostToDevice), "batch plan upload");
}

template <typename V>
qsv_status launch_batch(qsv_batch_s* b, cudaStream_t stream) {
  constexpr int RF = fwd_bits<V>(), RB = bwd_bits<V>();
  unsigned char* p = static_cast<unsigned char*>(b->plan);
  BArgs a;
  a.jobs = reinterpret_cast<const BJob*>(p + b->off_jobs);
  a.njobs = b->njobs;
  a.stages = reinterpret_cast<const BStage*>(p + b->off_stages);
  a.passes = reinterpret_cast<const gx::GxPassDev*>(p + b->off_passes);
  a.ops = reinterpret_cast<const uint32_t*>(p + b->off_ops);
  a.coefs = p + b->off_coefs;
  a.runoff = reinterpret_cast<const uint64_t*>(p + b->off_runoff);
  a.groups = reinterpret_cast<const BGroup*>(p + b->off_groups);
  a.terms = reinterpret_cast<const BTerm*>(p + b->off_terms);
  a.red_slots = reinterpret_cast<const int32_t*>(p + b->off_red);
  a.work = b->work;
  a.work_stride = b->work_bytes > 256 ? b->work_bytes / sizeof(V) / b->blocks : 0;
  a.results = b->results;
  a.counter = b->counter;
  a.team_sync = b->team_sync;
  a.team_part = b->team_part;
  a.error = b->error;
  a.vec16 = 1;
  a.tile_elems = 1 << b->tile_bits;
  // zero the results (gradients accumulate), the work counter, the team
  // barriers and partial sums (one memset: they share one allocation)
  if (qsv_status st = cuda_status(cudaMemsetAsync(b->results, 0, b->zero_bytes, stream),
                                  "batch results reset"))
    return st;
  if (b->gen)
    k_batch<V, RF, RB, true><<<b->blocks, b->threads, b->smem, stream>>>(a);
  else
    k_batch<V, RF, RB, false><<<b->blocks, b->threads, b->smem, stream>>>(a);
  count_launch();
  return cuda_status(cudaGetLastError(), "batch kernel launch");
}

qsv_status launch_any(qsv_batch_s* b, cudaStream_t stream) {
  switch (b->dtype) {
    case QSV_C64: return launch_batch<float2>(b, stream);
    case QSV_C128: return launch_batch<double2>(b, stream);
    default: return fail(QSV_ERROR_DTYPE, "batched sweeps need a complex dtype");
  }
}

}  // namespace

extern "C" {

qsv_status qsv_batch_create(qsv_dtype dtype, int nCircuits, const int* nbQubits,
                            const qsv_gate* gates, const size_t* gate_offsets,
                            const char* paulis, const double* coefs, const size_t* term_offsets,
                            const int* nParams, const qsv_batch_opts* opts, qsv_batch* out) {
  if (!out) return fail(QSV_ERROR_INVALID_VALUE, "null output handle");
  *out = nullptr;
  if (nCircuits < 1 || !nbQubits || !gates || !gate_offsets || !term_offsets || !nParams)
    return fail(QSV_ERROR_INVALID_VALUE, "null or empty batch description");
  if (dtype != QSV_C64 && dtype != QSV_C128)
    return fail(QSV_ERROR_DTYPE, "batched sweeps need complex<float> or complex<double>");
  // term strings: circuit c's terms are nbQubits[c] characters each, back
  // to back, so circuit c starts at character char_off[c]
  std::vector<size_t> char_off(nCircuits + 1, 0);
  for (int c = 0; c < nCircuits; ++c)
    char_off[c + 1] = char_off[c] + (term_offsets[c + 1] - term_offsets[c]) * (size_t)nbQubits[c];
  if (char_off[nCircuits] && (!paulis || !coefs))
    return fail(QSV_ERROR_INVALID_VALUE, "null observable");
  auto* b = new qsv_batch_s();
  b->dtype = dtype;
  b->ncirc = nCircuits;
  const qsv_status st = (dtype == QSV_C64)
      ? build_batch<float2>(b, nCircuits, nbQubits, gates, gate_offsets, paulis, char_off.data(),
                            coefs, term_offsets, nParams, opts)
      : build_batch<double2>(b, nCircuits, nbQubits, gates, gate_offsets, paulis, char_off.data(),
                             coefs, term_offsets, nParams, opts);
  if (st) {
    qsv_batch_destroy(b);
    return st;
  }
  *out = b;
  return QSV_SUCCESS;
}

qsv_status qsv_batch_run(qsv_batch b, void* cuda_stream, int use_graph) {
  if (!b) return fail(QSV_ERROR_INVALID_VALUE, "null batch");
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  if (!use_graph) return launch_any(b, stream);
  if (!b->exec || b->captured_on != stream) {
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    cudaStream_t cap = stream;
    bool own = false;
    if (cap == nullptr) {  // the legacy stream cannot be captured
      if (qsv_status st = cuda_status(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking),
                                      "capture stream"))
        return st;
      own = true;
    }
    if (qsv_status st = cuda_status(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal),
                                    "batch graph capture"))
      return st;
    qsv_status lst = launch_any(b, cap);
    cudaGraph_t g = nullptr;
    qsv_status est = cuda_status(cudaStreamEndCapture(cap, &g), "batch graph end capture");
    if (lst || est) {
      if (g) cudaGraphDestroy(g);
      if (own) cudaStreamDestroy(cap);
      return lst ? lst : est;
    }
    b->graph = g;
    if (qsv_status st = cuda_status(cudaGraphInstantiate(&b->exec, g, 0), "batch graph instantiate")) {
      if (own) cudaStreamDestroy(cap);
      return st;
    }
    if (own) cudaStreamDestroy(cap);
    b->captured_on = stream;
  }
  count_launch();
  return cuda_status(cudaGraphLaunch(b->exec, stream), "batch graph launch");
}

qsv_status qsv_batch_results(qsv_batch b, void* cuda_stream, double* energies, double* grads) {
  if (!b) return fail(QSV_ERROR_INVALID_VALUE, "null batch");
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  std::vector<double> host(b->nresults);
  if (qsv_status st = cuda_status(cudaMemcpyAsync(host.data(), b->results,
                                                  b->nresults * sizeof(double),
                                                  cudaMemcpyDeviceToHost, stream), "batch results copy"))
    return st;
  unsigned err = 0;
  if (qsv_status st = cuda_status(cudaMemcpyAsync(&err, b->error, sizeof(err),
                                                  cudaMemcpyDeviceToHost, stream),
                                  "batch error flag copy"))
    return st;
  if (qsv_status st = cuda_status(cudaStreamSynchronize(stream), "batch results synchronize"))
    return st;
  if (err)
    return fail(QSV_ERROR_TIMEOUT, "a team of the batch gave up waiting at a barrier "
                                   "(results invalid)");
  if (energies) std::memcpy(energies, host.data(), b->ncirc * sizeof(double));
  if (grads && b->nresults > (size_t)b->ncirc)
    std::memcpy(grads, host.data() + b->ncirc, (b->nresults - b->ncirc) * sizeof(double));
  return QSV_SUCCESS;
}

qsv_status qsv_batch_info(qsv_batch b, int* blocks, int* threads, int* tile_bits,
                          size_t* workspace_bytes) {
  if (!b) return fail(QSV_ERROR_INVALID_VALUE, "null batch");
  if (blocks) *blocks = b->blocks;
  if (threads) *threads = b->threads;
  if (tile_bits) *tile_bits = b->tile_bits;
  if (workspace_bytes) *workspace_bytes = b->work_bytes;
  return QSV_SUCCESS;
}

qsv_status qsv_batch_work(qsv_batch b, double* global_bytes, double* amplitude_updates) {
  if (!b) return fail(QSV_ERROR_INVALID_VALUE, "null batch");
  if (global_bytes) *global_bytes = b->global_bytes;
  if (amplitude_updates) *amplitude_updates = b->amp_updates;
  return QSV_SUCCESS;
}

qsv_status qsv_batch_destroy(qsv_batch b) {
  if (!b) return QSV_SUCCESS;
  cudaDeviceSynchronize();
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->plan) cudaFree(b->plan);
  if (b->work) cudaFree(b->work);
  if (b->results) cudaFree(b->results);
  delete b;
  return QSV_SUCCESS;
}

}  // extern "C"

// FP64 reductions over state vectors: norm, inner product, Pauli-sum
// expectation values, and the application of a Pauli-sum observable.
//
// QCLAB++ has no observables; these follow the plain definitions
//   <psi|P|psi> = sum_j conj(psi_j) (P psi)_j,
//   (P psi)_j   = i^{ny} (-1)^{popcount((j ^ f) & zy)} psi_{j ^ f}
// for a Pauli string with X/Y on the flip mask f, Y/Z on zy and ny Y's
// (Y|b> = i (-1)^b |1-b>).  Every sum is formed in double precision with a
// fixed-order two-stage reduction (per-CTA partials, then one block), so a
// repeated call returns the same bits.
//
// Terms are evaluated tile by tile (tile.cuh): terms whose flip bits fit in
// one m-bit tile set S are grouped, each group is one pass over the state,
// and every partner amplitude psi_{j^f} is read from shared memory.
#include <algorithm>
#include <cstring>
#include <vector>
#include "internal.hpp"
#include "tile.cuh"

namespace qsv {
namespace {

__host__ __device__ inline size_t fx_align16(size_t b) { return (b + 15) & ~size_t(15); }

constexpr int kRedThreads = 512;
constexpr int kRedBlocks = 148 * 8;

struct DTerm {
  uint32_t flip_local;
  uint32_t zy_local;  // the tile bits of zy, as local bits (tiled groups)
  uint64_t flip;   // global flip mask
  uint64_t zy;     // global sign mask
  double wr, wi;   // coef * i^ny
};

// A term as a tile group's kernels stage it in shared memory: its sign on
// the tile's fixed bits, parity((base ^ flip) & zy), folded into the weight,
// so the sign of local element e is that weight times (-1)^popc(e & zy_local)
// -- no global index per element and term.
struct STerm {
  uint32_t flip_local, zy_local;
  double wr, wi;
};

__device__ __forceinline__ void stage_terms(STerm* ts, const DTerm* __restrict__ terms, int nterms,
                                            uint64_t base) {
  for (int t = threadIdx.x; t < nterms; t += blockDim.x) {
    const DTerm T = terms[t];
    const bool odd = __popcll((base ^ T.flip) & T.zy) & 1;
    ts[t] = STerm{T.flip_local, T.zy_local, odd ? -T.wr : T.wr, odd ? -T.wi : T.wi};
  }
}

template <typename V>
__global__ void __launch_bounds__(kRedThreads)
k_norm2(const V* __restrict__ st, uint64_t N, double2* __restrict__ partial) {
  __shared__ double2 red[32];
  double acc = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 v = to_d2(st[i]);
    acc = fma(v.x, v.x, fma(v.y, v.y, acc));
  }
  const double2 s = block_sum(make_double2(acc, 0.0), red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

template <typename V>
__global__ void __launch_bounds__(kRedThreads)
k_inner(const V* __restrict__ a, const V* __restrict__ b, uint64_t N, double2* __restrict__ partial) {
  __shared__ double2 red[32];
  double2 acc = make_double2(0.0, 0.0);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 x = to_d2(a[i]), y = to_d2(b[i]);
    // conj(x) * y
    acc.x = fma(x.x, y.x, fma(x.y, y.y, acc.x));
    acc.y = fma(x.x, y.y, fma(-x.y, y.x, acc.y));
  }
  const double2 s = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// x *= s (s formed in FP64, applied in the element's precision)
template <typename V>
__global__ void __launch_bounds__(kRedThreads)
k_scale_real(V* __restrict__ st, uint64_t N, double s) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
       i += (uint64_t)gridDim.x * blockDim.x)
    st[i] = from_d2<V>(make_double2(to_d2(st[i]).x * s, to_d2(st[i]).y * s));
}

// Fixed-order sum of `count` partials by one block.
__global__ void __launch_bounds__(1024)
k_final(const double2* __restrict__ partial, int count, double2* __restrict__ out) {
  __shared__ double2 red[32];
  double2 acc = make_double2(0.0, 0.0);
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    acc.x += partial[i].x;
    acc.y += partial[i].y;
  }
  const double2 s = block_sum(acc, red);
  if (threadIdx.x == 0) *out = s;
}

__device__ __forceinline__ double sgn_of(uint64_t x) {
  return (__popcll(x) & 1) ? -1.0 : 1.0;
}

// Signed weight sum of a group's first ndiag terms (those without flip bits,
// Z-strings): S(e) = sum_t w_t (-1)^popc(e & zy_t), so that they contribute
// S(e) |x_e|^2 (expectation) or S(e) x_e (observable) with one product.
__device__ __forceinline__ double2 diag_weight(const STerm* ts, int ndiag, uint32_t e) {
  double sr = 0.0, si = 0.0;
  for (int t = 0; t < ndiag; ++t) {
    const STerm& T = ts[t];
    const bool odd = __popc(e & T.zy_local) & 1;
    sr += odd ? -T.wr : T.wr;
    si += odd ? -T.wi : T.wi;
  }
  return make_double2(sr, si);
}

// sum_t w_t sum_{j in tile} conj(psi_j) (-1)^{pop((j^f)&zy)} psi_{j^f}; the
// group's first ndiag terms have no flip bits
template <typename V>
__global__ void __launch_bounds__(kRedThreads)
k_expect(const V* __restrict__ st, TileArgs ta, const DTerm* __restrict__ terms, int nterms,
         int ndiag, double2* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* tile = reinterpret_cast<V*>(smem_raw);
  const uint32_t size = 1u << ta.m;
  STerm* ts = reinterpret_cast<STerm*>(smem_raw + fx_align16(size_t(size) * sizeof(V)));
  __shared__ double2 red[32];
  const uint64_t base = tile_base(ta, blockIdx.x);
  for (uint32_t e = threadIdx.x; e < size; e += blockDim.x)
    tile[e] = st[tile_global(ta, ta.runoff, base, e)];
  stage_terms(ts, terms, nterms, base);
  __syncthreads();
  // sum_t w_t sum_e conj(x_e) (-1)^popc(e & zy_t) x_{e ^ f_t}
  double2 acc = make_double2(0.0, 0.0);
  for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) {
    const double2 x = to_d2(tile[e]);
    if (ndiag > 0) {
      const double2 S = diag_weight(ts, ndiag, e);
      const double p = fma(x.x, x.x, x.y * x.y);
      acc.x = fma(S.x, p, acc.x);
      acc.y = fma(S.y, p, acc.y);
    }
    for (int t = ndiag; t < nterms; ++t) {
      const STerm T = ts[t];
      const double2 y = to_d2(tile[e ^ T.flip_local]);
      const double re = fma(x.x, y.x, x.y * y.y), im = fma(x.x, y.y, -x.y * y.x);
      const double sg = (__popc(e & T.zy_local) & 1) ? -1.0 : 1.0;
      acc.x = fma(sg * T.wr, re, fma(-sg * T.wi, im, acc.x));
      acc.y = fma(sg * T.wr, im, fma(sg * T.wi, re, acc.y));
    }
  }
  const double2 r = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

// dst (+)= sum_t w_t P_t src over one tile group (first ndiag terms without
// flip bits)
template <typename V>
__global__ void __launch_bounds__(kRedThreads)
k_observable(const V* __restrict__ src, V* __restrict__ dst, TileArgs ta,
             const DTerm* __restrict__ terms, int nterms, int ndiag, int accumulate) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* tile = reinterpret_cast<V*>(smem_raw);
  const uint32_t size = 1u << ta.m;
  STerm* ts = reinterpret_cast<STerm*>(smem_raw + fx_align16(size_t(size) * sizeof(V)));
  const uint64_t base = tile_base(ta, blockIdx.x);
  for (uint32_t e = threadIdx.x; e < size; e += blockDim.x)
    tile[e] = src[tile_global(ta, ta.runoff, base, e)];
  stage_terms(ts, terms, nterms, base);
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) {
    const uint64_t g = tile_global(ta, ta.runoff, base, e);
    double2 acc = accumulate ? to_d2(dst[g]) : make_double2(0.0, 0.0);
    if (ndiag > 0) {
      const double2 S = diag_weight(ts, ndiag, e);
      const double2 x = to_d2(tile[e]);
      acc.x = fma(S.x, x.x, fma(-S.y, x.y, acc.x));
      acc.y = fma(S.x, x.y, fma(S.y, x.x, acc.y));
    }
    for (int t = ndiag; t < nterms; ++t) {
      const STerm T = ts[t];
      const double2 y = to_d2(tile[e ^ T.flip_local]);
      const double sg = (__popc(e & T.zy_local) & 1) ? -1.0 : 1.0;
      acc.x = fma(sg * T.wr, y.x, fma(-sg * T.wi, y.y, acc.x));
      acc.y = fma(sg * T.wr, y.y, fma(sg * T.wi, y.x, acc.y));
    }
    dst[g] = from_d2<V>(acc);
  }
}

// Terms whose flip bits do not fit in a tile (|f | low bits| > m) are
// evaluated against global memory: the partner psi_{j^f} of consecutive j
// stays inside the same aligned 2^low block, so the reads remain coalesced.
template <typename V>
__global__ void __launch_bounds__(kRedThreads)
k_expect_wide(const V* __restrict__ st, uint64_t N, DTerm T, double2* __restrict__ partial) {
  __shared__ double2 red[32];
  double2 s = make_double2(0.0, 0.0);
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < N;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const double2 x = to_d2(st[j]);
    const double2 y = to_d2(st[j ^ T.flip]);
    const double sg = sgn_of((j ^ T.flip) & T.zy);
    s.x = fma(sg * x.x, y.x, fma(sg * x.y, y.y, s.x));
    s.y = fma(sg * x.x, y.y, fma(-sg * x.y, y.x, s.y));
  }
  const double2 acc = make_double2(T.wr * s.x - T.wi * s.y, T.wr * s.y + T.wi * s.x);
  const double2 r = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

template <typename V>
__global__ void __launch_bounds__(kRedThreads)
k_observable_wide(const V* __restrict__ src, V* __restrict__ dst, uint64_t N, DTerm T,
                  int accumulate) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < N;
       j += (uint64_t)gridDim.x * blockDim.x) {
    double2 acc = accumulate ? to_d2(dst[j]) : make_double2(0.0, 0.0);
    const double2 y = to_d2(src[j ^ T.flip]);
    const double sg = sgn_of((j ^ T.flip) & T.zy);
    acc.x = fma(sg * T.wr, y.x, fma(-sg * T.wi, y.y, acc.x));
    acc.y = fma(sg * T.wr, y.y, fma(sg * T.wi, y.x, acc.y));
    dst[j] = from_d2<V>(acc);
  }
}

struct HTerm {
  uint64_t flip, zy;
  int ny;
  double coef;
};

qsv_status parse_terms(int n, const char* paulis, const double* coefs, size_t nterms,
                       std::vector<HTerm>* out) {
  if (nterms && (!paulis || !coefs)) return fail(QSV_ERROR_INVALID_VALUE, "null observable");
  out->clear();
  for (size_t t = 0; t < nterms; ++t) {
    HTerm h{0, 0, 0, coefs[t]};
    for (int q = 0; q < n; ++q) {
      const char c = paulis[t * (size_t)n + q];
      const uint64_t b = 1ull << (n - 1 - q);
      switch (c) {
        case 'I': case 'i': break;
        case 'X': case 'x': h.flip |= b; break;
        case 'Y': case 'y': h.flip |= b; h.zy |= b; ++h.ny; break;
        case 'Z': case 'z': h.zy |= b; break;
        default:
          return fail(QSV_ERROR_INVALID_VALUE, "term %zu: '%c' is not one of I, X, Y, Z", t, c);
      }
    }
    out->push_back(h);
  }
  return QSV_SUCCESS;
}

struct Group {
  int bits[64];
  int m;
  std::vector<int> terms;
};

// Greedy grouping of terms so that each group's flip bits fit one tile
// (low bits included, at most m bits).  Terms that cannot fit go to `wide`.
std::vector<Group> group_terms(const std::vector<HTerm>& T, int n, int m, int low,
                               std::vector<int>* wide) {
  std::vector<int> order;
  for (int i = 0; i < (int)T.size(); ++i) order.push_back(i);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return T[a].flip < T[b].flip; });
  const uint64_t lowmask = (1ull << low) - 1ull;
  std::vector<uint64_t> sets;
  std::vector<std::vector<int>> members;
  wide->clear();
  for (int i : order) {
    const uint64_t f = T[i].flip;
    if (__builtin_popcountll(lowmask | f) > m) {
      wide->push_back(i);
      continue;
    }
    bool placed = false;
    for (size_t g = 0; g < sets.size() && !placed; ++g) {
      if (__builtin_popcountll(sets[g] | f) <= m) {
        sets[g] |= f;
        members[g].push_back(i);
        placed = true;
      }
    }
    if (!placed) {
      sets.push_back(lowmask | f);
      members.push_back({i});
    }
  }
  std::vector<Group> out;
  for (size_t g = 0; g < sets.size(); ++g) {
    Group G;
    G.m = tile_bits_of(sets[g], n, m, G.bits);
    G.terms = members[g];
    out.push_back(G);
  }
  return out;
}

template <typename V>
qsv_status run_tiled(qsv_state_s* s, const V* src, V* dst, const std::vector<HTerm>& T,
                     bool expect, double* out_re) {
  const int n = s->n;
  int m = std::min(n, sizeof(V) >= 16 ? 12 : 13);
  int low = std::min(m, sizeof(V) >= 16 ? 4 : 5);
  if (T.empty()) {
    if (expect) *out_re = 0.0;
    else if (dst) return cuda_status(cudaMemsetAsync(dst, 0, dim(n) * sizeof(V), s->stream), "memset");
    return QSV_SUCCESS;
  }
  std::vector<int> wide;
  std::vector<Group> groups = group_terms(T, n, m, low, &wide);
  for (const Group& G : groups)
    if (G.m != m) return fail(QSV_ERROR_INVALID_VALUE, "internal: term group of %d bits", G.m);
  const uint64_t N = dim(n);
  const uint64_t ntiles = 1ull << (n - m);
  const int nruns = 1 << (m - low);
  const unsigned wblocks =
      (unsigned)std::min<uint64_t>(kRedBlocks, (N + kRedThreads - 1) / kRedThreads);
  const size_t nparts = ntiles * groups.size() + (size_t)wblocks * wide.size();
  // scratch layout: [partials double2][out double2][terms][runoffs]
  const size_t part_bytes = expect ? nparts * sizeof(double2) : 0;
  const size_t out_off = part_bytes;
  const size_t term_off = (out_off + sizeof(double2) + 255) & ~size_t(255);
  const size_t term_bytes = T.size() * sizeof(DTerm);
  const size_t run_off = (term_off + term_bytes + 255) & ~size_t(255);
  const size_t total = run_off + groups.size() * nruns * sizeof(uint64_t);
  if (qsv_status st = ensure_scratch(s, total)) return st;
  unsigned char* dev = static_cast<unsigned char*>(s->scratch);

  std::vector<DTerm> dt;
  std::vector<uint64_t> runoffs;
  std::vector<size_t> term0;
  std::vector<int> ndiag;
  for (const Group& G : groups) {
    int local_of[64];
    for (int j = 0; j < 64; ++j) local_of[j] = -1;
    for (int j = 0; j < G.m; ++j) local_of[G.bits[j]] = j;
    term0.push_back(dt.size());
    // terms without flip bits first (their contributions share one product)
    std::vector<int> order;
    for (int ti : G.terms)
      if (T[ti].flip == 0) order.push_back(ti);
    ndiag.push_back((int)order.size());
    for (int ti : G.terms)
      if (T[ti].flip != 0) order.push_back(ti);
    for (int ti : order) {
      const HTerm& h = T[ti];
      DTerm d{};
      for (int b = 0; b < n; ++b) {
        if ((h.flip >> b) & 1ull) d.flip_local |= 1u << local_of[b];
        if (((h.zy >> b) & 1ull) && local_of[b] >= 0) d.zy_local |= 1u << local_of[b];
      }
      d.flip = h.flip;
      d.zy = h.zy;
      // coef * i^ny
      static const double pr[4] = {1, 0, -1, 0}, pi[4] = {0, 1, 0, -1};
      d.wr = h.coef * pr[h.ny & 3];
      d.wi = h.coef * pi[h.ny & 3];
      dt.push_back(d);
    }
    tile_runoffs(G.bits, G.m, low, &runoffs);
  }
  std::vector<DTerm> wt;
  for (int ti : wide) {
    const HTerm& h = T[ti];
    static const double pr[4] = {1, 0, -1, 0}, pi[4] = {0, 1, 0, -1};
    DTerm d{};
    d.flip = h.flip;
    d.zy = h.zy;
    d.wr = h.coef * pr[h.ny & 3];
    d.wi = h.coef * pi[h.ny & 3];
    wt.push_back(d);
  }
  if (runoffs.size() != groups.size() * (size_t)nruns)
    return fail(QSV_ERROR_INVALID_VALUE, "internal: run table size");
  std::vector<unsigned char> host(total - term_off);
  std::memcpy(host.data(), dt.data(), dt.size() * sizeof(DTerm));
  std::memcpy(host.data() + (run_off - term_off), runoffs.data(), runoffs.size() * 8);
  if (qsv_status st = cuda_status(cudaMemcpyAsync(dev + term_off, host.data(), host.size(),
                                                  cudaMemcpyHostToDevice, s->stream),
                                  "observable upload"))
    return st;
  size_t max_terms = 0;
  for (const Group& G : groups) max_terms = std::max(max_terms, G.terms.size());
  const size_t smem = fx_align16((size_t(1) << m) * sizeof(V)) + max_terms * sizeof(STerm);
  if (smem > 200 * 1024)
    return fail(QSV_ERROR_SIZE, "observable group of %zu terms exceeds shared memory", max_terms);
  auto kern_e = k_expect<V>;
  auto kern_o = k_observable<V>;
  if (qsv_status st = cuda_status(cudaFuncSetAttribute(expect ? (const void*)kern_e : (const void*)kern_o,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)smem), "reduction smem attribute"))
    return st;
  const int threads = std::min<int>(kRedThreads, std::max<int>(32, (1 << m) / 8));
  double2* partial = reinterpret_cast<double2*>(dev);
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    TileArgs ta;
    ta.n = n;
    ta.m = groups[gi].m;
    ta.low = low;
    for (int j = 0; j < 64; ++j) ta.bits[j] = (j < ta.m) ? (int8_t)groups[gi].bits[j] : 0;
    ta.runoff = reinterpret_cast<const uint64_t*>(dev + run_off) + gi * nruns;
    const DTerm* terms = reinterpret_cast<const DTerm*>(dev + term_off) + term0[gi];
    const int nt = (int)groups[gi].terms.size();
    if (expect)
      k_expect<V><<<(unsigned)ntiles, threads, smem, s->stream>>>(src, ta, terms, nt, ndiag[gi],
                                                                 partial + gi * ntiles);
    else
      k_observable<V><<<(unsigned)ntiles, threads, smem, s->stream>>>(src, dst, ta, terms, nt,
                                                                      ndiag[gi], gi > 0 ? 1 : 0);
    count_launch();
    if (qsv_status st = cuda_status(cudaGetLastError(), "tiled reduction launch")) return st;
  }
  for (size_t wi = 0; wi < wt.size(); ++wi) {
    if (expect)
      k_expect_wide<V><<<wblocks, kRedThreads, 0, s->stream>>>(
          src, N, wt[wi], partial + ntiles * groups.size() + wi * wblocks);
    else
      k_observable_wide<V><<<wblocks, kRedThreads, 0, s->stream>>>(
          src, dst, N, wt[wi], (groups.size() + wi) > 0 ? 1 : 0);
    count_launch();
    if (qsv_status st = cuda_status(cudaGetLastError(), "wide-term launch")) return st;
  }
  if (!expect) return QSV_SUCCESS;
  double2* dout = reinterpret_cast<double2*>(dev + out_off);
  k_final<<<1, 1024, 0, s->stream>>>(partial, (int)nparts, dout);
  count_launch();
  if (qsv_status st = cuda_status(cudaGetLastError(), "final reduction launch")) return st;
  double2 h;
  if (qsv_status st = cuda_status(cudaMemcpyAsync(&h, dout, sizeof(h), cudaMemcpyDeviceToHost,
                                                  s->stream), "reduction result copy"))
    return st;
  if (qsv_status st = cuda_status(cudaStreamSynchronize(s->stream), "reduction synchronize"))
    return st;
  *out_re = h.x;
  return QSV_SUCCESS;
}

template <typename V>
qsv_status norm2_typed(qsv_state_s* s, double* out) {
  const uint64_t N = dim(s->n);
  const unsigned blocks = (unsigned)std::min<uint64_t>(kRedBlocks, (N + kRedThreads - 1) / kRedThreads);
  if (qsv_status st = ensure_scratch(s, (blocks + 1) * sizeof(double2))) return st;
  double2* partial = static_cast<double2*>(s->scratch);
  k_norm2<V><<<blocks, kRedThreads, 0, s->stream>>>(static_cast<const V*>(s->d), N, partial);
  k_final<<<1, 1024, 0, s->stream>>>(partial, (int)blocks, partial + blocks);
  count_launch(2);
  if (qsv_status st = cuda_status(cudaGetLastError(), "norm launch")) return st;
  double2 h;
  if (qsv_status st = cuda_status(cudaMemcpyAsync(&h, partial + blocks, sizeof(h),
                                                  cudaMemcpyDeviceToHost, s->stream), "norm copy"))
    return st;
  if (qsv_status st = cuda_status(cudaStreamSynchronize(s->stream), "norm synchronize")) return st;
  *out = h.x;
  return QSV_SUCCESS;
}

template <typename V>
qsv_status inner_typed(qsv_state_s* a, qsv_state_s* b, double* out) {
  const uint64_t N = dim(a->n);
  const unsigned blocks = (unsigned)std::min<uint64_t>(kRedBlocks, (N + kRedThreads - 1) / kRedThreads);
  if (qsv_status st = ensure_scratch(a, (blocks + 1) * sizeof(double2))) return st;
  double2* partial = static_cast<double2*>(a->scratch);
  k_inner<V><<<blocks, kRedThreads, 0, a->stream>>>(static_cast<const V*>(a->d),
                                                    static_cast<const V*>(b->d), N, partial);
  k_final<<<1, 1024, 0, a->stream>>>(partial, (int)blocks, partial + blocks);
  count_launch(2);
  if (qsv_status st = cuda_status(cudaGetLastError(), "inner launch")) return st;
  double2 h;
  if (qsv_status st = cuda_status(cudaMemcpyAsync(&h, partial + blocks, sizeof(h),
                                                  cudaMemcpyDeviceToHost, a->stream), "inner copy"))
    return st;
  if (qsv_status st = cuda_status(cudaStreamSynchronize(a->stream), "inner synchronize")) return st;
  out[0] = h.x;
  out[1] = h.y;
  return QSV_SUCCESS;
}

qsv_status check(qsv_state s) {
  if (!s || !s->d) return fail(QSV_ERROR_INVALID_VALUE, "null state");
  return QSV_SUCCESS;
}

// <a|b> and max |a_j - b_j| for states of possibly different element types.
template <typename VA, typename VB>
__global__ void __launch_bounds__(kRedThreads)
k_compare(const VA* __restrict__ a, const VB* __restrict__ b, uint64_t N,
          double2* __restrict__ partial, double* __restrict__ pmax) {
  __shared__ double2 red[32];
  __shared__ double mx[32];
  double2 acc = make_double2(0.0, 0.0);
  double m = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 x = to_d2(a[i]), y = to_d2(b[i]);
    acc.x = fma(x.x, y.x, fma(x.y, y.y, acc.x));
    acc.y = fma(x.x, y.y, fma(-x.y, y.x, acc.y));
    const double dx = x.x - y.x, dy = x.y - y.y;
    m = fmax(m, sqrt(fma(dx, dx, dy * dy)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) mx[threadIdx.x >> 5] = m;
  const double2 s = block_sum(acc, red);  // synchronises the block
  if (threadIdx.x == 0) {
    double bm = 0.0;
    for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) bm = fmax(bm, mx[w]);
    partial[blockIdx.x] = s;
    pmax[blockIdx.x] = bm;
  }
}

__global__ void k_max(const double* __restrict__ v, int count, double* __restrict__ out) {
  __shared__ double mx[32];
  double m = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) m = fmax(m, v[i]);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) mx[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double bm = 0.0;
    for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) bm = fmax(bm, mx[w]);
    *out = bm;
  }
}

template <typename VA, typename VB>
qsv_status compare_typed(qsv_state_s* a, qsv_state_s* b, double* out) {
  const uint64_t N = dim(a->n);
  const unsigned blocks = (unsigned)std::min<uint64_t>(kRedBlocks, (N + kRedThreads - 1) / kRedThreads);
  const size_t bytes = (blocks + 1) * sizeof(double2) + (blocks + 1) * sizeof(double);
  if (qsv_status st = ensure_scratch(a, bytes)) return st;
  double2* partial = static_cast<double2*>(a->scratch);
  double* pmax = reinterpret_cast<double*>(partial + blocks + 1);
  k_compare<VA, VB><<<blocks, kRedThreads, 0, a->stream>>>(
      static_cast<const VA*>(a->d), static_cast<const VB*>(b->d), N, partial, pmax);
  k_final<<<1, 1024, 0, a->stream>>>(partial, (int)blocks, partial + blocks);
  k_max<<<1, 1024, 0, a->stream>>>(pmax, (int)blocks, pmax + blocks);
  count_launch(3);
  if (qsv_status st = cuda_status(cudaGetLastError(), "compare launch")) return st;
  double2 h;
  double hm;
  if (qsv_status st = cuda_status(cudaMemcpyAsync(&h, partial + blocks, sizeof(h),
                                                  cudaMemcpyDeviceToHost, a->stream), "compare copy"))
    return st;
  if (qsv_status st = cuda_status(cudaMemcpyAsync(&hm, pmax + blocks, sizeof(hm),
                                                  cudaMemcpyDeviceToHost, a->stream), "compare copy"))
    return st;
  if (qsv_status st = cuda_status(cudaStreamSynchronize(a->stream), "compare synchronize")) return st;
  out[0] = h.x;
  out[1] = h.y;
  out[2] = hm;
  return QSV_SUCCESS;
}

template <typename VA>
qsv_status compare_b(qsv_state_s* a, qsv_state_s* b, double* out) {
  switch (b->dtype) {
    case QSV_C128: return compare_typed<VA, double2>(a, b, out);
    case QSV_C64:  return compare_typed<VA, float2>(a, b, out);
    case QSV_F64:  return compare_typed<VA, double>(a, b, out);
    case QSV_F32:  return compare_typed<VA, float>(a, b, out);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

qsv_status compare_dispatch(qsv_state_s* a, qsv_state_s* b, double* out) {
  switch (a->dtype) {
    case QSV_C128: return compare_b<double2>(a, b, out);
    case QSV_C64:  return compare_b<float2>(a, b, out);
    case QSV_F64:  return compare_b<double>(a, b, out);
    case QSV_F32:  return compare_b<float>(a, b, out);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

}  // namespace

qsv_status expectation_internal(qsv_state_s* s, const char* paulis, const double* coefs,
                                size_t nterms, double* out) {
  std::vector<HTerm> T;
  if (qsv_status st = parse_terms(s->n, paulis, coefs, nterms, &T)) return st;
  switch (s->dtype) {
    case QSV_C128: return run_tiled<double2>(s, (const double2*)s->d, nullptr, T, true, out);
    case QSV_C64:  return run_tiled<float2>(s, (const float2*)s->d, nullptr, T, true, out);
    case QSV_F64:  return run_tiled<double>(s, (const double*)s->d, nullptr, T, true, out);
    case QSV_F32:  return run_tiled<float>(s, (const float*)s->d, nullptr, T, true, out);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

qsv_status inner_internal(qsv_state_s* a, qsv_state_s* b, double* out) {
  switch (a->dtype) {
    case QSV_C128: return inner_typed<double2>(a, b, out);
    case QSV_C64:  return inner_typed<float2>(a, b, out);
    case QSV_F64:  return inner_typed<double>(a, b, out);
    case QSV_F32:  return inner_typed<float>(a, b, out);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

qsv_status observable_internal(qsv_state_s* dst, qsv_state_s* src, const char* paulis,
                               const double* coefs, size_t nterms) {
  std::vector<HTerm> T;
  if (qsv_status st = parse_terms(src->n, paulis, coefs, nterms, &T)) return st;
  if (dtype_real(src->dtype))
    for (const HTerm& h : T)
      if (h.ny & 1) return fail(QSV_ERROR_DTYPE, "a term with an odd number of Y is imaginary on a real state");
  switch (src->dtype) {
    case QSV_C128: return run_tiled<double2>(src, (const double2*)src->d, (double2*)dst->d, T, false, nullptr);
    case QSV_C64:  return run_tiled<float2>(src, (const float2*)src->d, (float2*)dst->d, T, false, nullptr);
    case QSV_F64:  return run_tiled<double>(src, (const double*)src->d, (double*)dst->d, T, false, nullptr);
    case QSV_F32:  return run_tiled<float>(src, (const float*)src->d, (float*)dst->d, T, false, nullptr);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

}  // namespace qsv

using namespace qsv;

extern "C" {

qsv_status qsv_norm2(qsv_state s, double* out) {
  if (qsv_status st = check(s)) return st;
  if (!out) return fail(QSV_ERROR_INVALID_VALUE, "null output");
  switch (s->dtype) {
    case QSV_C128: return norm2_typed<double2>(s, out);
    case QSV_C64:  return norm2_typed<float2>(s, out);
    case QSV_F64:  return norm2_typed<double>(s, out);
    case QSV_F32:  return norm2_typed<float>(s, out);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

qsv_status qsv_normalize(qsv_state s, double* norm2_out) {
  double nrm = 0.0;
  if (qsv_status st = qsv_norm2(s, &nrm)) return st;
  if (norm2_out) *norm2_out = nrm;
  if (!(nrm > 0.0)) return fail(QSV_ERROR_INVALID_VALUE, "cannot normalise a zero state");
  const double inv = 1.0 / std::sqrt(nrm);
  const uint64_t N = dim(s->n);
  const unsigned blocks = (unsigned)std::min<uint64_t>(kRedBlocks, (N + kRedThreads - 1) / kRedThreads);
  switch (s->dtype) {
    case QSV_C128: k_scale_real<double2><<<blocks, kRedThreads, 0, s->stream>>>((double2*)s->d, N, inv); break;
    case QSV_C64:  k_scale_real<float2><<<blocks, kRedThreads, 0, s->stream>>>((float2*)s->d, N, inv); break;
    case QSV_F64:  k_scale_real<double><<<blocks, kRedThreads, 0, s->stream>>>((double*)s->d, N, inv); break;
    case QSV_F32:  k_scale_real<float><<<blocks, kRedThreads, 0, s->stream>>>((float*)s->d, N, inv); break;
  }
  count_launch();
  return cuda_status(cudaGetLastError(), "normalise launch");
}

qsv_status qsv_inner(qsv_state a, qsv_state b, double* out) {
  if (qsv_status st = check(a)) return st;
  if (qsv_status st = check(b)) return st;
  if (!out) return fail(QSV_ERROR_INVALID_VALUE, "null output");
  if (a->n != b->n || a->dtype != b->dtype)
    return fail(QSV_ERROR_SIZE, "qsv_inner: states differ in size or dtype");
  if (b->stream != a->stream) {
    // order b's pending work before the reduction on a's stream
    if (qsv_status st = cuda_status(cudaStreamSynchronize(b->stream), "inner stream sync")) return st;
  }
  switch (a->dtype) {
    case QSV_C128: return inner_typed<double2>(a, b, out);
    case QSV_C64:  return inner_typed<float2>(a, b, out);
    case QSV_F64:  return inner_typed<double>(a, b, out);
    case QSV_F32:  return inner_typed<float>(a, b, out);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

qsv_status qsv_expectation(qsv_state s, const char* paulis, const double* coefs, size_t nterms,
                           double* out) {
  if (qsv_status st = check(s)) return st;
  if (!out) return fail(QSV_ERROR_INVALID_VALUE, "null output");
  return expectation_internal(s, paulis, coefs, nterms, out);
}

qsv_status qsv_compare(qsv_state a, qsv_state b, double* out) {
  if (qsv_status st = check(a)) return st;
  if (qsv_status st = check(b)) return st;
  if (!out) return fail(QSV_ERROR_INVALID_VALUE, "null output");
  if (a->n != b->n) return fail(QSV_ERROR_SIZE, "qsv_compare: states differ in size");
  if (b->stream != a->stream)
    if (qsv_status st = cuda_status(cudaStreamSynchronize(b->stream), "compare stream sync"))
      return st;
  return compare_dispatch(a, b, out);
}

qsv_status qsv_apply_observable(qsv_state dst, qsv_state src, const char* paulis,
                                const double* coefs, size_t nterms) {
  if (qsv_status st = check(dst)) return st;
  if (qsv_status st = check(src)) return st;
  if (dst == src || dst->d == src->d)
    return fail(QSV_ERROR_INVALID_VALUE, "qsv_apply_observable needs distinct states");
  if (dst->n != src->n || dst->dtype != src->dtype)
    return fail(QSV_ERROR_SIZE, "states differ in size or dtype");
  // dst is written on src's stream: after dst's pending work, and dst's
  // later work waits for the write
  if (qsv_status st = stream_wait(src->stream, dst->stream)) return st;
  if (qsv_status st = observable_internal(dst, src, paulis, coefs, nterms)) return st;
  return stream_wait(dst->stream, src->stream);
}

}  // extern "C"

// ---- allocation-free expectation value --------------------------------------
//
// qsv_expectation_noalloc: the tiled expectation value above, for callers
// that cannot allocate device memory.  Its work memory (term table, run
// offsets, per-CTA partial sums, result) is the file-scope array below; the
// CTAs loop over the tiles so the partial sums stay bounded whatever the
// state size.
#include <mutex>

namespace qsv {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(1) << 20;  // 1 MiB per device
constexpr unsigned kNoAllocBlocks = 148 * 4;
constexpr int kNoAllocMaxDevices = 64;

// Held by every GPU that loads this library, until process exit.  In host
// code this name is only a stand-in for the symbol; kernels get the device
// address obtained with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up on
// the first call per device (that device current).
qsv_status noalloc_scratch(void** out) {
  int dev = 0;
  if (qsv_status st = cuda_status(cudaGetDevice(&dev), "cudaGetDevice")) return st;
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return fail(QSV_ERROR_NOT_SUPPORTED, "device ordinal %d beyond %d", dev, kNoAllocMaxDevices);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    if (qsv_status st = cuda_status(cudaGetSymbolAddress(&p, g_noalloc_scratch),
                                    "cudaGetSymbolAddress(no-alloc scratch)"))
      return st;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return QSV_SUCCESS;
}

// k_expect with the CTAs striding over tiles: one partial per CTA.
template <typename V>
__global__ void __launch_bounds__(kRedThreads)
k_expect_tiles(const V* __restrict__ st, TileArgs ta, const DTerm* __restrict__ terms,
               int nterms, uint64_t ntiles, double2* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* tile = reinterpret_cast<V*>(smem_raw);
  __shared__ double2 red[32];
  const uint32_t size = 1u << ta.m;
  double2 acc = make_double2(0.0, 0.0);
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint64_t base = tile_base(ta, t);
    __syncthreads();  // the previous tile is no longer read
    for (uint32_t e = threadIdx.x; e < size; e += blockDim.x)
      tile[e] = st[tile_global(ta, ta.runoff, base, e)];
    __syncthreads();
    for (int k = 0; k < nterms; ++k) {
      const DTerm T = terms[k];
      double2 s = make_double2(0.0, 0.0);
      for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) {
        const uint64_t g = tile_global(ta, ta.runoff, base, e);
        const double2 x = to_d2(tile[e]);
        const double2 y = to_d2(tile[e ^ T.flip_local]);
        const double sg = sgn_of((g ^ T.flip) & T.zy);
        s.x = fma(sg * x.x, y.x, fma(sg * x.y, y.y, s.x));
        s.y = fma(sg * x.x, y.y, fma(-sg * x.y, y.x, s.y));
      }
      acc.x += T.wr * s.x - T.wi * s.y;
      acc.y += T.wr * s.y + T.wi * s.x;
    }
  }
  const double2 r = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

template <typename V>
qsv_status expect_noalloc_typed(const V* src, int n, cudaStream_t stream,
                                const std::vector<HTerm>& T, double* out) {
  if (T.empty()) {
    *out = 0.0;
    return QSV_SUCCESS;
  }
  const int m = std::min(n, sizeof(V) >= 16 ? 12 : 13);
  const int low = std::min(m, sizeof(V) >= 16 ? 4 : 5);
  std::vector<int> wide;
  std::vector<Group> groups = group_terms(T, n, m, low, &wide);
  for (const Group& G : groups)
    if (G.m != m) return fail(QSV_ERROR_INVALID_VALUE, "internal: term group of %d bits", G.m);
  const uint64_t N = dim(n);
  const uint64_t ntiles = 1ull << (n - m);
  const int nruns = 1 << (m - low);
  const unsigned gblocks = (unsigned)std::min<uint64_t>(kNoAllocBlocks, ntiles);
  const unsigned wblocks =
      (unsigned)std::min<uint64_t>(kNoAllocBlocks, (N + kRedThreads - 1) / kRedThreads);
  const size_t nparts = (size_t)gblocks * groups.size() + (size_t)wblocks * wide.size();
  // layout: [partials double2][out double2][terms][runoffs]
  const size_t out_off = nparts * sizeof(double2);
  const size_t term_off = (out_off + sizeof(double2) + 255) & ~size_t(255);
  const size_t term_bytes = T.size() * sizeof(DTerm);
  const size_t run_off = (term_off + term_bytes + 255) & ~size_t(255);
  const size_t total = run_off + groups.size() * (size_t)nruns * sizeof(uint64_t);
  if (total > kNoAllocScratchBytes)
    return fail(QSV_ERROR_SIZE,
                "observable needs %zu bytes of work memory; the allocation-free entry point "
                "has %zu (use qsv_expectation)", total, kNoAllocScratchBytes);
  void* sp = nullptr;
  if (qsv_status st = noalloc_scratch(&sp)) return st;
  unsigned char* dev = static_cast<unsigned char*>(sp);

  static const double pr[4] = {1, 0, -1, 0}, pi[4] = {0, 1, 0, -1};
  std::vector<DTerm> dt;
  std::vector<uint64_t> runoffs;
  std::vector<size_t> term0;
  for (const Group& G : groups) {
    int local_of[64];
    for (int j = 0; j < 64; ++j) local_of[j] = -1;
    for (int j = 0; j < G.m; ++j) local_of[G.bits[j]] = j;
    term0.push_back(dt.size());
    for (int ti : G.terms) {
      const HTerm& h = T[ti];
      DTerm d{};
      for (int b = 0; b < n; ++b)
        if ((h.flip >> b) & 1ull) d.flip_local |= 1u << local_of[b];
      d.flip = h.flip;
      d.zy = h.zy;
      d.wr = h.coef * pr[h.ny & 3];
      d.wi = h.coef * pi[h.ny & 3];
      dt.push_back(d);
    }
    tile_runoffs(G.bits, G.m, low, &runoffs);
  }
  std::vector<DTerm> wt;
  for (int ti : wide) {
    const HTerm& h = T[ti];
    DTerm d{};
    d.flip = h.flip;
    d.zy = h.zy;
    d.wr = h.coef * pr[h.ny & 3];
    d.wi = h.coef * pi[h.ny & 3];
    wt.push_back(d);
  }
  if (runoffs.size() != groups.size() * (size_t)nruns)
    return fail(QSV_ERROR_INVALID_VALUE, "internal: run table size");
  std::vector<unsigned char> host(total - term_off);
  std::memcpy(host.data(), dt.data(), dt.size() * sizeof(DTerm));
  std::memcpy(host.data() + (run_off - term_off), runoffs.data(), runoffs.size() * 8);
  if (qsv_status st = cuda_status(cudaMemcpyAsync(dev + term_off, host.data(), host.size(),
                                                  cudaMemcpyHostToDevice, stream),
                                  "no-alloc observable upload"))
    return st;
  const size_t smem = (size_t(1) << m) * sizeof(V);
  if (qsv_status st = cuda_status(cudaFuncSetAttribute((const void*)k_expect_tiles<V>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)smem), "no-alloc smem attribute"))
    return st;
  const int threads = std::min<int>(kRedThreads, std::max<int>(32, (1 << m) / 8));
  double2* partial = reinterpret_cast<double2*>(dev);
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    TileArgs ta;
    ta.n = n;
    ta.m = groups[gi].m;
    ta.low = low;
    for (int j = 0; j < 64; ++j) ta.bits[j] = (j < ta.m) ? (int8_t)groups[gi].bits[j] : 0;
    ta.runoff = reinterpret_cast<const uint64_t*>(dev + run_off) + gi * nruns;
    const DTerm* terms = reinterpret_cast<const DTerm*>(dev + term_off) + term0[gi];
    k_expect_tiles<V><<<gblocks, threads, smem, stream>>>(
        src, ta, terms, (int)groups[gi].terms.size(), ntiles, partial + gi * gblocks);
    count_launch();
    if (qsv_status st = cuda_status(cudaGetLastError(), "no-alloc expectation launch")) return st;
  }
  for (size_t wi = 0; wi < wt.size(); ++wi) {
    k_expect_wide<V><<<wblocks, kRedThreads, 0, stream>>>(
        src, N, wt[wi], partial + (size_t)gblocks * groups.size() + wi * wblocks);
    count_launch();
    if (qsv_status st = cuda_status(cudaGetLastError(), "no-alloc wide-term launch")) return st;
  }
  double2* dout = reinterpret_cast<double2*>(dev + out_off);
  k_final<<<1, 1024, 0, stream>>>(partial, (int)nparts, dout);
  count_launch();
  if (qsv_status st = cuda_status(cudaGetLastError(), "no-alloc final reduction")) return st;
  double2 h;
  if (qsv_status st = cuda_status(cudaMemcpyAsync(&h, dout, sizeof(h), cudaMemcpyDeviceToHost,
                                                  stream), "no-alloc result copy"))
    return st;
  if (qsv_status st = cuda_status(cudaStreamSynchronize(stream), "no-alloc synchronize"))
    return st;
  *out = h.x;
  return QSV_SUCCESS;
}

}  // namespace
}  // namespace qsv

extern "C" qsv_status qsv_expectation_noalloc(const void* state, int nbQubits, qsv_dtype dtype,
                                              void* cuda_stream, const char* paulis,
                                              const double* coefs, size_t nTerms, double* out) {
  using namespace qsv;
  if (!state) return fail(QSV_ERROR_INVALID_VALUE, "null state pointer");
  if (!out) return fail(QSV_ERROR_INVALID_VALUE, "null output");
  if (!dtype_valid(dtype)) return fail(QSV_ERROR_INVALID_VALUE, "bad dtype %d", (int)dtype);
  if (nbQubits < 1 || nbQubits > kMaxQubits)
    return fail(QSV_ERROR_SIZE, "nbQubits %d outside [1,%d]", nbQubits, kMaxQubits);
  std::vector<HTerm> T;
  if (qsv_status st = parse_terms(nbQubits, paulis, coefs, nTerms, &T)) return st;
  // the state must live on the current device, whose copy of the work array
  // the kernels use
  cudaPointerAttributes attr{};
  if (qsv_status st = cuda_status(cudaPointerGetAttributes(&attr, state),
                                  "cudaPointerGetAttributes(state)"))
    return st;
  int dev = 0;
  if (qsv_status st = cuda_status(cudaGetDevice(&dev), "cudaGetDevice")) return st;
  if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)
    return fail(QSV_ERROR_INVALID_VALUE, "qsv_expectation_noalloc: state is not device memory");
  if (attr.type == cudaMemoryTypeDevice && attr.device != dev)
    return fail(QSV_ERROR_INVALID_VALUE,
                "qsv_expectation_noalloc: state on device %d, current device %d", attr.device, dev);
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  switch (dtype) {
    case QSV_C128: return expect_noalloc_typed<double2>((const double2*)state, nbQubits, stream, T, out);
    case QSV_C64:  return expect_noalloc_typed<float2>((const float2*)state, nbQubits, stream, T, out);
    case QSV_F64:  return expect_noalloc_typed<double>((const double*)state, nbQubits, stream, T, out);
    case QSV_F32:  return expect_noalloc_typed<float>((const float*)state, nbQubits, stream, T, out);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

// Tensor-memory-accelerator (TMA) staging of stage tiles: host-side tensor
// maps over a state vector and the device copies that move one tile between
// global and shared memory (cp.async.bulk.tensor, completion on an
// mbarrier for loads and bulk groups for stores).  No multicast.
//
// A tile (tile.cuh) is the 2^m amplitudes that agree on every index bit
// outside an ascending bit set S whose lowest bits are the `low` lowest
// bits of the index.  The state is viewed as an array of 8-byte words
// (complex<float>: one word per amplitude; complex<double>: two, the word
// bit 0 selecting the component), and the tile's word bits are grouped into
// runs of consecutive bits.  Each run is one tensor-map dimension: the
// dimension spans the word bits from the run's first bit up to the next
// run's first bit (the last one up to the top of the index), and the box
// covers the run itself at the bottom of that span.  So one box of a 5-D
// map covers the five lowest runs of a tile and lands in shared memory in
// box order, which is the tile's local index order; tile bits above the
// fifth run are iterated, one copy per value, each copy landing at its
// offset (those bits are the top local bits).
//
// Shared-memory layout: the swizzle mode whose span equals the innermost
// box (16 bytes: none; 32, 64, 128 bytes: the 32/64/128-byte swizzle -- a
// box row narrower than the span would be padded to it), which XORs
// address bits [4, 4+B) (16-byte unit within the row) with address bits
// [7, 7+B), B = log2(span / 16); every copy starts on a 1024-byte boundary,
// so 16-byte unit u of the tile sits at u ^ ((u >> 3) & (2^B - 1))
// (phys_tma_host).
//
// Limits checked on the host: box extent <= 256 per dimension, an innermost
// box of 16, 32, 64 or 128 bytes, at least 1024 bytes per copy, coordinates
// below 2^31.  Stages that do not
// meet them stage their tiles with 16-byte cp.async instead.
#pragma once

#include <cuda.h>
#include <cstdint>

#include "tcgen05.cuh"

namespace qsv {

constexpr int kTmaMaxIter = 12;  // iterated tile bits (copies = 2^nit)

// Device description of a stage's TMA geometry (kernel argument).
struct TmaGeo {
  int use;             // 1: tiles move by TMA with the maps passed beside
  int nit;             // tile word bits iterated over copies
  uint32_t box_bytes;  // bytes per copy and vector
  int wshift;          // log2(words per amplitude)
  int swz;             // B: log2(innermost box bytes / 16), the swizzle's XOR width
  int relayout;        // 1: the kernel converts the tile to the cp.async layout after
                       // the load and back before the store (relayout_rows)
  int8_t dstart[5];    // first word bit of each dimension's span
  int8_t dbits[5];     // width of each dimension's span (0: padding dimension)
  int8_t it[kTmaMaxIter];  // word bits of the iterated tile bits, ascending
};

namespace tma {

// Global word index of copy i of the tile whose first amplitude is `base`.
__device__ __forceinline__ uint64_t copy_word(const TmaGeo& g, uint64_t base, uint32_t i) {
  uint64_t w = base << g.wshift;
  for (int k = 0; k < g.nit; ++k)
    if ((i >> k) & 1u) w |= 1ull << g.it[k];
  return w;
}

__device__ __forceinline__ void coords(const TmaGeo& g, uint64_t w, int (&c)[5]) {
#pragma unroll
  for (int k = 0; k < 5; ++k)
    c[k] = g.dbits[k] ? (int)((w >> g.dstart[k]) & ((1ull << g.dbits[k]) - 1ull)) : 0;
}

__device__ __forceinline__ void load(void* dst, const CUtensorMap* map, const int (&c)[5],
                                     uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
      ::"r"(tc::smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c[0]), "r"(c[1]),
        "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(tc::smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void store(const CUtensorMap* map, const int (&c)[5], const void* src) {
  asm volatile(
      "cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];"
      ::"l"(reinterpret_cast<uint64_t>(map)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]),
        "r"(c[4]), "r"(tc::smem_addr(src))
      : "memory");
}

__device__ __forceinline__ void expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               ::"r"(tc::smem_addr(bar)), "r"(bytes) : "memory");
}

// Waits for the mbarrier phase of the given parity: at most `limit`
// suspended polls of up to 1 ms each.  False when the phase did not complete.
__device__ __forceinline__ bool wait_phase(uint64_t* bar, uint32_t parity, int limit) {
  const uint32_t a = tc::smem_addr(bar);
  for (int it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(a), "r"(parity), "r"(1000000u) : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void store_commit_and_wait() {
  asm volatile("cp.async.bulk.commit_group;\ncp.async.bulk.wait_group 0;" ::: "memory");
}

// ---- one stage tile (NV vectors of tile_bytes each) ------------------------
// The stage kernels call, in order: tile_fits (every thread; false: the
// copies would not land inside the launch's shared memory on 1024-byte
// boundaries -- flag 2 is set and the kernel returns), tile_start (one
// thread initialises the mbarrier and issues the loads), their own
// independent work, tile_wait (every thread; false: the bounded wait gave
// up -- flag 1 is set, the copies are given time to drain, the kernel
// returns), the passes, tile_store (every thread; one issues the stores and
// waits for them).

template <int NV>
__device__ __forceinline__ bool tile_fits(const TmaGeo& g, const void* smem_dyn, const void* t0,
                                          uint32_t tile_bytes, uint32_t smem_bytes,
                                          unsigned* err) {
  const uint32_t off = tc::smem_addr(t0) - tc::smem_addr(smem_dyn);
  const uint32_t copies = 1u << g.nit;
  const bool ok = (tc::smem_addr(t0) & 1023u) == 0 && (g.box_bytes & 1023u) == 0 &&
                  copies * g.box_bytes == tile_bytes &&
                  off + uint64_t(NV) * tile_bytes <= smem_bytes;
  if (!ok && threadIdx.x == 0) atomicOr(err, 2u);
  return ok;
}

template <int NV>
__device__ __forceinline__ void tile_start(const TmaGeo& g, const CUtensorMap* m0,
                                           const CUtensorMap* m1, void* t0, void* t1,
                                           uint64_t base, uint64_t* bar) {
  if (threadIdx.x != 0) return;
  const uint32_t copies = 1u << g.nit;
  tc::bar_init(bar, 1);
  tc::bar_init_fence();
  expect_tx(bar, copies * g.box_bytes * NV);
  for (uint32_t i = 0; i < copies; ++i) {
    int c[5];
    coords(g, copy_word(g, base, i), c);
    load(static_cast<unsigned char*>(t0) + i * g.box_bytes, m0, c, bar);
    if (NV == 2) load(static_cast<unsigned char*>(t1) + i * g.box_bytes, m1, c, bar);
  }
}

__device__ __forceinline__ bool tile_wait(uint64_t* bar, unsigned* err, int limit) {
  __syncthreads();  // the mbarrier's initialisation, for the other threads
  const bool ok = wait_phase(bar, 0, limit);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      atomicOr(err, 1u);
      (void)wait_phase(bar, 0, limit);
    }
    return false;
  }
  return true;
}

template <int NV>
__device__ __forceinline__ void tile_store(const TmaGeo& g, const CUtensorMap* m0,
                                           const CUtensorMap* m1, const void* t0, const void* t1,
                                           uint64_t base) {
  tc::fence_proxy_async();  // this thread's shared-memory writes, for the copy engine
  __syncthreads();
  if (threadIdx.x != 0) return;
  const uint32_t copies = 1u << g.nit;
  for (uint32_t i = 0; i < copies; ++i) {
    int c[5];
    coords(g, copy_word(g, base, i), c);
    store(m0, c, static_cast<const unsigned char*>(t0) + i * g.box_bytes);
    if (NV == 2) store(m1, c, static_cast<const unsigned char*>(t1) + i * g.box_bytes);
  }
  store_commit_and_wait();
}

constexpr int kTileWaitLimit = 2000;  // suspended polls (up to 1 ms each) for a tile load

// Moves a tile between the TMA layout (unit u at u ^ ((u >> 3) & (2^B - 1)))
// and the four-level XOR layout of the cp.async path (unit u at
// u ^ ((u>>3 ^ u>>6 ^ u>>9 ^ u>>12) & 7), stage_exec.cuh phys): both keep
// each 128-byte row in place and permute its eight 16-byte units by an XOR
// that depends on the row r alone, so one layout becomes the other by
// XOR-ing each row's unit index with
//   d(r) = (r & (2^B - 1)) ^ ((r ^ r>>3 ^ r>>6 ^ r>>9) & 7)
// -- an involution, the same call converts either way.  A warp takes four
// whole rows at a time (lane = row * 8 + unit), reads them, then writes
// them back permuted.  The caller synchronises the block around it.
__device__ __forceinline__ void relayout_rows(void* tile, uint32_t rows, int B) {
  float4* t = static_cast<float4*>(tile);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const uint32_t mask = (1u << B) - 1u;
  for (uint32_t r0 = warp * 4; r0 < rows; r0 += nwarps * 4) {
    const uint32_t r = r0 + (lane >> 3), c = lane & 7u;
    const bool ok = r < rows;
    const uint32_t d = ((r & mask) ^ ((r ^ (r >> 3) ^ (r >> 6) ^ (r >> 9)) & 7u));
    float4 v;
    if (ok && d) v = t[r * 8 + c];
    __syncwarp();
    if (ok && d) t[r * 8 + (c ^ d)] = v;
  }
}

// Dynamic shared memory from the next 1024-byte boundary (the launch
// reserves 1024 bytes more than it uses).
__device__ __forceinline__ unsigned char* align1024(unsigned char* p) {
  return p + ((1024u - (tc::smem_addr(p) & 1023u)) & 1023u);
}

}  // namespace tma

// ---- host ---------------------------------------------------------------------
// Shared-memory position of local element e of a TMA-staged tile
// (epu elements per 16-byte unit) under a swizzle of XOR width B: unit
// u -> u ^ ((u >> 3) & (2^B - 1)).  Linear over GF(2) in e.
inline uint32_t phys_tma_host(uint32_t e, uint32_t epu, int B) {
  const uint32_t u = e / epu;
  return (u ^ ((u >> 3) & ((1u << B) - 1u))) * epu + e % epu;
}

// Builds the map (one per vector, same geometry) and the device geometry for
// a stage with ascending tile bits bits[0..m-1] of an n-qubit state of
// elem_bytes-byte amplitudes at `data`.  Returns false where the stage's
// tiles cannot move by TMA (the caller then uses cp.async).
bool tma_stage_map(const int* bits, int m, int n, size_t elem_bytes, const void* data,
                   CUtensorMap* map, TmaGeo* geo);

}  // namespace qsv

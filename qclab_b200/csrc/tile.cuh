// Tile geometry shared by the fused sweeps and the tiled reductions.
//
// A tile is the set of 2^m amplitudes that agree on every index bit outside
// a chosen bit set S (|S| = m, S holds the `low` lowest bits so a tile is
// 2^(m-low) contiguous runs of 2^low amplitudes).  Local index e (m bits,
// local bit j <-> global bit bits[j]) maps to
//   global(e) = base(tile) | runoff[e >> low] | (e & (2^low - 1)).
#pragma once

#include <cstdint>
#include <vector>
#include "common.cuh"

namespace qsv {

struct TileArgs {
  int n, m, low;
  int8_t bits[64];          // local bit -> global bit, ascending
  const uint64_t* runoff;   // 2^(m-low) offsets of the runs
};

// Base index of tile t: t spread over the bits outside S.
__device__ __forceinline__ uint64_t tile_base(const TileArgs& a, uint64_t t) {
  uint64_t base = t << a.low;
  for (int j = a.low; j < a.m; ++j) base = insert_zero(base, a.bits[j]);
  return base;
}

__device__ __forceinline__ uint64_t tile_global(const TileArgs& a, const uint64_t* runoff,
                                                uint64_t base, uint32_t e) {
  return base | runoff[e >> a.low] | (e & ((1u << a.low) - 1u));
}

// Host: run offsets of a tile bit set (ascending bits[0..m-1], bits[j] = j
// for j < low).
inline void tile_runoffs(const int* bits, int m, int low, std::vector<uint64_t>* out) {
  const uint32_t nruns = 1u << (m - low);
  for (uint32_t r = 0; r < nruns; ++r) {
    uint64_t off = 0;
    for (int j = low; j < m; ++j)
      if ((r >> (j - low)) & 1u) off |= 1ull << bits[j];
    out->push_back(off);
  }
}

// Host: the ascending bit list of a bit mask, filled with the lowest unused
// bits up to m bits (n >= m).
inline int tile_bits_of(uint64_t S, int n, int m, int* bits) {
  for (int b = 0; b < n && __builtin_popcountll(S) < m; ++b)
    if (!((S >> b) & 1ull)) S |= 1ull << b;
  int k = 0;
  for (int b = 0; b < n; ++b)
    if ((S >> b) & 1ull) bits[k++] = b;
  return k;
}

// ---- FP64 views of elements --------------------------------------------------
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ double2 to_d2(double v) { return make_double2(v, 0.0); }
__device__ __forceinline__ double2 to_d2(float v) { return make_double2((double)v, 0.0); }

template <typename V> __device__ __forceinline__ V from_d2(double2 v);
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}
template <> __device__ __forceinline__ double from_d2<double>(double2 v) { return v.x; }
template <> __device__ __forceinline__ float from_d2<float>(double2 v) { return (float)v.x; }

// Sum of a double2 over the block (all threads must call); valid in thread 0.
__device__ __forceinline__ double2 block_sum(double2 v, double2* red /* >= 32 */) {
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  if (w == 0) {
    v = (l < nw) ? red[l] : make_double2(0.0, 0.0);
    for (int o = 16; o > 0; o >>= 1) {
      v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
      v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
  }
  return v;
}

}  // namespace qsv

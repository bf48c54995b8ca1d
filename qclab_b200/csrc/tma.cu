// Host side of the TMA tile staging (tma.cuh): tensor maps of stage tiles.
#include <cuda_runtime.h>
#include <mutex>
#include <vector>

#include "tma.cuh"

namespace qsv {

namespace {

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver the runtime uses (no link-time
// dependency on libcuda).
EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}

struct Run {
  int start, len;
};

}  // namespace

bool tma_stage_map(const int* bits, int m, int n, size_t elem_bytes, const void* data,
                   CUtensorMap* map, TmaGeo* geo) {
  *geo = TmaGeo{};
  if (elem_bytes != 8 && elem_bytes != 16) return false;
  if ((reinterpret_cast<uintptr_t>(data) & 15u) != 0) return false;
  const EncodeTiled encode = encoder();
  if (!encode) return false;
  const int ws = elem_bytes == 16 ? 1 : 0;
  const int nw = n + ws;
  if (nw > 36) return false;
  // the tile's word bits, ascending, in runs: the innermost box at most 128
  // bytes (16 words), every other box extent at most 256
  std::vector<int> tw;
  if (ws) tw.push_back(0);
  for (int j = 0; j < m; ++j) tw.push_back(bits[j] + ws);
  std::vector<Run> runs;
  for (int b : tw) {
    const int cap = runs.size() == 1 ? 4 : 8;  // the run being extended is runs.back()
    if (!runs.empty() && runs.back().start + runs.back().len == b && runs.back().len < cap)
      ++runs.back().len;
    else
      runs.push_back({b, 1});
  }
  if (runs.empty() || runs[0].start != 0 || runs[0].len < 1) return false;
  // innermost box of 16..128 bytes; the swizzle span is set equal to it
  if (runs[0].len < 1 || runs[0].len > 4) return false;
  const int swz = runs[0].len - 1;
  static const CUtensorMapSwizzle kModes[4] = {
      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_SWIZZLE_64B,
      CU_TENSOR_MAP_SWIZZLE_128B};
  const int D = (int)std::min<size_t>(5, runs.size());
  int boxbits = 0;
  for (int k = 0; k < D; ++k) boxbits += runs[k].len;
  int nit = 0;
  for (size_t k = D; k < runs.size(); ++k)
    for (int b = 0; b < runs[k].len; ++b) {
      if (nit >= kTmaMaxIter) return false;
      geo->it[nit++] = (int8_t)(runs[k].start + b);
    }
  if (boxbits < 7) return false;  // every copy a whole number of 1024-byte swizzle blocks
  // both vectors' tiles within one mbarrier transaction count (< 2^20 bytes)
  if ((elem_bytes << m) * 2 >= (1ull << 20)) return false;
  // dimension spans; the last one is split while its coordinates would not
  // fit in 31 bits
  int dstart[5], dend[5], dbox[5];
  int nd = D;
  for (int k = 0; k < D; ++k) {
    dstart[k] = runs[k].start;
    dend[k] = (k + 1 < D) ? runs[k + 1].start : nw;
    dbox[k] = runs[k].len;
  }
  while (dend[nd - 1] - dstart[nd - 1] > 31 && nd < 5) {
    const int cut = dstart[nd - 1] + 31;
    dstart[nd] = cut;
    dend[nd] = dend[nd - 1];
    dbox[nd] = 0;
    dend[nd - 1] = cut;
    ++nd;
  }
  for (int k = 0; k < nd; ++k)
    if (dend[k] - dstart[k] > 31) return false;
  cuuint64_t gdim[5], gstride[4];
  cuuint32_t box[5], estride[5];
  for (int k = 0; k < 5; ++k) {
    estride[k] = 1;
    if (k < nd) {
      gdim[k] = 1ull << (dend[k] - dstart[k]);
      box[k] = 1u << dbox[k];
      if (k > 0) gstride[k - 1] = 8ull << dstart[k];
    } else {  // padding dimension of extent 1
      gdim[k] = 1;
      box[k] = 1;
      gstride[k - 1] = 8ull << nw;
    }
  }
  for (int k = 0; k < 4; ++k)
    if (gstride[k] % 16 != 0 || gstride[k] >= (1ull << 40)) return false;
  const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 5, const_cast<void*>(data), gdim,
                            gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, kModes[swz],
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return false;
  geo->use = 1;
  geo->nit = nit;
  geo->box_bytes = 8u << boxbits;
  geo->wshift = ws;
  geo->swz = swz;
  for (int k = 0; k < 5; ++k) {
    geo->dstart[k] = (int8_t)(k < nd ? dstart[k] : 0);
    geo->dbits[k] = (int8_t)(k < nd ? dend[k] - dstart[k] : 0);
  }
  return true;
}

}  // namespace qsv

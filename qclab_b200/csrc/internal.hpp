// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <vector>
#include "qclab_b200.h"
#include "lower.hpp"

struct qsv_state_s {
  int n = 0;
  qsv_dtype dtype = QSV_C128;
  void* d = nullptr;        // 2^n elements on `device`
  bool owns = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  void* scratch = nullptr;  // device scratch owned by the state (plans, partial sums)
  size_t scratch_bytes = 0;
  void* aux = nullptr;      // device work vectors (the adjoint's lambda and partials)
  size_t aux_bytes = 0;
};

namespace qsv {

void set_error(const char* fmt, ...);
qsv_status fail(qsv_status st, const char* fmt, ...);
qsv_status cuda_status(cudaError_t e, const char* what);
void count_launch(uint64_t k = 1);
// one stage launch whose tiles move by TMA
void count_tma_launch();
// Makes `waiter` wait (on the device, no host synchronisation) for the work
// issued to `producer` so far; a no-op for the same stream.
qsv_status stream_wait(cudaStream_t waiter, cudaStream_t producer);

inline size_t elem_bytes(qsv_dtype t) {
  switch (t) {
    case QSV_C64: return 8;
    case QSV_C128: return 16;
    case QSV_F32: return 4;
    case QSV_F64: return 8;
  }
  return 0;
}
inline bool dtype_valid(int t) { return t >= QSV_C64 && t <= QSV_F64; }
inline bool dtype_real(qsv_dtype t) { return t == QSV_F32 || t == QSV_F64; }
inline bool dtype_double(qsv_dtype t) { return t == QSV_C128 || t == QSV_F64; }
inline uint64_t dim(int n) { return 1ull << n; }

// Maximum register size: 2^40 amplitudes would already exceed any single
// GPU's memory; bounds all 64-bit index arithmetic.
constexpr int kMaxQubits = 40;

// Lowers a gate list for a state (dispatches on the state's real type).
// fp64: lower in double whatever the state's precision (the fused sweeps);
// otherwise in the state's real type, as the reference's templates do.
qsv_status lower_for_state(const qsv_state_s* s, const qsv_gate* gates,
                           size_t count, char op, int offset,
                           std::vector<Lowered>* out, bool fp64 = false);

// Grows the state's device scratch buffer to at least `bytes` (stream-ordered
// with respect to earlier work on the state's stream).
qsv_status ensure_scratch(qsv_state_s* s, size_t bytes);
qsv_status ensure_aux(qsv_state_s* s, size_t bytes);

// Unfused launch of one lowered gate (reference-exact kernels).
qsv_status launch_unfused(qsv_state_s* s, const Lowered& L);

// Fused execution of a lowered gate list.
qsv_status run_fused(qsv_state_s* s, const std::vector<Lowered>& gates,
                     const qsv_fuse_opts* opts);

}  // namespace qsv

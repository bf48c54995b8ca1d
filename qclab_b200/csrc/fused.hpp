// Interface of the fused stage executor (apply_fused.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>
#include "internal.hpp"

namespace qsv {

struct ExecArgs {
  qsv_state_s* s = nullptr;              // stream, size, dtype and plan scratch
  const std::vector<Lowered>* items = nullptr;
  void* v0 = nullptr;                    // vector the gates act on (psi)
  void* v1 = nullptr;                    // second vector (lambda), nv == 2
  int nv = 1;
  const qsv_fuse_opts* opts = nullptr;
  double* partial = nullptr;             // [nslots][ntiles] partial sums (SH_RED)
  size_t partial_bytes = 0;
  int nslots = 0;
  double* rows_out = nullptr;            // nslots row sums (device)
  uint64_t* ntiles_out = nullptr;
};

int default_tile_bits(size_t elem_bytes, int nv);

// Per-stage CUDA-event timing of a fused sweep (qsv_fuse_opts.profile): an
// event before the first stage and after each one, on the sweep's stream;
// finish() waits for the last event and stores the durations for
// qsv_last_stage_times.  Does nothing when off.
class StageTimer {
 public:
  StageTimer(bool on, size_t nstages, cudaStream_t stream);
  ~StageTimer();
  qsv_status start();
  qsv_status mark(size_t stage);
  qsv_status finish();

 private:
  bool on_;
  cudaStream_t stream_;
  std::vector<cudaEvent_t> ev_;
};

// Sweep of a complex<double> / complex<float> state (x.nv = 1) or of psi
// and lambda with gradient terms (x.nv = 2) on the gate-specialised engine
// (apply_gates.cu) with tiles of 2^m amplitudes; QSV_ERROR_NOT_SUPPORTED,
// with nothing launched, when the items do not fit it.
template <typename V>
qsv_status execute_gates(const ExecArgs& x, int m, int low, int max_gates, bool vec16);
// Register bits of its passes: single-vector 4 for 16-byte elements, 5 for
// 8-byte ones (4 with qsv_fuse_opts.reg_bits = 4); two-vector 3 (16-byte)
// or 4 (8-byte).
int gate_pass_bits(size_t elem_bytes, const qsv_fuse_opts* opts, int nv = 1);
// Fixed-order sum of x.partial's rows (x.nslots rows of ntiles tile sums)
// into x.rows_out, on the state's stream.
qsv_status reduce_rows(const ExecArgs& x, uint64_t ntiles);
// Its plan statistics: ops and passes per stage.
qsv_status gate_plan_counts(const std::vector<Lowered>& items, int n, int m, int low,
                            const qsv_fuse_opts* opts, int max_gates, size_t elem_bytes,
                            std::vector<int>* ops, std::vector<int>* passes);
int default_low_bits(size_t elem_bytes);
// low bits of complex single-vector gate-pass sweeps (engine 5) when unset
int gate_default_low(size_t elem_bytes);

// Plans the items into stages and runs them.
qsv_status execute_fused(const ExecArgs& x);

// QSV_ERROR_TIMEOUT once (and clears it) if a tcgen05 sweep's bounded wait
// gave up since the last call; reads the device flag on `stream` (call after
// that stream has synchronised; nothing is read before a tcgen05 launch).
qsv_status tc_check_status(cudaStream_t stream);
// Device flag that a sweep kernel sets when one of its bounded waits gave
// up (read and cleared by tc_check_status at the next synchronisation);
// null if its address cannot be had.
unsigned* sweep_wait_flag();

// Tile bits the executor uses for nv vectors of an n-qubit state: the
// requested (or default) size, at most 14 and n, and at most 256 threads of
// 2^r amplitudes (times the groups a thread takes per pass).
int effective_tile_bits(size_t elem_bytes, int nv, int n, const qsv_fuse_opts* opts);

// Number of tiles the executor will use for nv vectors of a state.
inline uint64_t fused_tiles(int n, size_t elem_bytes, int nv, const qsv_fuse_opts* opts) {
  return 1ull << (n - effective_tile_bits(elem_bytes, nv, n, opts));
}

// Tiled reductions (reduce.cu).
qsv_status observable_internal(qsv_state_s* dst, qsv_state_s* src, const char* paulis,
                               const double* coefs, size_t nterms);
qsv_status inner_internal(qsv_state_s* a, qsv_state_s* b, double* out);
qsv_status expectation_internal(qsv_state_s* s, const char* paulis, const double* coefs,
                                size_t nterms, double* out);

}  // namespace qsv

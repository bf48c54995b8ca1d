// Adjoint (reverse-mode) gradient of an expectation value.
//
//   E(theta) = <psi_N| H |psi_N>,  psi_N = U_N ... U_1 psi_0
//   dE/dtheta_k = 2 Re <lam_k| dU_k psi_{k-1}>
//               = w_k Im(<lam_k| Pi_k P_k |psi_k>)
// with lam_k = U_{k+1}^+ ... U_N^+ H psi_N and the generator (w, Pi, P) of
// gate k (lower.hpp: Generator).  The forward sweep and the backward sweep
// are fused sweeps (apply_fused.cu); the backward sweep carries psi and lam
// through each shared-memory tile together, applying U_k^+ to both and
// evaluating each gradient term inside the tile, so no intermediate state is
// stored and the state is streamed once per stage, not once per gate.
// (Jones and Gacon, "Efficient calculation of gradients in classical
// simulations of variational quantum algorithms", 2020.)
#include <algorithm>
#include <vector>
#include "fused.hpp"
#include "internal.hpp"

namespace qsv {
namespace {

// Partial-sum rows per backward segment: bounds the partial buffer.
constexpr size_t kMaxPartialBytes = size_t(256) << 20;

}  // namespace
}  // namespace qsv

using namespace qsv;

extern "C" qsv_status qsv_adjoint_gradient(qsv_state s, const qsv_gate* gates, size_t nGates,
                                           const char* paulis, const double* coefs,
                                           size_t nTerms, double* grads, int nParams,
                                           double* expval) {
  if (!s || !s->d) return fail(QSV_ERROR_INVALID_VALUE, "null state");
  if (nGates && !gates) return fail(QSV_ERROR_INVALID_VALUE, "null gate list");
  if (nParams > 0 && !grads) return fail(QSV_ERROR_INVALID_VALUE, "null gradient buffer");
  if (nParams < 0) return fail(QSV_ERROR_INVALID_VALUE, "negative nParams");
  const int n = s->n;
  // generators of the parametric gates
  std::vector<Generator> gens(nGates);
  for (size_t k = 0; k < nGates; ++k) {
    if (gates[k].param < 0) continue;
    if (gates[k].param >= nParams)
      return fail(QSV_ERROR_INVALID_VALUE, "gate %zu: param %d >= nParams %d", k, gates[k].param,
                  nParams);
    if (!generator_of(gates[k], 0, n, &gens[k]))
      return fail(QSV_ERROR_NOT_SUPPORTED, "gate %zu (kind %d) has no trainable angle", k,
                  gates[k].kind);
  }
  // forward sweep
  std::vector<Lowered> fwd;
  if (qsv_status st = lower_for_state(s, gates, nGates, 'N', 0, &fwd)) return st;
  if (qsv_status st = run_fused(s, fwd, nullptr)) return st;

  // lam = H psi_N in the work vector
  const size_t eb = elem_bytes(s->dtype);
  const size_t vec_bytes = dim(n) * eb;
  const uint64_t ntiles = fused_tiles(n, eb, 2, nullptr);
  int nslots_total = 0;
  for (size_t k = 0; k < nGates; ++k) nslots_total += gates[k].param >= 0;
  const size_t rows_bytes = ((size_t)std::max(nslots_total, 1) * sizeof(double) + 255) & ~size_t(255);
  const int seg_slots = (int)std::max<size_t>(1, std::min<size_t>(
      (size_t)std::max(nslots_total, 1), kMaxPartialBytes / (ntiles * sizeof(double))));
  const size_t part_bytes = (size_t)seg_slots * ntiles * sizeof(double);
  if (qsv_status st = ensure_aux(s, vec_bytes + rows_bytes + part_bytes)) return st;
  unsigned char* aux = static_cast<unsigned char*>(s->aux);
  qsv_state_s lam;
  lam.n = n;
  lam.dtype = s->dtype;
  lam.d = aux;
  lam.owns = false;
  lam.stream = s->stream;
  if (qsv_status st = observable_internal(&lam, s, paulis, coefs, nTerms)) return st;
  double e[2] = {0.0, 0.0};
  if (qsv_status st = inner_internal(s, &lam, e)) return st;

  // backward sweep: [RED_k] U_k^+ for k = N..1, in segments of <= seg_slots reductions
  double* rows = reinterpret_cast<double*>(aux + vec_bytes);
  double* partial = reinterpret_cast<double*>(aux + vec_bytes + rows_bytes);
  std::vector<int> slot_param;
  std::vector<Lowered> items;
  const bool dbl = dtype_double(s->dtype), real = dtype_real(s->dtype);
  int seg_first_slot = 0;
  auto flush = [&]() -> qsv_status {
    if (items.empty()) return QSV_SUCCESS;
    ExecArgs x;
    x.s = s;
    x.items = &items;
    x.v0 = s->d;
    x.v1 = lam.d;
    x.nv = 2;
    x.partial = partial;
    x.partial_bytes = part_bytes;
    x.nslots = (int)slot_param.size() - seg_first_slot;
    x.rows_out = rows + seg_first_slot;
    qsv_status st = execute_fused(x);
    items.clear();
    seg_first_slot = (int)slot_param.size();
    return st;
  };
  for (size_t i = 0; i < nGates; ++i) {
    const size_t k = nGates - 1 - i;
    if (gates[k].param >= 0) {
      if ((int)slot_param.size() - seg_first_slot == seg_slots)
        if (qsv_status st = flush()) return st;
      Lowered R;
      R.shape = SH_RED;
      R.gen = gens[k];
      R.slot = (int)slot_param.size() - seg_first_slot;
      R.param = gates[k].param;
      items.push_back(R);
      slot_param.push_back(gates[k].param);
    }
    Lowered inv;
    qsv_status st = dbl ? lower_gate<double>(gates[k], 'C', 0, n, real, &inv)
                        : lower_gate<float>(gates[k], 'C', 0, n, real, &inv);
    if (st) return fail(st, "gate %zu could not be inverted", k);
    if (inv.shape != SH_NONE) items.push_back(inv);
  }
  if (qsv_status st = flush()) return st;

  std::vector<double> host(slot_param.size());
  if (!host.empty()) {
    if (qsv_status st = cuda_status(cudaMemcpyAsync(host.data(), rows, host.size() * sizeof(double),
                                                    cudaMemcpyDeviceToHost, s->stream),
                                    "gradient copy"))
      return st;
  }
  if (qsv_status st = cuda_status(cudaStreamSynchronize(s->stream), "gradient synchronize"))
    return st;
  for (int p = 0; p < nParams; ++p) grads[p] = 0.0;
  for (size_t r = 0; r < host.size(); ++r) grads[slot_param[r]] += host[r];
  if (expval) *expval = e[0];
  return QSV_SUCCESS;
}

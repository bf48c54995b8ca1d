// Host check of the gate-specialised engine's plan (gate_plan.hpp): lowers
// gate records in FP64, plans and factors them into register-pass ops
// exactly as the GPU executor does, and applies the plan with the host
// mirror of the device ops (same stage, tile, pass and op order).  Built
// with g++ (no CUDA) by tests/test_gate_plan.py, which compares the output
// with the C oracle.
//
//   gate_plan_test n R m low op offset records.bin state_in.bin state_out.bin
// records.bin: qsv_gate[]; states: complex<double>[2^n].  Prints
// "stages passes ops" of the plan.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "gate_plan.hpp"

// adjoint mode: gate_plan_test adjoint n R m low records psi lam rows_out
// builds the backward list of qsv_adjoint_gradient ([gradient term] U_k^+
// for k = N..1), packs it for two vectors and writes one gradient term per
// parametric gate, in backward order.
static int adjoint_main(char** argv) {
  const int n = std::atoi(argv[2]), R = std::atoi(argv[3]), m = std::atoi(argv[4]);
  const int low = std::atoi(argv[5]);
  auto slurp = [](const char* path) {
    std::vector<char> buf;
    FILE* f = std::fopen(path, "rb");
    if (!f) return buf;
    char tmp[65536];
    size_t k;
    while ((k = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + k);
    std::fclose(f);
    return buf;
  };
  const std::vector<char> rb = slurp(argv[6]), pb = slurp(argv[7]), lb = slurp(argv[8]);
  const size_t ng = rb.size() / sizeof(qsv_gate), N = size_t(1) << n;
  const qsv_gate* g = reinterpret_cast<const qsv_gate*>(rb.data());
  std::vector<qsv::Lowered> items;
  int slot = 0;
  for (size_t i = 0; i < ng; ++i) {
    const size_t k = ng - 1 - i;
    if (g[k].param >= 0) {
      qsv::Lowered red;
      red.shape = qsv::SH_RED;
      if (!qsv::generator_of(g[k], 0, n, &red.gen)) return 3;
      red.slot = slot++;
      items.push_back(red);
    }
    qsv::Lowered inv;
    if (qsv::lower_gate<double>(g[k], 'C', 0, n, false, &inv) != QSV_SUCCESS) return 3;
    if (inv.shape != qsv::SH_NONE) items.push_back(inv);
  }
  qsv::gx::GxPlan plan;
  if (!qsv::gx::pack_gate_plan(items, n, m, low, R, 256, 16384, 16, &plan, true)) return 4;
  std::vector<std::complex<double>> psi(N), lam(N);
  std::memcpy(psi.data(), pb.data(), N * sizeof(psi[0]));
  std::memcpy(lam.data(), lb.data(), N * sizeof(lam[0]));
  std::vector<double> rows(slot > 0 ? slot : 1, 0.0);
  qsv::gx::host_apply_plan(plan, n, psi, &lam, rows.data());
  FILE* f = std::fopen(argv[9], "wb");
  std::fwrite(rows.data(), sizeof(double), (size_t)slot, f);
  std::fclose(f);
  std::printf("%zu %zu %zu\n", plan.stages.size(), plan.passes.size(), plan.ops.size());
  return 0;
}

int main(int argc, char** argv) {
  if (argc == 10 && std::string(argv[1]) == "adjoint") return adjoint_main(argv);
  if (argc != 10) {
    std::fprintf(stderr, "usage: %s n R m low op offset records state_in state_out\n", argv[0]);
    return 2;
  }
  const int n = std::atoi(argv[1]), R = std::atoi(argv[2]), m = std::atoi(argv[3]);
  const int low = std::atoi(argv[4]);
  const char op = argv[5][0];
  const int offset = std::atoi(argv[6]);
  auto slurp = [](const char* path) {
    std::vector<char> buf;
    FILE* f = std::fopen(path, "rb");
    if (!f) return buf;
    char tmp[65536];
    size_t k;
    while ((k = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + k);
    std::fclose(f);
    return buf;
  };
  const std::vector<char> rb = slurp(argv[7]), sb = slurp(argv[8]);
  const size_t ng = rb.size() / sizeof(qsv_gate);
  const size_t N = size_t(1) << n;
  if (sb.size() != N * sizeof(std::complex<double>)) {
    std::fprintf(stderr, "state size mismatch\n");
    return 2;
  }
  const qsv_gate* g = reinterpret_cast<const qsv_gate*>(rb.data());
  std::vector<qsv::Lowered> items(ng);
  size_t bad = 0;
  if (qsv::lower_list<double>(g, ng, op, offset, n, false, items.data(), &bad) != QSV_SUCCESS) {
    std::fprintf(stderr, "lowering failed at gate %zu\n", bad);
    return 3;
  }
  qsv::gx::GxPlan plan;
  if (!qsv::gx::pack_gate_plan(items, n, m, low, R, 256, 16384, 16, &plan)) {
    std::fprintf(stderr, "plan not supported\n");
    return 4;
  }
  std::vector<std::complex<double>> v(N);
  std::memcpy(v.data(), sb.data(), sb.size());
  qsv::gx::host_apply_plan(plan, n, v);
  FILE* f = std::fopen(argv[9], "wb");
  std::fwrite(v.data(), sizeof(v[0]), N, f);
  std::fclose(f);
  std::printf("%zu %zu %zu\n", plan.stages.size(), plan.passes.size(), plan.ops.size());
  return 0;
}

// Drives include/qclab_b200/adapter.hpp with genuine QCLAB++ objects and
// compares the GPU results with QCLAB++'s own CPU simulate/apply.
// Built by oracle/Makefile (needs the reference tree) into
// oracle/_ref/adapter_test; run by tests/test_gpu_adapter.py on a GPU.
#include <complex>
#include <cstdio>
#include <random>

#include <cuda_runtime.h>

#include "qclab_b200/adapter.hpp"

using namespace qclab::qgates;

template <typename T>
struct UserGate2 : public QGate2<T> {  // a non-symmetric user 2-qubit gate
  UserGate2(int a, int b) : q_{std::min(a, b), std::max(a, b)} {}
  bool fixed() const override { return true; }
  bool controlled() const override { return false; }
  int qubit() const override { return q_[0]; }
  std::vector<int> qubits() const override { return {q_[0], q_[1]}; }
  void setQubits(const int* q) override { q_[0] = q[0]; q_[1] = q[1]; }
  qclab::dense::SquareMatrix<T> matrix() const override {
    using R = qclab::real_t<T>;
    const R s = R(0.5);
    // a real orthogonal, non-symmetric 4x4 (Hadamard-like with a sign twist)
    return qclab::dense::SquareMatrix<T>(s, s, s, s, s, -s, s, -s, s, s, -s, -s, -s, s, s, -s);
  }
  int toQASM(std::ostream&, const int = 0) const override { return -1; }
 protected:
  bool equals(const qclab::QObject<T>&) const override { return false; }
  int q_[2];
};

template <typename T>
int run(const char* name, const qclab::QCircuit<T>& c, std::mt19937_64& rng, bool fused) {
  const int n = c.nbQubits();
  std::normal_distribution<double> N01;
  std::vector<T> v(size_t(1) << n);
  for (auto& x : v) {
    if constexpr (qclab::is_complex_v<T>) x = T(N01(rng), N01(rng));
    else x = T(N01(rng));
  }
  int bad = 0;
  for (char opc : {'N', 'T', 'C'}) {
    const qclab::Op op = static_cast<qclab::Op>(opc);
    std::vector<T> ref = v, gpu = v;
    c.apply(op, n, ref);                       // QCLAB++ CPU path
    qclab_b200::apply(c, op, n, gpu, 0, fused);  // B200 path
    double err = 0;
    bool same = true;
    for (size_t i = 0; i < v.size(); ++i) {
      err = std::max(err, (double)std::abs(ref[i] - gpu[i]));
      same = same && (ref[i] == gpu[i]);
    }
    // fused sweeps reorder commuting gates: rounding-level differences on the
    // unnormalised N(0,1) inputs (complex<double> 1e-10, complex<float> 5e-5)
    const double tol = sizeof(qclab::real_t<T>) == 8 ? 1e-10 : 5e-5;
    const bool ok = fused ? err <= tol : same;
    if (!ok) ++bad;
    std::printf("%-28s op=%c fused=%d max_abs=%.3e %s\n", name, opc, (int)fused, err,
                ok ? "ok" : "FAIL");
  }
  return bad;
}

// apply_device / simulate_device on cudaMalloc'd memory (the offload
// build's device-pointer surface) against QCLAB++'s CPU apply/simulate, for
// every op and a nonzero offset (the object acting on the upper qubits of a
// larger register).
template <typename T>
int run_device(const char* name, const qclab::QCircuit<T>& c, std::mt19937_64& rng, bool fused) {
  const int n = c.nbQubits() + 2, off = 2;
  std::normal_distribution<double> N01;
  std::vector<T> v(size_t(1) << n);
  for (auto& x : v) {
    if constexpr (qclab::is_complex_v<T>) x = T(N01(rng), N01(rng));
    else x = T(N01(rng));
  }
  const size_t bytes = v.size() * sizeof(T);
  T* d = nullptr;
  if (cudaMalloc(&d, bytes) != cudaSuccess) {
    std::printf("%-28s cudaMalloc failed\n", name);
    return 1;
  }
  const double tol = sizeof(qclab::real_t<T>) == 8 ? 1e-10 : 5e-5;
  int bad = 0;
  auto compare = [&](const char* what, char opc, const std::vector<T>& ref) {
    std::vector<T> gpu(v.size());
    cudaMemcpy(gpu.data(), d, bytes, cudaMemcpyDeviceToHost);
    double err = 0;
    bool same = true;
    for (size_t i = 0; i < v.size(); ++i) {
      err = std::max(err, (double)std::abs(ref[i] - gpu[i]));
      same = same && (ref[i] == gpu[i]);
    }
    const bool ok = fused ? err <= tol : same;
    if (!ok) ++bad;
    std::printf("%-28s %-15s op=%c fused=%d max_abs=%.3e %s\n", name, what, opc, (int)fused, err,
                ok ? "ok" : "FAIL");
  };
  for (char opc : {'N', 'T', 'C'}) {
    const qclab::Op op = static_cast<qclab::Op>(opc);
    std::vector<T> ref = v;
    c.apply(op, n, ref, off);  // QCLAB++ CPU path
    cudaMemcpy(d, v.data(), bytes, cudaMemcpyHostToDevice);
    qclab_b200::apply_device(c, op, n, d, off, fused);
    compare("apply_device", opc, ref);
  }
  {
    std::vector<T> w(size_t(1) << c.nbQubits());
    for (auto& x : w) {
      if constexpr (qclab::is_complex_v<T>) x = T(N01(rng), N01(rng));
      else x = T(N01(rng));
    }
    std::vector<T> ref = w;
    c.simulate(ref);
    v = w;
    cudaMemcpy(d, w.data(), w.size() * sizeof(T), cudaMemcpyHostToDevice);
    qclab_b200::simulate_device(c, d, fused);
    std::vector<T> gpu(w.size());
    cudaMemcpy(gpu.data(), d, w.size() * sizeof(T), cudaMemcpyDeviceToHost);
    double err = 0;
    bool same = true;
    for (size_t i = 0; i < w.size(); ++i) {
      err = std::max(err, (double)std::abs(ref[i] - gpu[i]));
      same = same && (ref[i] == gpu[i]);
    }
    const bool ok = fused ? err <= tol : same;
    if (!ok) ++bad;
    std::printf("%-28s %-15s op=N fused=%d max_abs=%.3e %s\n", name, "simulate_device",
                (int)fused, err, ok ? "ok" : "FAIL");
  }
  cudaFree(d);
  return bad;
}

template <typename T>
qclab::QCircuit<T> mixed(int n, unsigned seed) {
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(0, 6.283185307179586);
  auto q = [&](int k) { return (int)(rng() % (unsigned)k); };
  qclab::QCircuit<T> c(n);
  static std::vector<std::unique_ptr<QGate1<T>>> keep;  // PointerGate1 targets
  for (int i = 0; i < 60; ++i) {
    const int a = q(n);
    int b = q(n);
    if (b == a) b = (a + 1) % n;
    const int cs = (int)(rng() & 1);
    switch (q(24)) {
      case 0: c.push_back(std::make_unique<Hadamard<T>>(a)); break;
      case 1: c.push_back(std::make_unique<PauliX<T>>(a)); break;
      case 2: c.push_back(std::make_unique<PauliY<T>>(a)); break;
      case 3: c.push_back(std::make_unique<PauliZ<T>>(a)); break;
      case 4: c.push_back(std::make_unique<RotationX<T>>(a, U(rng))); break;
      case 5: c.push_back(std::make_unique<RotationY<T>>(a, U(rng))); break;
      case 6: c.push_back(std::make_unique<RotationZ<T>>(a, U(rng))); break;
      case 7: c.push_back(std::make_unique<Phase<T>>(a, U(rng))); break;
      case 8: c.push_back(std::make_unique<Phase45<T>>(a)); break;
      case 9: c.push_back(std::make_unique<Phase90<T>>(a)); break;
      case 10: c.push_back(std::make_unique<CX<T>>(a, b, cs)); break;
      case 11: c.push_back(std::make_unique<CY<T>>(a, b, cs)); break;
      case 12: c.push_back(std::make_unique<CZ<T>>(a, b, cs)); break;
      case 13: c.push_back(std::make_unique<CPhase<T>>(a, b, U(rng), cs)); break;
      case 14: c.push_back(std::make_unique<CRotationX<T>>(a, b, U(rng), cs)); break;
      case 15: c.push_back(std::make_unique<CRotationY<T>>(a, b, U(rng), cs)); break;
      case 16: c.push_back(std::make_unique<CRotationZ<T>>(a, b, U(rng), cs)); break;
      case 17: c.push_back(std::make_unique<SWAP<T>>(a, b)); break;
      case 18: c.push_back(std::make_unique<iSWAP<T>>(a, b)); break;
      case 19: c.push_back(std::make_unique<RotationXX<T>>(a, b, U(rng))); break;
      case 20: c.push_back(std::make_unique<RotationYY<T>>(a, b, U(rng))); break;
      case 21: c.push_back(std::make_unique<RotationZZ<T>>(a, b, U(rng))); break;
      case 22: c.push_back(std::make_unique<UserGate2<T>>(a, b)); break;
      default: {
        keep.push_back(std::make_unique<RotationY<T>>(0, U(rng)));
        if (a + 0 < n) c.push_back(std::make_unique<PointerGate1<T>>(keep.back().get(), a));
      }
    }
  }
  return c;
}

int main() {
  using C = std::complex<double>;
  using F = std::complex<float>;
  std::mt19937_64 rng(7);
  int bad = 0;
  for (bool fused : {false, true}) {
    {
      qclab::QCircuit<C> c(9);
      auto sub = std::make_unique<qclab::QCircuit<C>>(4, 3);  // nested, offset 3
      sub->push_back(std::make_unique<Hadamard<C>>(0));
      sub->push_back(std::make_unique<CX<C>>(0, 3));
      sub->push_back(std::make_unique<RotationZ<C>>(2, 0.7));
      c.push_back(std::make_unique<RotationY<C>>(8, 0.2));
      c.push_back(std::move(sub));
      c.push_back(std::make_unique<CZ<C>>(8, 0));
      bad += run("nested-offset-circuit", c, rng, fused);
    }
    bad += run("mixed12-complex<double>", mixed<C>(12, 1), rng, fused);
    bad += run("mixed10-complex<float>", mixed<F>(10, 2), rng, fused);
    bad += run_device("device-mixed11-c<double>", mixed<C>(11, 3), rng, fused);
    bad += run_device("device-mixed9-c<float>", mixed<F>(9, 4), rng, fused);
  }
  std::printf("adapter_test: %s\n", bad ? "FAILED" : "all passed");
  return bad ? 1 : 0;
}

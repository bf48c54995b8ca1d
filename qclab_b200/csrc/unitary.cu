// Unitaries on the device.  Replaces QObject<T>::apply(Side, Op, nbQubits,
// SquareMatrix<T>&, offset) (QCircuit.hpp:176-204, per gate e.g.
// src/qgates/QGate1.cpp:27-80), QCircuit::matrix() (QCircuit.hpp:120-126)
// and nrmF (QCircuit.hpp:407-430).
//
// A 2^n x 2^n matrix is held column-major -- entry (r, c) at r + c 2^n, the
// layout of qclab::dense::SquareMatrix -- in a state object of 2n qubits.
// Bit b of the row index is index bit b and bit b of the column index is
// index bit n + b.  With qubit Q of the 2n-qubit object at index bit 2n-1-Q,
// qubit q of the rows is Q = n + q and qubit q of the columns is Q = q, so
// every matrix update is a state-vector sweep of the existing kernels:
//   Right  matrix <- op(G) matrix  :  op(G) on qubits offset + n + q
//   Left   matrix <- matrix op(G)  :  op(G)^T on qubits offset + q, i.e.
//          NoTrans -> Trans, Trans -> NoTrans, ConjTrans -> conj, NoTrans, conj
// The gate order per (side, op) follows QCircuit::apply(Side, ...): Right
// NoTrans and Left [Conj]Trans run the gates forwards, the other two in
// reverse, which is what the state sweep does for the mapped op.
#include <algorithm>
#include <cmath>
#include "internal.hpp"
#include "tile.cuh"

namespace qsv {
namespace {

constexpr int kThreads = 512;
constexpr int kBlocks = 148 * 8;

template <typename V>
__global__ void __launch_bounds__(kThreads) k_identity(V* __restrict__ m, uint64_t N, uint64_t dim1) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
       i += (uint64_t)gridDim.x * blockDim.x)
    m[i] = from_d2<V>(make_double2(i % dim1 == 0 ? 1.0 : 0.0, 0.0));
}

template <typename V>
__global__ void __launch_bounds__(kThreads) k_conj(V* __restrict__ m, uint64_t N) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 v = to_d2(m[i]);
    m[i] = from_d2<V>(make_double2(v.x, -v.y));
  }
}

// pass 1: per-block max |a - b|
template <typename VA, typename VB>
__global__ void __launch_bounds__(kThreads)
k_diff_max(const VA* __restrict__ a, const VB* __restrict__ b, uint64_t N, double* __restrict__ part) {
  __shared__ double mx[32];
  double m = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 x = to_d2(a[i]), y = to_d2(b[i]);
    m = fmax(m, hypot(x.x - y.x, x.y - y.y));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) mx[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double bm = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) bm = fmax(bm, mx[w]);
    part[blockIdx.x] = bm;
  }
}

// final max; a zero maximum becomes 1 (the reference's scale rule)
__global__ void __launch_bounds__(1024) k_scale_of(const double* __restrict__ part, int count,
                                                   double* __restrict__ scale) {
  __shared__ double mx[32];
  double m = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) m = fmax(m, part[i]);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) mx[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double bm = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) bm = fmax(bm, mx[w]);
    *scale = bm == 0.0 ? 1.0 : bm;
  }
}

// pass 2: per-block sum of |(a - b) / scale|^2
template <typename VA, typename VB>
__global__ void __launch_bounds__(kThreads)
k_diff_sum(const VA* __restrict__ a, const VB* __restrict__ b, uint64_t N,
           const double* __restrict__ scale, double2* __restrict__ part) {
  __shared__ double2 red[32];
  const double s = *scale;
  double acc = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 x = to_d2(a[i]), y = to_d2(b[i]);
    const double re = (x.x - y.x) / s, im = (x.y - y.y) / s;
    acc = fma(re, re, fma(im, im, acc));
  }
  const double2 t = block_sum(make_double2(acc, 0.0), red);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void __launch_bounds__(1024) k_sum_rows(const double2* __restrict__ part, int count,
                                                   double2* __restrict__ out) {
  __shared__ double2 red[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) acc += part[i].x;
  const double2 t = block_sum(make_double2(acc, 0.0), red);
  if (threadIdx.x == 0) *out = t;
}

unsigned blocks_for(uint64_t N) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(kBlocks, (N + kThreads - 1) / kThreads));
}

template <typename V>
qsv_status identity_typed(qsv_state_s* s) {
  const uint64_t N = dim(s->n), d1 = dim(s->n / 2) + 1;
  k_identity<V><<<blocks_for(N), kThreads, 0, s->stream>>>(static_cast<V*>(s->d), N, d1);
  count_launch();
  return cuda_status(cudaGetLastError(), "identity launch");
}

template <typename V>
qsv_status conj_typed(qsv_state_s* s) {
  const uint64_t N = dim(s->n);
  k_conj<V><<<blocks_for(N), kThreads, 0, s->stream>>>(static_cast<V*>(s->d), N);
  count_launch();
  return cuda_status(cudaGetLastError(), "conjugate launch");
}

qsv_status conj_state(qsv_state_s* s) {
  switch (s->dtype) {
    case QSV_C128: return conj_typed<double2>(s);
    case QSV_C64:  return conj_typed<float2>(s);
    default:       return QSV_SUCCESS;  // real matrices are their own conjugate
  }
}

template <typename VA, typename VB>
qsv_status nrmf_typed(qsv_state_s* a, qsv_state_s* b, double* out) {
  const uint64_t N = dim(a->n);
  const unsigned blocks = blocks_for(N);
  // [blocks] maxima | scale | pad to 16 B | [blocks] double2 sums | total
  const size_t sum_off = ((blocks + 1) * sizeof(double) + 15) & ~size_t(15);
  const size_t bytes = sum_off + (blocks + 1) * sizeof(double2);
  if (qsv_status st = ensure_scratch(a, bytes)) return st;
  double* pmax = static_cast<double*>(a->scratch);
  double* scale = pmax + blocks;
  double2* psum = reinterpret_cast<double2*>(static_cast<unsigned char*>(a->scratch) + sum_off);
  const VA* da = static_cast<const VA*>(a->d);
  const VB* db = static_cast<const VB*>(b->d);
  k_diff_max<VA, VB><<<blocks, kThreads, 0, a->stream>>>(da, db, N, pmax);
  k_scale_of<<<1, 1024, 0, a->stream>>>(pmax, (int)blocks, scale);
  k_diff_sum<VA, VB><<<blocks, kThreads, 0, a->stream>>>(da, db, N, scale, psum);
  k_sum_rows<<<1, 1024, 0, a->stream>>>(psum, (int)blocks, psum + blocks);
  count_launch(4);
  if (qsv_status st = cuda_status(cudaGetLastError(), "nrmF launch")) return st;
  double h[2];
  double2 t;
  if (qsv_status st = cuda_status(cudaMemcpyAsync(h, scale, sizeof(double), cudaMemcpyDeviceToHost,
                                                  a->stream), "nrmF copy"))
    return st;
  if (qsv_status st = cuda_status(cudaMemcpyAsync(&t, psum + blocks, sizeof(t),
                                                  cudaMemcpyDeviceToHost, a->stream), "nrmF copy"))
    return st;
  if (qsv_status st = cuda_status(cudaStreamSynchronize(a->stream), "nrmF synchronize")) return st;
  *out = h[0] * std::sqrt(t.x);
  return QSV_SUCCESS;
}

template <typename VA>
qsv_status nrmf_b(qsv_state_s* a, qsv_state_s* b, double* out) {
  switch (b->dtype) {
    case QSV_C128: return nrmf_typed<VA, double2>(a, b, out);
    case QSV_C64:  return nrmf_typed<VA, float2>(a, b, out);
    case QSV_F64:  return nrmf_typed<VA, double>(a, b, out);
    case QSV_F32:  return nrmf_typed<VA, float>(a, b, out);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

qsv_status check_matrix(qsv_state_s* s) {
  if (!s || !s->d) return fail(QSV_ERROR_INVALID_VALUE, "null matrix");
  if (s->n % 2) return fail(QSV_ERROR_SIZE, "a matrix object has an even number (2n) of qubits, got %d", s->n);
  return QSV_SUCCESS;
}

}  // namespace
}  // namespace qsv

using namespace qsv;

extern "C" {

qsv_status qsv_set_identity(qsv_state m) {
  if (qsv_status st = check_matrix(m)) return st;
  switch (m->dtype) {
    case QSV_C128: return identity_typed<double2>(m);
    case QSV_C64:  return identity_typed<float2>(m);
    case QSV_F64:  return identity_typed<double>(m);
    case QSV_F32:  return identity_typed<float>(m);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

qsv_status qsv_apply_matrix(qsv_state m, const qsv_gate* gates, size_t nGates, char side, char op,
                            int offset, int fused) {
  if (qsv_status st = check_matrix(m)) return st;
  const int n = m->n / 2;
  if (side != 'L' && side != 'R') return fail(QSV_ERROR_INVALID_VALUE, "side must be 'L' or 'R'");
  if (op != 'N' && op != 'T' && op != 'C') return fail(QSV_ERROR_INVALID_VALUE, "op must be 'N', 'T' or 'C'");
  if (offset < 0) return fail(QSV_ERROR_QUBIT, "negative offset");
  // gates must address the n matrix qubits, not the 2n of the storage object
  for (size_t k = 0; k < nGates; ++k) {
    const int hi = std::max(gates[k].qubit0, gates[k].qubit1) + offset;
    if (hi >= n) return fail(QSV_ERROR_QUBIT, "gate %zu acts on qubit %d of a %d-qubit matrix", k, hi, n);
  }
  auto sweep = [&](char o, int off) {
    return fused ? qsv_apply_fused(m, gates, nGates, o, off, nullptr)
                 : qsv_apply(m, gates, nGates, o, off);
  };
  if (side == 'R') return sweep(op, offset + n);
  if (op == 'N') return sweep('T', offset);
  if (op == 'T') return sweep('N', offset);
  if (qsv_status st = conj_state(m)) return st;
  if (qsv_status st = sweep('N', offset)) return st;
  return conj_state(m);
}

qsv_status qsv_nrmF(qsv_state a, qsv_state b, double* out) {
  if (!a || !a->d || !b || !b->d) return fail(QSV_ERROR_INVALID_VALUE, "null matrix");
  if (!out) return fail(QSV_ERROR_INVALID_VALUE, "null output");
  if (a->n != b->n) return fail(QSV_ERROR_SIZE, "nrmF: matrices differ in size");
  if (b->stream != a->stream)
    if (qsv_status st = cuda_status(cudaStreamSynchronize(b->stream), "nrmF stream sync")) return st;
  switch (a->dtype) {
    case QSV_C128: return nrmf_b<double2>(a, b, out);
    case QSV_C64:  return nrmf_b<float2>(a, b, out);
    case QSV_F64:  return nrmf_b<double>(a, b, out);
    case QSV_F32:  return nrmf_b<float>(a, b, out);
  }
  return fail(QSV_ERROR_INVALID_VALUE, "bad dtype");
}

}  // extern "C"

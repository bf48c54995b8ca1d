// C ABI entry points: library info, state vectors, gate application.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>
#include "common.cuh"
#include "fused.hpp"
#include "internal.hpp"

namespace qsv {

static thread_local char g_err[1024] = "";
static thread_local uint64_t g_launches = 0;
static thread_local uint64_t g_tma_launches = 0;

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

qsv_status fail(qsv_status st, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return st;
}

qsv_status cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return QSV_SUCCESS;
  set_error("%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? QSV_ERROR_OUT_OF_MEMORY : QSV_ERROR_CUDA;
}

void count_launch(uint64_t k) { g_launches += k; }
void count_tma_launch() { ++g_tma_launches; }

qsv_status stream_wait(cudaStream_t waiter, cudaStream_t producer) {
  if (waiter == producer) return QSV_SUCCESS;
  cudaEvent_t ev;
  if (qsv_status st = cuda_status(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming),
                                  "cudaEventCreateWithFlags"))
    return st;
  qsv_status st = cuda_status(cudaEventRecord(ev, producer), "cudaEventRecord");
  if (!st) st = cuda_status(cudaStreamWaitEvent(waiter, ev, 0), "cudaStreamWaitEvent");
  cudaEventDestroy(ev);  // released once the recorded work completes
  return st;
}

qsv_status ensure_aux(qsv_state_s* s, size_t bytes) {
  if (s->aux_bytes >= bytes) return QSV_SUCCESS;
  if (s->aux) {
    qsv_status st = cuda_status(cudaStreamSynchronize(s->stream), "aux resize synchronize");
    if (st) return st;
    cudaFree(s->aux);
    s->aux = nullptr;
    s->aux_bytes = 0;
  }
  cudaError_t e = cudaMalloc(&s->aux, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    s->aux = nullptr;
    return fail(QSV_ERROR_OUT_OF_MEMORY, "work-vector cudaMalloc of %zu bytes failed", bytes);
  }
  s->aux_bytes = bytes;
  return QSV_SUCCESS;
}

qsv_status ensure_scratch(qsv_state_s* s, size_t bytes) {
  if (s->scratch_bytes >= bytes) return QSV_SUCCESS;
  if (s->scratch) {
    // earlier kernels on the stream may still read the old buffer
    qsv_status st = cuda_status(cudaStreamSynchronize(s->stream), "scratch resize synchronize");
    if (st) return st;
    cudaFree(s->scratch);
    s->scratch = nullptr;
    s->scratch_bytes = 0;
  }
  size_t cap = 1 << 16;
  while (cap < bytes) cap <<= 1;
  cudaError_t e = cudaMalloc(&s->scratch, cap);
  if (e != cudaSuccess) {
    cudaGetLastError();
    s->scratch = nullptr;
    return fail(QSV_ERROR_OUT_OF_MEMORY, "scratch cudaMalloc of %zu bytes failed", cap);
  }
  s->scratch_bytes = cap;
  return QSV_SUCCESS;
}

namespace {

template <typename V>
__global__ void k_set_one(V* st, uint64_t index);
template <>
__global__ void k_set_one<double2>(double2* st, uint64_t index) { st[index] = make_double2(1.0, 0.0); }
template <>
__global__ void k_set_one<float2>(float2* st, uint64_t index) { st[index] = make_float2(1.f, 0.f); }
template <>
__global__ void k_set_one<double>(double* st, uint64_t index) { st[index] = 1.0; }
template <>
__global__ void k_set_one<float>(float* st, uint64_t index) { st[index] = 1.f; }

qsv_status set_basis(qsv_state_s* s, uint64_t index) {
  const size_t bytes = dim(s->n) * elem_bytes(s->dtype);
  qsv_status st = cuda_status(cudaMemsetAsync(s->d, 0, bytes, s->stream), "cudaMemsetAsync");
  if (st) return st;
  switch (s->dtype) {
    case QSV_C128: k_set_one<double2><<<1, 1, 0, s->stream>>>((double2*)s->d, index); break;
    case QSV_C64:  k_set_one<float2><<<1, 1, 0, s->stream>>>((float2*)s->d, index); break;
    case QSV_F64:  k_set_one<double><<<1, 1, 0, s->stream>>>((double*)s->d, index); break;
    case QSV_F32:  k_set_one<float><<<1, 1, 0, s->stream>>>((float*)s->d, index); break;
  }
  count_launch();
  return cuda_status(cudaGetLastError(), "set_basis kernel");
}

qsv_status check_state(qsv_state s) {
  if (!s) return fail(QSV_ERROR_INVALID_VALUE, "null state");
  if (!s->d) return fail(QSV_ERROR_INVALID_VALUE, "state has no device memory");
  return QSV_SUCCESS;
}

}  // namespace

qsv_status lower_for_state(const qsv_state_s* s, const qsv_gate* gates,
                           size_t count, char op, int offset,
                           std::vector<Lowered>* out, bool fp64) {
  if (!valid_op(op)) return fail(QSV_ERROR_INVALID_VALUE, "op must be 'N', 'T' or 'C' (got %d)", (int)op);
  if (count && !gates) return fail(QSV_ERROR_INVALID_VALUE, "null gate list");
  out->assign(count, Lowered());
  size_t bad = 0;
  qsv_status st = (fp64 || dtype_double(s->dtype))
      ? lower_list<double>(gates, count, op, offset, s->n, dtype_real(s->dtype), out->data(), &bad)
      : lower_list<float>(gates, count, op, offset, s->n, dtype_real(s->dtype), out->data(), &bad);
  if (st != QSV_SUCCESS) {
    const qsv_gate& g = gates[bad];
    if (st == QSV_ERROR_QUBIT)
      return fail(st, "gate %zu (kind %d): qubits (%d,%d)+offset %d outside [0,%d) or repeated",
                  bad, g.kind, g.qubit0, g.qubit1, offset, s->n);
    if (st == QSV_ERROR_DTYPE)
      return fail(st, "gate %zu (kind %d) has complex coefficients; not defined for a real state",
                  bad, g.kind);
    return fail(st, "gate %zu: invalid gate record (kind %d, control_state %d)", bad, g.kind,
                g.control_state);
  }
  return QSV_SUCCESS;
}

}  // namespace qsv

using namespace qsv;

extern "C" {

int qsv_abi_version(void) { return QSV_ABI_VERSION; }

const char* qsv_last_error(void) { return g_err; }

uint64_t qsv_launch_count(void) { return g_launches; }

uint64_t qsv_tma_launch_count(void) { return g_tma_launches; }

const char* qsv_status_string(qsv_status status) {
  switch (status) {
    case QSV_SUCCESS: return "QSV_SUCCESS";
    case QSV_ERROR_INVALID_VALUE: return "QSV_ERROR_INVALID_VALUE";
    case QSV_ERROR_QUBIT: return "QSV_ERROR_QUBIT";
    case QSV_ERROR_SIZE: return "QSV_ERROR_SIZE";
    case QSV_ERROR_CUDA: return "QSV_ERROR_CUDA";
    case QSV_ERROR_OUT_OF_MEMORY: return "QSV_ERROR_OUT_OF_MEMORY";
    case QSV_ERROR_DTYPE: return "QSV_ERROR_DTYPE";
    case QSV_ERROR_TIMEOUT: return "QSV_ERROR_TIMEOUT";
    case QSV_ERROR_NOT_SUPPORTED: return "QSV_ERROR_NOT_SUPPORTED";
  }
  return "QSV_ERROR_UNKNOWN";
}

qsv_status qsv_create(int nbQubits, qsv_dtype dtype, qsv_state* out) {
  if (!out) return fail(QSV_ERROR_INVALID_VALUE, "null output handle");
  *out = nullptr;
  if (!dtype_valid(dtype)) return fail(QSV_ERROR_INVALID_VALUE, "bad dtype %d", (int)dtype);
  if (nbQubits < 1 || nbQubits > kMaxQubits)
    return fail(QSV_ERROR_SIZE, "nbQubits %d outside [1,%d]", nbQubits, kMaxQubits);
  auto* s = new qsv_state_s();
  s->n = nbQubits;
  s->dtype = dtype;
  s->owns = true;
  cudaGetDevice(&s->device);
  const size_t bytes = dim(nbQubits) * elem_bytes(dtype);
  cudaError_t e = cudaMalloc(&s->d, bytes);
  if (e != cudaSuccess) {
    delete s;
    cudaGetLastError();
    return fail(QSV_ERROR_OUT_OF_MEMORY, "cudaMalloc of %zu bytes for a %d-qubit state failed: %s",
                bytes, nbQubits, cudaGetErrorString(e));
  }
  qsv_status st = set_basis(s, 0);
  if (st) {
    cudaFree(s->d);
    delete s;
    return st;
  }
  *out = s;
  return QSV_SUCCESS;
}

qsv_status qsv_wrap(int nbQubits, qsv_dtype dtype, void* device_ptr, qsv_state* out) {
  if (!out) return fail(QSV_ERROR_INVALID_VALUE, "null output handle");
  *out = nullptr;
  if (!device_ptr) return fail(QSV_ERROR_INVALID_VALUE, "null device pointer");
  if (!dtype_valid(dtype)) return fail(QSV_ERROR_INVALID_VALUE, "bad dtype %d", (int)dtype);
  if (nbQubits < 1 || nbQubits > kMaxQubits)
    return fail(QSV_ERROR_SIZE, "nbQubits %d outside [1,%d]", nbQubits, kMaxQubits);
  if (reinterpret_cast<uintptr_t>(device_ptr) % elem_bytes(dtype) != 0)
    return fail(QSV_ERROR_INVALID_VALUE, "device pointer not aligned to the element size");
  auto* s = new qsv_state_s();
  s->n = nbQubits;
  s->dtype = dtype;
  s->d = device_ptr;
  s->owns = false;
  cudaGetDevice(&s->device);
  *out = s;
  return QSV_SUCCESS;
}

qsv_status qsv_destroy(qsv_state s) {
  if (!s) return QSV_SUCCESS;
  qsv_status st = QSV_SUCCESS;
  if (s->scratch || s->aux) cudaStreamSynchronize(s->stream);
  if (s->scratch) cudaFree(s->scratch);
  if (s->aux) cudaFree(s->aux);
  if (s->owns && s->d) st = cuda_status(cudaFree(s->d), "cudaFree");
  delete s;
  return st;
}

qsv_status qsv_set_stream(qsv_state s, void* stream) {
  if (qsv_status st = check_state(s)) return st;
  s->stream = static_cast<cudaStream_t>(stream);
  return QSV_SUCCESS;
}

qsv_status qsv_info(qsv_state s, int* n, qsv_dtype* dtype, void** ptr) {
  if (qsv_status st = check_state(s)) return st;
  if (n) *n = s->n;
  if (dtype) *dtype = s->dtype;
  if (ptr) *ptr = s->d;
  return QSV_SUCCESS;
}

qsv_status qsv_upload(qsv_state s, const void* host, size_t bytes) {
  if (qsv_status st = check_state(s)) return st;
  if (!host) return fail(QSV_ERROR_INVALID_VALUE, "null host pointer");
  const size_t need = dim(s->n) * elem_bytes(s->dtype);
  if (bytes != need) return fail(QSV_ERROR_SIZE, "upload of %zu bytes, state holds %zu", bytes, need);
  qsv_status st = cuda_status(cudaMemcpyAsync(s->d, host, bytes, cudaMemcpyHostToDevice, s->stream),
                              "upload cudaMemcpyAsync");
  if (st) return st;
  return cuda_status(cudaStreamSynchronize(s->stream), "upload synchronize");
}

qsv_status qsv_download(qsv_state s, void* host, size_t bytes) {
  if (qsv_status st = check_state(s)) return st;
  if (!host) return fail(QSV_ERROR_INVALID_VALUE, "null host pointer");
  const size_t need = dim(s->n) * elem_bytes(s->dtype);
  if (bytes != need) return fail(QSV_ERROR_SIZE, "download of %zu bytes, state holds %zu", bytes, need);
  qsv_status st = cuda_status(cudaMemcpyAsync(host, s->d, bytes, cudaMemcpyDeviceToHost, s->stream),
                              "download cudaMemcpyAsync");
  if (st) return st;
  if ((st = cuda_status(cudaStreamSynchronize(s->stream), "download synchronize"))) return st;
  return tc_check_status(s->stream);
}

qsv_status qsv_copy(qsv_state dst, qsv_state src) {
  if (qsv_status st = check_state(dst)) return st;
  if (qsv_status st = check_state(src)) return st;
  if (dst->n != src->n || dst->dtype != src->dtype)
    return fail(QSV_ERROR_SIZE, "qsv_copy: states differ in size or dtype");
  const size_t bytes = dim(src->n) * elem_bytes(src->dtype);
  // the copy runs on dst's stream: after src's pending work, and src's
  // later work waits for the copy to finish reading it
  if (qsv_status st = stream_wait(dst->stream, src->stream)) return st;
  if (qsv_status st = cuda_status(cudaMemcpyAsync(dst->d, src->d, bytes, cudaMemcpyDeviceToDevice,
                                                  dst->stream), "qsv_copy"))
    return st;
  return stream_wait(src->stream, dst->stream);
}

qsv_status qsv_set_basis(qsv_state s, uint64_t index) {
  if (qsv_status st = check_state(s)) return st;
  if (index >= dim(s->n)) return fail(QSV_ERROR_SIZE, "basis index %llu >= 2^%d",
                                      (unsigned long long)index, s->n);
  return set_basis(s, index);
}

qsv_status qsv_synchronize(qsv_state s) {
  if (qsv_status st = check_state(s)) return st;
  if (qsv_status st = cuda_status(cudaStreamSynchronize(s->stream), "qsv_synchronize")) return st;
  return tc_check_status(s->stream);
}

qsv_status qsv_apply(qsv_state s, const qsv_gate* gates, size_t nGates, char op, int offset) {
  if (qsv_status st = check_state(s)) return st;
  std::vector<Lowered> low;
  if (qsv_status st = lower_for_state(s, gates, nGates, op, offset, &low)) return st;
  for (const Lowered& L : low)
    if (qsv_status st = launch_unfused(s, L)) return st;
  return QSV_SUCCESS;
}

qsv_status qsv_apply_fused(qsv_state s, const qsv_gate* gates, size_t nGates, char op,
                           int offset, const qsv_fuse_opts* opts) {
  if (qsv_status st = check_state(s)) return st;
  std::vector<Lowered> low;
  // the fused sweeps multiply gates into dense matrices in FP64: lower every
  // gate in double (a complex<float> state's gates too), not in the state's
  // precision as the reference-exact path does
  if (qsv_status st = lower_for_state(s, gates, nGates, op, offset, &low, true)) return st;
  return run_fused(s, low, opts);
}

qsv_status qsv_apply_host(int nbQubits, qsv_dtype dtype, void* host, const qsv_gate* gates,
                          size_t nGates, char op, int offset, int fused) {
  if (!host) return fail(QSV_ERROR_INVALID_VALUE, "null host vector");
  qsv_state s = nullptr;
  if (qsv_status st = qsv_create(nbQubits, dtype, &s)) return st;
  const size_t bytes = dim(nbQubits) * elem_bytes(dtype);
  qsv_status st = qsv_upload(s, host, bytes);
  if (!st) st = fused ? qsv_apply_fused(s, gates, nGates, op, offset, nullptr)
                      : qsv_apply(s, gates, nGates, op, offset);
  if (!st) st = qsv_download(s, host, bytes);
  qsv_status st2 = qsv_destroy(s);
  return st ? st : st2;
}

}  // extern "C"

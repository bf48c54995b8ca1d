// Device capability probe: the FP64 tensor-core (mma.sync m8n8k4 f64) rate,
// the denominator of the fused complex sweep's tensor roofline.  Independent
// MMA chains per warp, no memory traffic besides one result per thread.
#include "internal.hpp"

namespace {

__global__ void __launch_bounds__(256) k_fp64_mma_rate(double* out, int iters) {
  const int l = threadIdx.x & 31;
  const double a = 1.0 + l * 1e-3, b = 1.0 - l * 1e-3;
  double c[8][2];
#pragma unroll
  for (int i = 0; i < 8; ++i) c[i][0] = c[i][1] = 0.0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%4, %5};"
                   : "=d"(c[i][0]), "=d"(c[i][1])
                   : "d"(a), "d"(b), "d"(c[i][0]), "d"(c[i][1]));
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += c[i][0] + c[i][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" qsv_status qsv_fp64_mma_peak(double* tflops) {
  using namespace qsv;
  if (!tflops) return fail(QSV_ERROR_INVALID_VALUE, "null output");
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8, threads = 256, iters = 4096;
  double* out = nullptr;
  if (qsv_status st = cuda_status(cudaMalloc(&out, sizeof(double) * blocks * threads), "probe buffer"))
    return st;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  qsv_status st = cuda_status(cudaEventCreate(&e0), "probe event");
  if (!st) st = cuda_status(cudaEventCreate(&e1), "probe event");
  if (!st) {
    k_fp64_mma_rate<<<blocks, threads>>>(out, 16);  // warm-up
    cudaEventRecord(e0);
    k_fp64_mma_rate<<<blocks, threads>>>(out, iters);
    cudaEventRecord(e1);
    count_launch(2);
    st = cuda_status(cudaEventSynchronize(e1), "probe run");
  }
  if (!st) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double flops = 2.0 * 256 * 8 * (double)iters * blocks * (threads / 32);
    *tflops = flops / (ms * 1e-3) / 1e12;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(out);
  return st;
}

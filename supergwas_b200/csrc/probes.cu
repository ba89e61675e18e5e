// probes.cu -- measured peaks that throughput figures are reported against:
// the FP64 FMA rate of the CUDA cores (the bound of the plain FP64 form) and
// the pinned host-to-device copy rate (the bound of the calls that stream
// rows from host memory).  Neither has a counterpart in the reference.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/kgwas_cuda.h"

namespace {

constexpr int kChains = 8;  // independent FMA chains per thread

// Each thread runs kChains independent dependency chains of DFMA; the
// results feed one conditional store so that nothing is optimised away.
__global__ void __launch_bounds__(256) dfma_loop(double* out, int iters, double a, double b) {
  double v[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) v[c] = 1.0 + 1e-3 * (threadIdx.x + c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = fma(v[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += v[c];
  if (s == -1.0) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // never true: v stays near 1
}

}  // namespace

extern "C" int kg_probe_fp64_tflops(int device, double* tflops) {
  if (!tflops) return KG_ERR_INVALID;
  *tflops = 0.0;
  if (cudaSetDevice(device) != cudaSuccess) return KG_ERR_CUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = sms * 8, threads = 256, iters = 1 << 14;
  double* out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * threads * sizeof(double)) != cudaSuccess) return KG_ERR_NOMEM;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = KG_OK;
  float best_ms = 0.0f;
  for (int rep = 0; rep < 4 && rc == KG_OK; ++rep) {  // the first launch warms up
    cudaEventRecord(e0);
    dfma_loop<<<blocks, threads>>>(out, iters, 0.999999, 1e-6);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = KG_ERR_CUDA;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && (best_ms == 0.0f || ms < best_ms)) best_ms = ms;
  }
  if (rc == KG_OK && best_ms > 0.0f)
    *tflops = 2.0 * kChains * (double)iters * blocks * threads / (best_ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return rc;
}

extern "C" int kg_probe_h2d_gbs(int device, uint64_t bytes, int reps, double* gbs) {
  if (!gbs || bytes == 0 || reps < 1) return KG_ERR_INVALID;
  *gbs = 0.0;
  if (cudaSetDevice(device) != cudaSuccess) return KG_ERR_CUDA;
  void* h = nullptr;
  void* d = nullptr;
  if (cudaHostAlloc(&h, bytes, cudaHostAllocDefault) != cudaSuccess) return KG_ERR_NOMEM;
  if (cudaMalloc(&d, bytes) != cudaSuccess) {
    cudaFreeHost(h);
    return KG_ERR_NOMEM;
  }
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = KG_OK;
  // warm-up copy, then `reps` copies of `bytes`, one cudaMemcpyAsync each
  if (cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = KG_ERR_CUDA;
  cudaEventRecord(e0, st);
  for (int r = 0; r < reps && rc == KG_OK; ++r)
    if (cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = KG_ERR_CUDA;
  cudaEventRecord(e1, st);
  if (cudaEventSynchronize(e1) != cudaSuccess) rc = KG_ERR_CUDA;
  if (rc == KG_OK) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms > 0.0f) *gbs = (double)bytes * reps / (ms * 1e-3) / 1e9;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  cudaFree(d);
  cudaFreeHost(h);
  return rc;
}

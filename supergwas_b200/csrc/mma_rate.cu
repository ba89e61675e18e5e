// mma_rate.cu -- measurement program (bin/mma_rate): the rate of back-to-back
// tcgen05.mma kind::i8 instructions per SM for M = 128 or 64 and several N,
// with A from tensor memory (M = 128) or shared memory.  One CTA per SM; thread 0 issues 4096
// MMAs, commits them to an mbarrier, waits (bounded, 2 s) and records the
// cycles.  It sets the ceiling of the association kernels: an instruction
// costs max(~62 cycles, N / 2 cycles), so N = 64 reaches half the int8 peak.
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#include "device.cuh"
using namespace kg;

template <int M, int N, bool ASMEM, int NACC>
__global__ void __launch_bounds__(128, 1) mma_bench(int iters, unsigned long long* out) {
  static_assert(M == 128 || ASMEM, "A from tensor memory is measured at M = 128 only");
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* g = smem_raw + (base - raw);
  const uint32_t sB = base, sA = base + N * 32 * 8, bar = sA + 4096 * 8;
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x;
  for (int i = tid; i < (N * 32 * 8 + 4096 * 8) / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(g)[i] = 0x01010101u * (i & 3);
  if (tid < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&s_tmem)) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) { mbar_init(bar, 1); mbar_fence_init(); }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  if (tid == 0) {
    constexpr uint32_t IDESC = idesc_i8(M, N);
    const uint64_t bdesc0 = sdesc_noswz(sB, N * 16, 128);
    const uint64_t adesc0 = sdesc_noswz(sA, M * 16, 128);
    constexpr uint32_t BSTEP = (2 * N * 16) >> 4, ASTEP = (2 * M * 16) >> 4;
    const unsigned long long t0 = clock64();
    for (int it = 0; it < iters; ++it) {
      const int st = it & 7;
      const uint32_t d = tmem + (it % NACC) * N;
      if (ASMEM) tc_mma_i8_ss(d, adesc0 + st * ASTEP, bdesc0 + st * BSTEP, IDESC, it >= NACC ? 1u : 0u);
      else tc_mma_i8_ts(d, tmem + 384 + st * 8, bdesc0 + st * BSTEP, IDESC, it >= NACC ? 1u : 0u);
    }
    const unsigned long long t1 = clock64();
    tc_commit(bar);
    unsigned long long dummy[4] = {0, 0, 0, 0};
    mbar_wait(bar, 0, dummy, 1);
    const unsigned long long t2 = clock64();
    out[3 * blockIdx.x] = t1 - t0;
    out[3 * blockIdx.x + 1] = t2 - t0;
    out[3 * blockIdx.x + 2] = dummy[2];
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (tid < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

template <int M, int N, bool ASMEM, int NACC>
void run(const char* name) {
  int iters = 4096;
  unsigned long long* d;
  cudaMalloc(&d, 148 * 3 * 8);
  const int need = N * 32 * 8 + 4096 * 8 + 8 + 1024;
  const int smem = need > 120 * 1024 ? need : 120 * 1024;  // one CTA per SM
  cudaFuncSetAttribute(mma_bench<M, N, ASMEM, NACC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  for (int rep = 0; rep < 3; ++rep) mma_bench<M, N, ASMEM, NACC><<<148, 128, smem>>>(iters, d);
  cudaError_t e = cudaDeviceSynchronize();
  unsigned long long h[148 * 3];
  cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  double issue = 0, total = 0;
  unsigned long long err = 0;
  for (int b = 0; b < 148; ++b) { issue += h[3 * b]; total += h[3 * b + 1]; err |= h[3 * b + 2]; }
  issue /= 148.0 * iters;
  total /= 148.0 * iters;
  const double macs = (double)M * N * 32;
  printf("%-22s M=%3d N=%3d  issue %.1f cyc/MMA  complete %.1f cyc/MMA  %.0f MAC/cyc/SM (%.1f%% of 8192)  %s err=%llu\n", name, M, N,
         issue, total, macs / total, 100.0 * macs / total / 8192.0, cudaGetErrorString(e), err);
  cudaFree(d);
}

int main() {
  run<128, 32, false, 1>("A tmem");
  run<128, 64, false, 1>("A tmem");
  run<128, 128, false, 1>("A tmem");
  run<128, 256, false, 1>("A tmem");
  run<128, 64, false, 2>("A tmem, 2 accum");
  run<128, 64, false, 4>("A tmem, 4 accum");
  run<128, 64, true, 1>("A smem");
  run<128, 128, true, 1>("A smem");
  run<128, 256, true, 1>("A smem");
  run<64, 64, true, 1>("A smem");
  run<64, 128, true, 1>("A smem");
  run<64, 256, true, 1>("A smem");
  return 0;
}

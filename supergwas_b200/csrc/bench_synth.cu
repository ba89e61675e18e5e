// bench_synth.cu -- seeded synthetic k-mer batches generated on the device in
// the packed row layout (libkgwas_bench.so; bench and test input, not part
// of the association library).
//
// Model (the Balding-Nichols generator of the benchmark configurations):
// k-mer j has an ancestral frequency p ~ Beta(0.5, 0.5), drawn as
// sin^2(pi u / 2) (the arcsine law), and per subpopulation s a frequency
// p_s ~ Beta(p (1 - F) / F, (1 - p)(1 - F) / F) with F = 0.1, drawn as
// G_a / (G_a + G_b) from two gamma variates (Marsaglia and Tsang, "A simple
// method for generating gamma variables", ACM TOMS 26(3), 2000; shapes
// below 1 through G(a) = G(a + 1) U^(1/a)).  Sample i belongs to
// subpopulation floor(i S / n) and carries the k-mer with probability
// p_s.  Every random number is a hash of (seed, k-mer index, draw index)
// (the "lowbias32" integer hash of Wellons' hash-prospector, applied to a
// Weyl sequence), so any chunk of k-mers can be regenerated on its own.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
// Uniform in (0, 1) from (key, draw).
__device__ __forceinline__ float unif(uint32_t key, uint32_t draw) {
  const uint32_t h = hash32(key ^ hash32(draw * 0x9e3779b9u + 0x632be5abu));
  return ((h >> 8) + 0.5f) * (1.0f / 16777216.0f);
}
__device__ __forceinline__ float normal(uint32_t key, uint32_t draw) {  // Box-Muller
  const float u1 = unif(key, draw), u2 = unif(key, draw + 1u);
  return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}
__device__ float gamma_draw(float a, uint32_t key, uint32_t draw) {
  float boost = 1.0f;
  if (a < 1.0f) {
    boost = powf(unif(key, draw), 1.0f / a);
    a += 1.0f;
    draw += 1u;
  }
  const float d = a - 1.0f / 3.0f, c = rsqrtf(9.0f * d);
  for (int it = 0; it < 64; ++it, draw += 3u) {
    const float z = normal(key, draw);
    float v = 1.0f + c * z;
    if (v <= 0.0f) continue;
    v = v * v * v;
    const float u = unif(key, draw + 2u);
    if (logf(u) < 0.5f * z * z + d - d * v + d * logf(v)) return boost * d * v;
  }
  return boost * d;  // not reached in practice (acceptance rate > 95 %)
}

constexpr float kFst = 0.1f;

// One warp per k-mer: lanes 0..S-1 draw the subpopulation frequencies, then
// the lanes write the row's words, lane l words l, l + 32, ...
__global__ void __launch_bounds__(256) synth_rows(uint64_t* __restrict__ out, unsigned long long m, int n, int wpk,
                                                  int S, unsigned long long first, unsigned long long seed) {
  __shared__ float s_ps[8][32];  // the subpopulation frequencies of each warp's k-mer
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x >> 5);
  const float cf = (1.0f - kFst) / kFst;
  for (unsigned long long j = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < m; j += warps) {
    const unsigned long long g = first + j;
    const uint32_t key = hash32((uint32_t)g ^ hash32((uint32_t)(g >> 32) + 0x51ed27u) ^ (uint32_t)seed) ^
                         hash32((uint32_t)(seed >> 32) + 0x2545f491u);
    const float u0 = unif(key, 0x7fffffffu);
    float p = sinpif(0.5f * u0);
    p = fminf(fmaxf(p * p, 1e-6f), 1.0f - 1e-6f);
    __syncwarp();
    if (lane < S) {
      const float ga = gamma_draw(p * cf, key, 0x10000000u + 512u * lane);
      const float gb = gamma_draw((1.0f - p) * cf, key, 0x20000000u + 512u * lane);
      s_ps[wib][lane] = ga + gb > 0.0f ? ga / (ga + gb) : 0.5f;
    }
    __syncwarp();
    for (int w = lane; w < wpk; w += 32) {
      uint64_t word = 0;
      const int i0 = 64 * w;
      if (i0 < n) {
        const int i1 = i0 + 64 < n ? i0 + 64 : n;
        int sp = (int)(((long long)i0 * S) / n);                       // subpopulation of sample i0
        long long next = ((long long)(sp + 1) * n + S - 1) / S;         // first sample of the next one
        float pr = s_ps[wib][sp];
        for (int i = i0; i < i1; ++i) {
          while (i >= next) {
            ++sp;
            next = ((long long)(sp + 1) * n + S - 1) / S;
            pr = s_ps[wib][sp];
          }
          if (unif(key, (uint32_t)i) < pr) word |= 1ull << (i - i0);
        }
      }
      out[j * (unsigned long long)wpk + w] = word;
    }
  }
}

}  // namespace

// Rows first .. first + m - 1 of the seeded batch (n samples, S
// subpopulations) into d_out (m x wpk words, device).  0 on success.
extern "C" int kg_synth_rows(uint64_t* d_out, uint64_t m, int n, int wpk, int S, uint64_t first, uint64_t seed,
                             void* stream) {
  if (!d_out || n <= 0 || wpk * 64 < n || S < 1 || S > 32) return 1;
  if (m == 0) return 0;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  unsigned long long blocks = (m + 7) / 8;  // 8 warps (k-mers) per block
  if (blocks > (unsigned long long)sms * 64) blocks = (unsigned long long)sms * 64;
  synth_rows<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(d_out, m, n, wpk, S, first, seed);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

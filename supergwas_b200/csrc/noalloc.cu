// noalloc.cu -- an association-test entry point that allocates no device memory.
//
// Who needs it: callers that are not allowed to allocate GPU memory
// themselves or through this library.  Examples are a host framework that
// hands out every device byte from its own pool and forbids side
// allocations, a plugin loaded into such a process, and code whose device
// memory budget is fixed before it starts (a cudaMalloc there can fail, or
// can fragment a pool that another component relies on).
//
// How: the caller passes the packed rows (device memory) and a buffer for the
// emitted rows (device memory).  The only other device memory the split-
// precision test needs lives in the static array below: the launch's
// counters, the int8 limb image of U and y', the FP64 columns that the
// refinement of strong hits reads, and the list of those hits.  It is part of
// the library image, so every GPU that loads this library holds its
// KG_NOALLOC_SCRATCH_BYTES from module load until the process exits.
//
// The array's name, used in host code, is a host-side stand-in, not a device
// address.  Its device address is looked up with cudaGetSymbolAddress, with
// the device current, by the first call on each device (and again if that
// device's context has been destroyed and created anew since).  Make that
// first call on each device outside any stream capture.
//
// All calls share the one array and it keeps whatever the last call wrote:
// each call clears the counters before its kernels and rewrites the image, the
// columns and the list, so calls made one after the other are independent,
// but calls that overlap on the GPU (different streams, or different host
// threads on the same device) race on the array and must be serialised by the
// caller.
//
// Accuracy: the same as kg_set_structure + kg_launch_device.  k-mers whose
// split-form chi-square reaches 12 are recomputed in FP64 (the split form's
// quantisation of U would otherwise show in -log10 p at the 1e-6 level, since
// -log10 p grows like T / (2 ln 10)).  The refinement sums each byte's set
// samples in ascending order and adds the byte sums in row order: the sums
// the context path reads from its byte tables, without the tables (5 MB and
// more) in the scratch.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/kgwas_cuda.h"
#include "device.cuh"
#include "kernels.hpp"
#include "prep.hpp"

namespace {

constexpr size_t kCounterBytes = 256;  // tested, hits, error bits, candidates (+ padding)
constexpr size_t kImageOff = kCounterBytes;
constexpr size_t kColsOff = kImageOff + KG_NOALLOC_MAX_B_BYTES;
constexpr size_t kCandOff = kColsOff + KG_NOALLOC_MAX_V_BYTES;
constexpr size_t kScratchBytes = kCandOff + (size_t)KG_NOALLOC_MAX_REFINE * sizeof(unsigned long long);
static_assert(kScratchBytes == KG_NOALLOC_SCRATCH_BYTES, "scratch layout");
static_assert(kColsOff % 256 == 0 && kCandOff % 256 == 0, "scratch alignment");
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char kg_noalloc_scratch[kScratchBytes];

// ------------------------------------------------------ FP64 refinement
// One warp per candidate k-mer: the lanes own the FP64 columns [count,
// d_0 .. d_{k-1}, d_y] (V, sample-major, cm doubles per sample) and sum them
// over the row's set samples, one byte (8 samples) at a time from 0.0 in
// ascending sample order, the byte sums added in row order; then
// compute_hit (src/kgwas.cpp:44-56) in FP64 and the row is emitted when
// p <= p_thresh.
template <int CM>
__global__ void __launch_bounds__(256) noalloc_refine_kernel(const uint64_t* __restrict__ x, int wpk, int nwords,
                                                             const double* __restrict__ V,
                                                             const __grid_constant__ kg::EpiParams P,
                                                             const kg::DevOut O) {
  constexpr int JW = (CM + 31) / 32;
  const int lane = threadIdx.x & 31;
  const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x >> 5);
  unsigned long long ncand = O.counters[3];
  if (ncand > O.cand_cap) ncand = O.cand_cap;
  for (unsigned long long w = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < ncand;
       w += warps) {
    const unsigned long long g = O.cand[w];
    const uint64_t* row = x + (g - O.kmer_offset) * (unsigned long long)wpk;
    double acc[JW];
#pragma unroll
    for (int jj = 0; jj < JW; ++jj) acc[jj] = 0.0;
    for (int wd = 0; wd < nwords; ++wd) {
      const uint64_t bits = __ldg(row + wd);  // one address for the whole warp
      for (int t = 0; t < 8; ++t) {
        const unsigned byte = (unsigned)(bits >> (8 * t)) & 255u;
        if (!byte) continue;  // warp-uniform
        double part[JW];
#pragma unroll
        for (int jj = 0; jj < JW; ++jj) part[jj] = 0.0;
        const double* Vb = V + ((size_t)wd * 64 + 8 * t) * CM;
#pragma unroll
        for (int s = 0; s < 8; ++s) {
          if ((byte >> s) & 1u) {
#pragma unroll
            for (int jj = 0; jj < JW; ++jj) {
              const int j = lane + 32 * jj;
              if (j < CM) part[jj] += __ldg(Vb + (size_t)s * CM + j);
            }
          }
        }
#pragma unroll
        for (int jj = 0; jj < JW; ++jj) acc[jj] += part[jj];
      }
    }
    int c;
    double ss, ey;
    kg::refine_reduce<CM>(P, acc, lane, c, ss, ey);
    if (lane == 0) {
      const double xxM = (double)c - ss, xyM = P.b * (double)c + ey;
      double effect = 0, T = 0, p = 1;
      const double eps = 1e-12;
      if (xxM > eps && P.yyM > eps) {
        double r2 = (xyM * xyM) / (xxM * P.yyM);
        if (r2 < 0) r2 = 0;
        if (r2 >= 1) r2 = 1 - 1e-15;
        T = (double)P.n * log(1.0 / (1.0 - r2));
        p = erfc(sqrt(0.5 * T));
        effect = xyM / (xxM * P.yyM);
      }
      if (p <= P.p_thresh) {
        const unsigned long long slot = atomicAdd(O.counters + 1, 1ull);
        if (slot < O.hit_cap) {
          kg_hit h;
          h.kmer = g;
          h.effect = effect;
          h.pval = p;
          h.chisq = T;
          O.hits[slot] = h;
        } else {
          atomicOr(O.counters + 2, (unsigned long long)kg::ERR_HIT_OVERFLOW);
        }
      }
    }
  }
}

template <int CM>
cudaError_t launch_refine_cm(const uint64_t* x, int wpk, int nwords, const double* V, const kg::EpiParams& P,
                             const kg::DevOut& O, int num_sms, cudaStream_t st) {
  noalloc_refine_kernel<CM><<<(unsigned)(num_sms * 4), 256, 0, st>>>(x, wpk, nwords, V, P, O);
  return cudaGetLastError();
}

cudaError_t launch_refine(int cm, const uint64_t* x, int wpk, int nwords, const double* V, const kg::EpiParams& P,
                          const kg::DevOut& O, int num_sms, cudaStream_t st) {
  switch (cm) {
    case 8: return launch_refine_cm<8>(x, wpk, nwords, V, P, O, num_sms, st);
    case 12: return launch_refine_cm<12>(x, wpk, nwords, V, P, O, num_sms, st);
    case 16: return launch_refine_cm<16>(x, wpk, nwords, V, P, O, num_sms, st);
    case 20: return launch_refine_cm<20>(x, wpk, nwords, V, P, O, num_sms, st);
    case 24: return launch_refine_cm<24>(x, wpk, nwords, V, P, O, num_sms, st);
    case 28: return launch_refine_cm<28>(x, wpk, nwords, V, P, O, num_sms, st);
    case 36: return launch_refine_cm<36>(x, wpk, nwords, V, P, O, num_sms, st);
    case 44: return launch_refine_cm<44>(x, wpk, nwords, V, P, O, num_sms, st);
    case 52: return launch_refine_cm<52>(x, wpk, nwords, V, P, O, num_sms, st);
    case 68: return launch_refine_cm<68>(x, wpk, nwords, V, P, O, num_sms, st);
    default: return cudaErrorInvalidValue;
  }
}

// -------------------------------------------------- device address set-up
std::mutex g_mu;
struct DevScratch {
  CUcontext ctx = nullptr;      // the context the address belongs to
  unsigned char* ptr = nullptr;
};
DevScratch g_scratch[kMaxDevices];

int set_err(char* err, size_t len, int code, const std::string& m) {
  if (err && len) std::snprintf(err, len, "%s", m.c_str());
  return code;
}

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(p);
  }
  return fn;
}

// Device address of the scratch array on the current device `dev`: looked
// up once per device and context (a destroyed and re-created context gets
// the array at a new address, so the lookup is repeated then).
int scratch_for(int dev, unsigned char** out, char* err, size_t len) {
  if (dev < 0 || dev >= kMaxDevices) return set_err(err, len, KG_ERR_UNSUPPORTED, "device ordinal too large");
  std::lock_guard<std::mutex> lk(g_mu);
  CUcontext cur = nullptr;
  const CtxGetCurrentFn get = ctx_get_current();
  const bool know_ctx = get && get(&cur) == CUDA_SUCCESS && cur;
  DevScratch& d = g_scratch[dev];
  if (!d.ptr || !know_ctx || d.ctx != cur) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, kg_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_err(err, len, KG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    d.ptr = static_cast<unsigned char*>(p);
    d.ctx = know_ctx ? cur : nullptr;
  }
  *out = d.ptr;
  return KG_OK;
}

}  // namespace

extern "C" int kg_run_device_noalloc(const uint64_t* d_xbits, uint64_t n_kmers, uint32_t words_per_kmer,
                                     const double* U_colmajor, int n, int k, const double* y,
                                     double corr_threshold, double log10_thresh, kg_hit* d_hits,
                                     uint64_t hit_capacity, uint64_t* counts_out, void* stream, char* err,
                                     size_t err_len) {
  if (err && err_len) err[0] = '\0';
  if (!counts_out) return set_err(err, err_len, KG_ERR_INVALID, "counts_out is NULL");
  counts_out[0] = counts_out[1] = 0;
  if (n_kmers > 0 && !d_xbits) return set_err(err, err_len, KG_ERR_INVALID, "d_xbits is NULL");
  if (hit_capacity > 0 && !d_hits) return set_err(err, err_len, KG_ERR_INVALID, "d_hits is NULL");
  if (words_per_kmer == 0 || (words_per_kmer & 1u))
    return set_err(err, err_len, KG_ERR_INVALID, "words_per_kmer must be even and > 0");
  if ((uint64_t)words_per_kmer * 64 < (uint64_t)(n > 0 ? n : 0))
    return set_err(err, err_len, KG_ERR_INVALID, "words_per_kmer*64 < n");

  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return set_err(err, err_len, KG_ERR_CUDA, cudaGetErrorString(ce));
  int cc_major = 0, cc_minor = 0, num_sms = 0;
  cudaDeviceGetAttribute(&cc_major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&cc_minor, cudaDevAttrComputeCapabilityMinor, dev);
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (cc_major != 10 || cc_minor != 0)
    return set_err(err, err_len, KG_ERR_UNSUPPORTED, "needs an sm_100 (B200) device");
  unsigned char* scratch = nullptr;
  int rc = scratch_for(dev, &scratch, err, err_len);
  if (rc) return rc;

  // Host-side FP64 preparation of the structure (host memory only).
  kg::Prepared P;
  std::string e = kg::prepare(U_colmajor, n, k, y, P);
  if (!e.empty()) return set_err(err, err_len, KG_ERR_INVALID, e);
  kg::LimbCols L;
  e = kg::make_limbs(P, nullptr, n, 3, 5, kg::tc_kc(), L);
  if (!e.empty()) return set_err(err, err_len, KG_ERR_UNSUPPORTED, e);
  if (!kg::tc_supported_n(L.N))
    return set_err(err, err_len, KG_ERR_UNSUPPORTED,
                   "contraction width N=" + std::to_string(L.N) + " not supported by the tensor-core kernel");
  const size_t b_bytes = (size_t)L.Kpad * L.N;
  if (b_bytes > KG_NOALLOC_MAX_B_BYTES)
    return set_err(err, err_len, KG_ERR_UNSUPPORTED,
                   "structure needs " + std::to_string(b_bytes) + " bytes of device scratch (samples rounded up to " +
                       std::to_string(L.Kpad) + " x " + std::to_string(L.N) + " limb columns); the maximum is " +
                       std::to_string((size_t)KG_NOALLOC_MAX_B_BYTES));
  // FP64 columns of the refinement: [count, d_0 .. d_{k-1}, d_y] per sample,
  // samples rounded up to 128
  const int cm = kg::fp64_cm(k + 2);
  if (cm < 0) return set_err(err, err_len, KG_ERR_UNSUPPORTED, "too many U columns for the FP64 refinement");
  const int vrows = kg::fp64_steps(n) * 128;
  const size_t v_bytes = (size_t)vrows * cm * sizeof(double);
  if (v_bytes > KG_NOALLOC_MAX_V_BYTES)
    return set_err(err, err_len, KG_ERR_UNSUPPORTED,
                   "FP64 refinement columns need " + std::to_string(v_bytes) + " bytes of device scratch (" +
                       std::to_string(vrows) + " samples x " + std::to_string(cm) + " columns); the maximum is " +
                       std::to_string((size_t)KG_NOALLOC_MAX_V_BYTES));
  std::vector<int8_t> img;
  kg::make_b_image(L, kg::tc_kc(), img);
  std::vector<double> V((size_t)vrows * cm, 0.0);
  for (int i = 0; i < n; ++i) {
    V[(size_t)i * cm] = 1.0;
    for (int j = 0; j <= k; ++j) V[(size_t)i * cm + 1 + j] = P.d[(size_t)j * n + i];
  }

  kg::EpiParams ep;
  std::memset(&ep, 0, sizeof(ep));
  ep.n = n;
  ep.k = k;
  ep.b = P.b;
  ep.kappa = P.kappa;
  ep.yyM = P.yyM;
  ep.ynorm = P.ynorm;
  ep.corr_thr = corr_threshold;
  ep.p_thresh = std::pow(10.0, -log10_thresh);
  ep.r2_cand = -1.0;  // evaluate p for every tested k-mer below the refinement cut
  ep.refine = 1;
  ep.r2_ref = -std::expm1(-kg::REFINE_CHISQ / (double)n);
  ep.thr2_ynorm2 = corr_threshold * corr_threshold * P.ynorm * P.ynorm;
  for (int j = 0; j < k; ++j) {
    ep.a[j] = P.a[j];
    ep.g[j] = P.g[j];
  }
  kg::LimbMap lm;
  std::memset(&lm, 0, sizeof(lm));
  lm.N = L.N;
  lm.count_col = L.count_col;
  for (int j = 0; j <= k; ++j) {
    lm.first[j] = L.first[j];
    lm.nl[j] = L.nl[j];
    lm.scale[j] = L.scale[j];
  }
  kg::set_limb_consts(lm);

  cudaStream_t st = (cudaStream_t)stream;
  unsigned long long* counters = reinterpret_cast<unsigned long long*>(scratch);
  int8_t* bimg = reinterpret_cast<int8_t*>(scratch + kImageOff);
  double* dV = reinterpret_cast<double*>(scratch + kColsOff);
  unsigned long long* cand = reinterpret_cast<unsigned long long*>(scratch + kCandOff);
  if ((ce = cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), st)) != cudaSuccess ||
      (ce = cudaMemcpyAsync(bimg, img.data(), b_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (ce = cudaMemcpyAsync(dV, V.data(), v_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return set_err(err, err_len, KG_ERR_CUDA, cudaGetErrorString(ce));

  // The k-mers go through in pieces whose refinement candidates fit the
  // fixed list: first all at once; a piece whose candidates overflow the list
  // is undone (counters put back) and run again in halves.  Candidates are
  // rare (chi-square >= 12), so one piece is the usual case.
  unsigned long long h[4] = {0, 0, 0, 0};  // counters after the last completed piece
  const int nwords = vrows / 64;
  uint64_t s0 = 0, piece = n_kmers;
  while (s0 < n_kmers) {
    const uint64_t cnt = piece < n_kmers - s0 ? piece : n_kmers - s0;
    kg::DevOut O;
    std::memset(&O, 0, sizeof(O));
    O.counters = counters;
    O.hits = d_hits;
    O.hit_cap = hit_capacity;
    O.kmer_offset = s0;
    O.cand = cand;
    O.cand_cap = KG_NOALLOC_MAX_REFINE;
    const uint64_t* xs = d_xbits + s0 * words_per_kmer;
    kg::LaunchTc Lt{xs, cnt, (int)words_per_kmer, L.Kpad / kg::tc_kc(), bimg, &ep, &lm, &O, num_sms};
    if ((ce = cudaMemsetAsync(counters + 3, 0, sizeof(unsigned long long), st)) != cudaSuccess)
      return set_err(err, err_len, KG_ERR_CUDA, cudaGetErrorString(ce));
    if ((ce = kg::launch_tc(Lt, st)) != cudaSuccess)
      return set_err(err, err_len, KG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(ce));
    if ((ce = launch_refine(cm, xs, (int)words_per_kmer, nwords, dV, ep, O, num_sms, st)) != cudaSuccess)
      return set_err(err, err_len, KG_ERR_CUDA, std::string("refinement launch: ") + cudaGetErrorString(ce));
    unsigned long long c[4] = {0, 0, 0, 0};
    if ((ce = cudaMemcpyAsync(c, counters, sizeof(c), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(st)) != cudaSuccess)
      return set_err(err, err_len, KG_ERR_CUDA, cudaGetErrorString(ce));
    if (c[2] & ~(unsigned long long)(kg::ERR_HIT_OVERFLOW | kg::ERR_CAND_OVERFLOW)) {
      counts_out[0] = c[0];
      counts_out[1] = c[1];
      return set_err(err, err_len, KG_ERR_TIMEOUT, "a bounded device-side wait gave up");
    }
    if (c[3] > KG_NOALLOC_MAX_REFINE && cnt > 128) {
      // undo this piece: tested and hit counts and error bits as before it
      if ((ce = cudaMemcpyAsync(counters, h, sizeof(h), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
          (ce = cudaStreamSynchronize(st)) != cudaSuccess)
        return set_err(err, err_len, KG_ERR_CUDA, cudaGetErrorString(ce));
      piece = ((cnt / 2 + 127) / 128) * 128;
      continue;
    }
    std::memcpy(h, c, sizeof(h));
    s0 += cnt;
  }
  counts_out[0] = h[0];
  counts_out[1] = h[1];
  if (h[1] > hit_capacity)
    return set_err(err, err_len, KG_ERR_INVALID,
                   "hit buffer holds " + std::to_string(hit_capacity) + " rows, " + std::to_string(h[1]) +
                       " were found; call again with a larger buffer");
  return KG_OK;
}

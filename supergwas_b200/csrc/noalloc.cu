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
// precision kernel needs -- the int8 limb image of U and y' and the
// launch's counters -- lives in the static array below.  It is part of the
// library image, so every GPU that loads this library holds its
// KG_NOALLOC_SCRATCH_BYTES from module load until the process exits.
//
// The array's name, used in host code, is a host-side stand-in, not a device
// address.  Its device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, the first time the entry
// point runs on that device.  Make that first call on each device outside
// any stream capture.
//
// All calls share the one array and it keeps whatever the last call wrote:
// each call clears the counters before its kernel and rewrites the limb
// image, so calls made one after the other are independent, but calls that
// overlap on the GPU (different streams, or different host threads on the
// same device) race on the array and must be serialised by the caller.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/kgwas_cuda.h"
#include "kernels.hpp"
#include "prep.hpp"

namespace {

constexpr size_t kCounterBytes = 256;  // tested, hits, error bits (+ padding)
constexpr size_t kScratchBytes = kCounterBytes + KG_NOALLOC_MAX_B_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char kg_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
unsigned char* g_scratch[kMaxDevices] = {};

int set_err(char* err, size_t len, int code, const std::string& m) {
  if (err && len) std::snprintf(err, len, "%s", m.c_str());
  return code;
}

// Device address of the scratch array on the current device (looked up once).
int scratch_for(int dev, unsigned char** out, char* err, size_t len) {
  if (dev < 0 || dev >= kMaxDevices) return set_err(err, len, KG_ERR_UNSUPPORTED, "device ordinal too large");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, kg_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_err(err, len, KG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch[dev];
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
  std::vector<int8_t> img;
  kg::make_b_image(L, kg::tc_kc(), img);

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
  ep.r2_cand = -1.0;  // evaluate p for every tested k-mer
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
  int8_t* bimg = reinterpret_cast<int8_t*>(scratch + kCounterBytes);
  if ((ce = cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), st)) != cudaSuccess ||
      (ce = cudaMemcpyAsync(bimg, img.data(), b_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return set_err(err, err_len, KG_ERR_CUDA, cudaGetErrorString(ce));
  if (n_kmers > 0) {
    kg::DevOut O;
    std::memset(&O, 0, sizeof(O));
    O.counters = counters;
    O.hits = d_hits;
    O.hit_cap = hit_capacity;
    O.kmer_offset = 0;
    kg::LaunchTc Lt{d_xbits, n_kmers, (int)words_per_kmer, L.Kpad / kg::tc_kc(), bimg, &ep, &lm, &O, num_sms};
    if ((ce = kg::launch_tc(Lt, st)) != cudaSuccess)
      return set_err(err, err_len, KG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(ce));
  }
  unsigned long long h[3] = {0, 0, 0};
  if ((ce = cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (ce = cudaStreamSynchronize(st)) != cudaSuccess)
    return set_err(err, err_len, KG_ERR_CUDA, cudaGetErrorString(ce));
  counts_out[0] = h[0];
  counts_out[1] = h[1];
  if (h[2] & ~(unsigned long long)kg::ERR_HIT_OVERFLOW)
    return set_err(err, err_len, KG_ERR_TIMEOUT, "a bounded device-side wait gave up");
  if (h[1] > hit_capacity)
    return set_err(err, err_len, KG_ERR_INVALID,
                   "hit buffer holds " + std::to_string(hit_capacity) + " rows, " + std::to_string(h[1]) +
                       " were found; call again with a larger buffer");
  return KG_OK;
}

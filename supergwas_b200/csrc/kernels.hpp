// kernels.hpp -- host-side launch interface of the association kernels.
#pragma once
#include <cuda_runtime.h>

#include "params.hpp"

struct CUtensorMap_st;

namespace kg {

struct LaunchFp64 {
  const uint64_t* x;          // packed rows (device)
  unsigned long long m;       // k-mers in this launch
  int wpk;                    // words per k-mer
  const double* V;            // nsteps*128 x cm FP64, sample-major, zero padded (device)
  int nsteps, cm;             // sample steps of 128; padded column count
  const EpiParams* P;
  const DevOut* O;
  int num_sms;
  const double* T = nullptr;  // refinement byte tables of V (refine_table_len doubles; device)
};

struct LaunchTc {
  const uint64_t* x;
  unsigned long long m;
  int wpk;
  int nchunk;                 // K chunks of tc_kc() samples
  const int8_t* Bimg;         // B operand shared-memory image, chunk after chunk (device)
  const EpiParams* P;
  const LimbMap* LM;
  const DevOut* O;
  int num_sms;
};

int fp64_cm(int C);           // padded column count for C contraction columns (-1: too many)
int fp64_steps(int n);        // 128-sample steps covering n samples
cudaError_t launch_fp64(const LaunchFp64& L, cudaStream_t st);
// FP64 recomputation of the split form's refinement candidates from the
// byte tables of V (LaunchFp64::T).
cudaError_t launch_refine(const LaunchFp64& L, cudaStream_t st);

// Byte tables of the FP64 columns, one block per phenotype: for the 8-sample
// group g of a packed row and a byte value b, entry (g*256 + b)*cm + j is the
// sum of column j of V over the samples of g whose bit is set in b.
struct LaunchTable {
  const double* V;            // nblocks blocks of vrows x cm FP64 (vstride doubles apart)
  int vrows, cm;              // vrows a multiple of 128
  unsigned long long vstride;
  int nblocks;
  double* T;                  // nblocks blocks of refine_table_len(vrows, cm) doubles
};
size_t refine_table_len(int vrows, int cm);
cudaError_t launch_refine_table(const LaunchTable& L, cudaStream_t st);

struct LaunchTs {
  const uint64_t* x;          // packed rows (device), 16-byte aligned
  unsigned long long m;
  int wpk;
  int kpad;                   // samples covered by the B image (multiple of 128)
  bool drop0;                 // U column 0 has no limbs (intercept handled in FP64)
  const int8_t* Bimg;         // make_b_image_ts layout (device)
  const EpiParams* P;
  const LimbMap* LM;
  const DevOut* O;
  int num_sms;
};

// TMEM-A kernel: 3 limbs per U column, 5 for y', N <= 128, B resident in smem.
bool ts_supported(int N, int limbs_u, int limbs_y, int kpad, int wpk);
cudaError_t launch_ts(const LaunchTs& L, cudaStream_t st);

// (columns per phenotype slot, phenotypes per group) pairs with a compiled
// many-phenotype kernel; the group width NP * PPG is at most 128.
#define KG_MP_GROUPS(X)                                                                      \
  X(16, 1) X(16, 2) X(16, 4) X(16, 8) X(32, 1) X(32, 2) X(32, 4) X(48, 1) X(48, 2) X(64, 1) \
  X(64, 2) X(80, 1) X(96, 1) X(112, 1) X(128, 1)

struct LaunchMp {
  const uint64_t* x;          // packed rows (device), 16-byte aligned
  unsigned long long m;
  int wpk;
  int kpad;                   // samples per phenotype group image (multiple of 128)
  int NP;                     // columns per phenotype slot (multiple of 16, <= 128)
  int PPG;                    // phenotypes per group (KG_MP_GROUPS)
  int G;                      // phenotype groups
  int xs, nb;                 // resident x tiles (1-2), B ring stages (2-8)
  int splits, nacc;           // split-K accumulators, accumulator buffers (0: default)
  const int8_t* Bimg;         // G x (kpad/128) chunks of 128 x N bytes (device)
  const MPheno* ph;           // per-phenotype constants (device)
  const DevOutMP* O;
  int num_sms;
};
struct LaunchMpRefine {
  const uint64_t* x;
  int wpk;
  const double* V;            // n_pheno blocks of vrows x cm FP64 (device)
  int vrows, cm;
  unsigned long long vstride;
  const MPheno* ph;
  const DevOutMP* O;
  int num_sms;
  const double* T = nullptr;  // byte tables of V, refine_table_len(vrows, cm) doubles per phenotype
};
bool mp_supported(int NP, int PPG, int wpk);
size_t mp_smem_bytes(int nbox, int xs, int nb, int N);
cudaError_t launch_mp(const LaunchMp& L, cudaStream_t st);
// 2-D TMA map of packed rows: 128-byte x 128-row boxes, 128-byte swizzle.
bool mp_tmap(const uint64_t* x, unsigned long long m, int wpk, CUtensorMap_st* tm);

// B-stationary many-phenotype kernel (kernel_mpb.cu): each group's image
// (make_b_image_ts layout, kpad x NP*PPG bytes) resident in shared memory for
// a pass over `bt` tile-iterations of every CTA.
struct LaunchMpb {
  const uint64_t* x;
  unsigned long long m;
  int wpk;
  int kpad;
  int NP, PPG, G;
  int bt;                     // tile-iterations per L2 block
  const int8_t* Bimg;         // G images of kpad x NP*PPG bytes (device)
  const MPheno* ph;
  const DevOutMP* O;
  int num_sms;
};
bool mpb_supported(int NP, int PPG, int kpad, int wpk);  // the image and the x ring fit in shared memory
size_t mpb_smem_bytes(int N, int kpad);
cudaError_t launch_mpb(const LaunchMpb& L, cudaStream_t st);
cudaError_t launch_mp_refine(const LaunchMpRefine& L, cudaStream_t st);

// Pair-of-SMs many-phenotype kernel (kernel_mpb2.cu): a cluster of two CTAs
// issues M = 256 tcgen05 MMAs (cta_group::2) over two phenotypes at once
// (N = 2 * NP), each CTA holding one phenotype's image (kpad x NP, the
// one-phenotype-per-group image of LaunchMpb with PPG = 1; L.G = phenotypes)
// and 128 k-mers of each 256-k-mer pair-tile.
bool mpb2_supported(int NP, int kpad, int wpk);
size_t mpb2_smem_bytes(int NP, int kpad);
cudaError_t launch_mpb2(const LaunchMpb& L, cudaStream_t st);

// 2-D pair test (kernel_pairs.cu): the TMEM-A pipeline on x_i AND x_j.
struct LaunchPairs {
  const uint64_t* x;          // packed rows (device), 16-byte aligned, wpk >= 16
  int wpk;
  int kpad;
  bool drop0;
  PairSched S;
  const int8_t* Bimg;         // make_b_image_ts layout (device)
  const EpiParams* P;
  const LimbMap* LM;
  const DevOutPairs* O;
  int num_sms;
};
struct LaunchPairRefine {
  const uint64_t* x;
  int wpk;
  const double* T;            // byte tables of V (refine_table_len(vrows, cm) doubles)
  int vrows, cm;
  const EpiParams* P;
  const DevOutPairs* O;
  int num_sms;
};
bool pairs_supported(int N, int limbs_u, int limbs_y, int kpad, int wpk);
cudaError_t launch_pairs(const LaunchPairs& L, cudaStream_t st);
cudaError_t launch_pair_refine(const LaunchPairRefine& L, cudaStream_t st);

int tc_kc();                  // samples per K chunk of the tensor-core kernel
bool tc_supported_n(int N);
cudaError_t launch_tc(const LaunchTc& L, cudaStream_t st);

}  // namespace kg

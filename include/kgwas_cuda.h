/*
 * kgwas_cuda.h -- C ABI of the B200 k-mer association test.
 *
 * The reference exposes no library API: its boundary is the `kgwas` process
 * (src/kgwas.cpp:67-126), whose COLS mode runs, inside one process,
 *   build_overlap + load_Ubin      (src/kgwas_utils.hpp:129-157, 285-314)
 *   Pearson pre-filter             (src/kgwas.cpp:182-218)
 *   compute_cols_stats             (src/kgwas.cpp:138-166)
 *   compute_hit + emit selection   (src/kgwas.cpp:44-56, 225-259)
 *   .count                         (src/kgwas.cpp:291-304)
 * This header replaces the internal seam between the file readers and that
 * arithmetic.  The `kgwas` program in this package keeps the reference's
 * command line, readers and output text and calls these functions; other
 * hosts (Python via ctypes, a job runner) can call them directly.
 *
 * Conventions
 *   - Every function returns KG_OK (0) or a KG_ERR_* code and never exits
 *     the process; kg_last_error() describes the last failure of a context.
 *   - One context per GPU.  A context owns its device buffers and its CUDA
 *     stream; calls on it must not overlap, and it may pass from one host
 *     thread to another between calls (every call selects its GPU).
 *   - Packed k-mer rows: k-mer-major, `words_per_kmer` uint64 words per
 *     k-mer (even, so every row starts on a 16-byte boundary); overlap
 *     sample i is bit (i % 64) of word (i / 64); bits at i >= n are ignored.
 */
#ifndef KGWAS_CUDA_H
#define KGWAS_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KG_OK              0
#define KG_ERR_INVALID     1  /* bad argument or shape                       */
#define KG_ERR_CUDA        2  /* CUDA runtime / launch failure              */
#define KG_ERR_NOMEM       3  /* device or pinned host allocation failed     */
#define KG_ERR_STATE       4  /* call out of order (e.g. no structure set)   */
#define KG_ERR_TIMEOUT     5  /* a bounded device-side wait gave up          */
#define KG_ERR_UNSUPPORTED 6  /* shape outside what the kernel supports      */

/* Arithmetic of the contraction U^T x, x.y'. */
#define KG_PREC_SPLIT_I8 0  /* tcgen05 kind::i8: x exact in int8, U/y' split
                               into signed int8 limbs, exact int32 TMEM
                               accumulation, FP64 epilogue (default)        */
#define KG_PREC_FP64     1  /* plain FP64 on CUDA cores                      */

typedef struct kg_ctx kg_ctx;

typedef struct kg_opts {
    int device;             /* CUDA device ordinal                                 */
    int precision;          /* KG_PREC_*                                           */
    double corr_threshold;  /* CORR_THRESHOLD, default 0.2 (src/kgwas.cpp:30)      */
    double log10_thresh;    /* emit rows with p <= 10^-log10_thresh, default 6
                               (src/kgwas.cpp:28,230)                              */
    int limbs_u;            /* int8 limbs per U column (0 = default 3, at most 4)   */
    int limbs_y;            /* int8 limbs for y' (0 = default 5, at most 5)         */
} kg_opts;

/* One emitted row (src/kgwas.cpp:247-255): k-mer index within the call's
 * input, effect = xyM/(xxM*yyM), p = erfc(sqrt(T/2)), T the 1-df chi-square. */
typedef struct kg_hit {
    uint64_t kmer;
    double effect;
    double pval;
    double chisq;
} kg_hit;

typedef struct kg_result {
    uint64_t n_kmers;   /* k-mers in the call                                       */
    uint64_t n_tested;  /* passed the pre-filter: the .count value (src/kgwas.cpp:301) */
    uint64_t n_hits;    /* rows with p <= 10^-log10_thresh                          */
    const kg_hit* hits; /* sorted by k-mer index; owned by the context, valid until
                           the next kg_run_* / kg_fetch / kg_destroy on it           */
} kg_result;

/* Optional per-k-mer host outputs, each of length n_kmers (any may be NULL).
 * Untested k-mers get tested=0, chisq=0, pval=1, effect=0, mlog10p=0. */
typedef struct kg_stats {
    uint8_t* tested;
    double* chisq;
    double* pval;
    double* effect;
    double* mlog10p;    /* -log10 p from a log-domain tail (no underflow)   */
    double* xxM;
    double* xyM;
    double* cor;        /* Pearson correlation of the pre-filter             */
} kg_stats;

/* Fill `opts` with the reference's defaults (device 0, split precision). */
void kg_default_opts(kg_opts* opts);

/* Create a context on opts->device.  Replaces the process set-up of
 * src/kgwas.cpp:527-532 / parse_args :67-126 for the arithmetic part. */
int kg_create(kg_ctx** out, const kg_opts* opts);

/* Set the structure and phenotype of one test.  U is n x k column-major
 * FP64 (the U.bin body, src/kgwas_utils.hpp:135-157), y the phenotype of the
 * n overlap samples in samples-file order (src/kgwas_utils.hpp:291-314).
 * Computes yyM = ||y||^2 - ||U^T y||^2 (src/kgwas_utils.hpp:151-153); stores
 * it in *yyM_out when non-NULL. */
int kg_set_structure(kg_ctx* ctx, const double* U_colmajor, int n, int k,
                     const double* y, double* yyM_out);

/* As kg_set_structure, for packed rows that hold more samples than the
 * overlap (e.g. every sample of samples.txt, or one row layout shared by many
 * phenotypes with different missing samples): overlap sample i is bit
 * sample_pos[i] of each row, rows hold n_row_samples samples, and bits at
 * every other position are ignored.  Replaces the overlap gather of
 * load_matrix_rows (src/kgwas_utils.hpp:236-240). */
int kg_set_structure_ex(kg_ctx* ctx, const double* U_colmajor, int n, int k,
                        const double* y, const int32_t* sample_pos, int n_row_samples,
                        double* yyM_out);

/* Run the test on host-resident packed rows (pageable or pinned).  Host to
 * device copies are chunked and overlapped with the kernels.  Replaces the
 * pre-filter, compute_cols_stats, compute_hit and the emit selection
 * (src/kgwas.cpp:182-259) plus the .count value (:301). */
int kg_run_host(kg_ctx* ctx, const uint64_t* xbits, uint64_t n_kmers,
                uint32_t words_per_kmer, kg_result* res, kg_stats* stats);

/* Same on device-resident rows.  Enqueues the kernels on `stream`
 * (a cudaStream_t; NULL selects the context's own stream, not the legacy
 * default stream) and returns without synchronising; kg_fetch() waits and
 * returns the result. */
int kg_launch_device(kg_ctx* ctx, const uint64_t* d_xbits, uint64_t n_kmers,
                     uint32_t words_per_kmer, void* stream);
int kg_fetch(kg_ctx* ctx, kg_result* res, kg_stats* stats);

/* As kg_launch_device, and also computes the per-k-mer statistics that the
 * next kg_fetch copies into its kg_stats (the reference keeps them only in
 * memory, src/kgwas.cpp:156-158,248). */
int kg_launch_device_stats(kg_ctx* ctx, const uint64_t* d_xbits, uint64_t n_kmers,
                           uint32_t words_per_kmer, void* stream);

/* Allocates now the buffers that kg_run_host needs for a batch of n_kmers
 * pageable rows of words_per_kmer words (its device chunks and page-locked
 * staging buffers, 2 x min(512 MB, the batch) of each), so that a program
 * can pay for them while it still reads its inputs, e.g. on the thread that
 * created the context.  They are kept for later calls; kg_run_host grows
 * them when a batch needs more.  Replaces nothing in the reference (it has
 * no device buffers). */
int kg_reserve_host(kg_ctx* ctx, uint64_t n_kmers, uint32_t words_per_kmer);

/* Page-locked host memory for packed rows, so that kg_run_host copies at full
 * link speed without staging; NULL on failure.  Free with kg_host_free. */
void* kg_host_alloc(size_t bytes);
void kg_host_free(void* p);

/* ---------------------------------------------------------------------
 * Many phenotypes over one batch.  The reference runs one kgwas process per
 * (phenotype, batch) pair (HPC/kgwas/kgwas_cols.sh:22-65), each re-reading
 * the batch; here one launch tests every phenotype against each k-mer tile
 * while the tile's packed rows stay on chip.  Rows hold n_row_samples
 * samples (e.g. all of samples.txt); phenotype p has its own overlap
 * (sample_pos, n), U.bin (U, k) and y, as if its own kgwas process had run
 * build_overlap + load_Ubin on it (src/kgwas_utils.hpp:129-157, 285-314).
 * The batch may be the concatenation of several shards (batch_* of uneven
 * length): tested counts are kept per shard, as the reference's .count
 * files are (src/kgwas.cpp:291-304).
 * ------------------------------------------------------------------- */
typedef struct kg_pheno {
    const double* U_colmajor;  /* n x k, column-major                          */
    int n;                     /* overlap samples of this phenotype            */
    int k;                     /* U.bin columns                                */
    const double* y;           /* n phenotype values, in row-position order    */
    const int32_t* sample_pos; /* bit position of overlap sample i in each row */
} kg_pheno;

typedef struct kg_phit {
    uint64_t kmer;     /* index within the launch's rows                       */
    int32_t pheno;     /* phenotype index                                      */
    int32_t shard;     /* shard index                                          */
    double effect;
    double pval;
    double chisq;
} kg_phit;

typedef struct kg_multi_result {
    uint64_t n_kmers;
    int n_pheno;
    int n_shards;
    const uint64_t* n_tested;  /* [shard * n_pheno + pheno]: the .count values */
    uint64_t n_hits;
    const kg_phit* hits;       /* sorted by (pheno, kmer); owned by the context */
} kg_multi_result;

/* Set the phenotypes of a context (split precision only). */
int kg_set_phenotypes(kg_ctx* ctx, const kg_pheno* phenos, int n_pheno, int n_row_samples);

/* Test every phenotype on device rows.  shard_start (host, n_shards entries,
 * ascending, shard_start[0] = 0) splits the rows into shards; NULL = one
 * shard.  Asynchronous on `stream` until kg_fetch_multi. */
int kg_launch_multi_device(kg_ctx* ctx, const uint64_t* d_xbits, uint64_t n_kmers,
                           uint32_t words_per_kmer, const uint64_t* shard_start, int n_shards,
                           void* stream);
int kg_fetch_multi(kg_ctx* ctx, kg_multi_result* res);

/* Tile shape of the many-phenotype launches, as kg_set_phenotypes and the
 * autotuner chose it (this build's own batching; the reference runs one
 * process per phenotype and batch, HPC/kgwas/kgwas_cols.sh:22-65). */
typedef struct kg_tile_shape {
    int kernel;   /* 1: each group's limb image resident in shared memory;
                     2: images streamed from L2;
                     3: pairs of SMs (cta_group::2), two phenotypes per M = 256
                        MMA, one phenotype's image resident in each SM       */
    int np;       /* limb columns per phenotype slot                         */
    int ppg;      /* phenotypes per MMA group (MMA N = np * ppg)             */
    int groups;   /* MMA groups                                              */
    int kpad;     /* samples per image (padded)                              */
    int bt;       /* kernel 1: tile-iterations per L2 block of the last launch */
    int xs, nb;   /* kernel 2: resident row tiles, image ring stages         */
} kg_tile_shape;
int kg_multi_shape(const kg_ctx* ctx, kg_tile_shape* out);

/* Same from host rows (chunked host-to-device copies overlapped with the kernels). */
int kg_run_multi_host(kg_ctx* ctx, const uint64_t* xbits, uint64_t n_kmers, uint32_t words_per_kmer,
                      const uint64_t* shard_start, int n_shards, kg_multi_result* res);

/* ---------------------------------------------------------------------
 * 2-D pair test (the reference's kgwas_2d, src/kgwas_2d.cpp:210-392).
 *
 * For every pair i < j of the n_kmers packed rows with row_start <= i <
 * row_end (the reference's --task-id/--num-tasks row range, :245-250), the
 * column x_i * x_j (AND of the rows) is tested like one k-mer of the 1-D
 * test against the structure and phenotype of kg_set_structure, without the
 * Pearson pre-filter: pairs with popcount(x_i * x_j) = 0, xxM <= 1e-12 or
 * yyM <= 1e-12 are skipped (:292-304), and pairs with p <= 10^-log10_thresh
 * are returned (:306-318).  Split precision only; every returned pair is
 * recomputed in FP64.
 * ------------------------------------------------------------------- */
typedef struct kg_pair {
    uint64_t a, b;      /* k-mer indices, a < b                               */
    double effect;      /* xyM / (xxM * yyM)                                  */
    double pval;        /* erfc(sqrt(T/2))                                    */
    double chisq;       /* T = n ln(1/(1 - r^2))                              */
} kg_pair;

typedef struct kg_pair_result {
    uint64_t n_kmers;
    uint64_t n_evaluated; /* pairs that received a p-value                  */
    uint64_t n_pairs;     /* pairs with p <= 10^-log10_thresh               */
    const kg_pair* pairs; /* sorted by (a, b); owned by the context, valid until
                             the next call on it                              */
} kg_pair_result;

/* Replaces build_stats2d_self + emit_pairs_self (src/kgwas_2d.cpp:210-392).
 * xbits: host rows as for kg_run_host; n_kmers < 2^32. */
int kg_pairs_run_host(kg_ctx* ctx, const uint64_t* xbits, uint64_t n_kmers, uint32_t words_per_kmer,
                      uint64_t row_start, uint64_t row_end, kg_pair_result* res);

/* Number of kernel launches the last kg_run_host / kg_launch_device made. */
int kg_last_launch_count(const kg_ctx* ctx);

/* Which association kernel the last launch used: "ts" (tensor cores, x
 * unpacked into tensor memory), "ss" (tensor cores, x unpacked into shared
 * memory; shapes the first does not cover) or "fp64" (CUDA cores). */
const char* kg_last_kernel(const kg_ctx* ctx);

/* Rows the last kg_run_host tested on the device when it used runs of equal
 * adjacent rows (0 when it tested every row).  Batches sorted by bit pattern
 * (src/convert_matrix.cpp:366-368) hold such runs; one row per run is tested,
 * counts once per row of its run in n_tested, and its hit is repeated for
 * every row of the run, so the result is the same as without runs.  Used for
 * pageable host rows (which are staged through the host anyway) when at least
 * 10% of sampled adjacent rows are equal, never when kg_stats outputs are
 * requested.  KG_DEDUP=0 in the environment turns it off, KG_DEDUP=1 uses it
 * for pinned rows too. */
uint64_t kg_last_unique_rows(const kg_ctx* ctx);

/* Bounded device-side waits.  Every wait between the roles of the
 * tensor-memory kernels' pipelines (row loads, tensor-memory slots,
 * accumulators, limb images; the single-phenotype, many-phenotype and pair
 * kernels) gives up after wait_ns nanoseconds: the kernel then stops,
 * waits for its own copies and MMAs in flight, frees its tensor memory and
 * returns, and the call reports KG_ERR_TIMEOUT while the context stays
 * usable.  0 restores the default of 2 s.  The reference has no device waits;
 * its failures end the process (die(), src/kgwas_utils.hpp:34-37). */
int kg_set_wait_limit(kg_ctx* ctx, uint64_t wait_ns);

/* Failure test hook of the bounded waits, off by default: for the next
 * launch of the single-phenotype tensor-memory kernel only, the row producer
 * of every CTA issues its first stop_after_loads row loads and then no more,
 * so that the waits of the roles it feeds run out (KG_ERR_TIMEOUT) instead of
 * completing.  No counterpart in the reference. */
int kg_inject_stall(kg_ctx* ctx, uint64_t stop_after_loads);

const char* kg_last_error(const kg_ctx* ctx);
void kg_destroy(kg_ctx* ctx);

/* Library version string. */
const char* kg_version(void);

/* Measured peaks that throughput figures are reported against; no
 * counterpart in the reference.  kg_probe_fp64_tflops: FP64 FMA rate of the
 * CUDA cores (independent FMA chains on every SM), in TFLOP/s -- the bound of
 * the KG_PREC_FP64 form.  kg_probe_h2d_gbs: pinned host-to-device copy rate,
 * `reps` copies of `bytes` with one cudaMemcpyAsync each, in GB/s -- the
 * bound of kg_run_host / kg_run_multi_host on rows from host memory.  Both
 * allocate their own buffers and synchronise. */
int kg_probe_fp64_tflops(int device, double* tflops);
int kg_probe_h2d_gbs(int device, uint64_t bytes, int reps, double* gbs);

/* Allocation-free run, for callers that may not allocate device memory (a
 * host framework that owns every device byte through its own pool, a plugin
 * inside such a process, a job with a fixed memory budget).  No counterpart
 * in the reference.
 *
 * Runs the split-precision test of kg_set_structure + kg_launch_device in one
 * call, without a context, with the same accuracy: k-mers whose split-form
 * chi-square reaches 12 are recomputed in FP64 before their rows are
 * emitted.  d_xbits (device, packed rows as above), U/y (host, as in
 * kg_set_structure), and d_hits (device, hit_capacity records, filled in
 * arbitrary order).  counts_out (host) receives {n_tested, n_hits}.  The call
 * blocks: it synchronises `stream` (a cudaStream_t, NULL = default stream)
 * before it returns.
 *
 * It calls no device allocator.  Its device scratch (the counters, the int8
 * limb image of the structure, the FP64 columns of the refinement and the
 * list of k-mers to refine) is one static array of KG_NOALLOC_SCRATCH_BYTES
 * that every GPU loading this library holds until the process exits.
 * Structures whose limb image exceeds KG_NOALLOC_MAX_B_BYTES (overlap samples
 * rounded up to 256, times the limb columns rounded up to 16) or whose FP64
 * columns exceed KG_NOALLOC_MAX_V_BYTES (overlap samples rounded up to 128,
 * times k + 2 columns rounded up to 8..68, times 8 bytes) are rejected with
 * KG_ERR_UNSUPPORTED.  At most KG_NOALLOC_MAX_REFINE k-mers are refined per
 * pass; a batch with more is run again in smaller pieces.  The first call on
 * a device (and the first after that device's context was destroyed and
 * created anew) looks up the array's device address with
 * cudaGetSymbolAddress; make it before any stream capture on that device.
 * Calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  More hits than hit_capacity return
 * KG_ERR_INVALID with counts_out still filled.  err (optional, err_len bytes)
 * receives a message on failure. */
#define KG_NOALLOC_MAX_B_BYTES (256u * 1024u)
#define KG_NOALLOC_MAX_V_BYTES (1024u * 1024u)
#define KG_NOALLOC_MAX_REFINE 32768u
#define KG_NOALLOC_SCRATCH_BYTES \
    (256u + KG_NOALLOC_MAX_B_BYTES + KG_NOALLOC_MAX_V_BYTES + 8u * KG_NOALLOC_MAX_REFINE)
int kg_run_device_noalloc(const uint64_t* d_xbits, uint64_t n_kmers, uint32_t words_per_kmer,
                          const double* U_colmajor, int n, int k, const double* y,
                          double corr_threshold, double log10_thresh,
                          kg_hit* d_hits, uint64_t hit_capacity, uint64_t* counts_out,
                          void* stream, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* KGWAS_CUDA_H */

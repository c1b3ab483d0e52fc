/*
 * dada2_b200.h -- C ABI of the B200 (sm_100a) implementation of the compare step
 * inside dada2-rs `dada` divisive clustering.
 *
 * Everything here is plain C: pointers, sizes and POD structs. Host buffers are
 * owned by the caller; device memory is owned by a context or by the call that
 * allocated it. Every function returns 0 on success or a negative DGPU_E_* code;
 * dgpu_last_error() then describes the failure (per calling thread). No call
 * traps or aborts on bad input; a device-side failure (for example an invalid
 * traceback pointer, where the reference panics) is reported as DGPU_E_DEVICE.
 *
 * Reference interfaces replaced (paths are within HPCBio/dada2-rs 0.2.0):
 *   dgpu_ctx_create      AlignParams + error matrix setup   src/nwalign.rs:63-90, src/dada.rs:54-101
 *   dgpu_upload_raws     Raw::from_qual_sums + raw_assign_kmers
 *                                                           src/containers.rs:128-137, src/kmers.rs:213-221
 *   dgpu_compare         the per-raw map of b_compare_parallel
 *                                                           src/cluster.rs:279-330
 *   dgpu_compare_store   map + serial store of b_compare_parallel
 *                                                           src/cluster.rs:239-423
 *   dgpu_dada            dada_uniques (plain: one sample)   src/dada.rs:225-592
 *   dgpu_dada_batch      many independent samples at once (the per-sample fan-out of
 *                        for_each_sample_concurrent)        src/main.rs:4648-4697
 *   dgpu_dada_sharded    dada_uniques with each compare call split over ranks
 *                        (the per-raw map of b_compare_parallel, src/cluster.rs:279-330)
 *   dgpu_align_debug     the aligners alone (test entry)    src/nwalign.rs:336-1140
 *
 * Threading: a context is used by one host thread at a time. Calls that take no
 * context are reentrant.
 */
#ifndef DADA2_B200_H
#define DADA2_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DGPU_OK 0
#define DGPU_E_INVALID (-1)     /* rejected input (same checks as dada_uniques_cached) */
#define DGPU_E_CUDA (-2)        /* a CUDA runtime call failed */
#define DGPU_E_DEVICE (-3)      /* a kernel reported an error flag */
#define DGPU_E_UNSUPPORTED (-4) /* a parameter combination this build does not cover */
#define DGPU_E_NOMEM (-5)

/* AlignParams (src/nwalign.rs:63-90); booleans are 0/1. */
typedef struct {
  int32_t match_score, mismatch, gap_p, homo_gap_p;
  int32_t use_kmers;
  double kdist_cutoff;
  int32_t kmer_size, band, vectorized, gapless;
} dgpu_align_params;

/* The DadaParams fields the clustering loop reads (src/dada.rs:54-101). */
typedef struct {
  dgpu_align_params align;
  double omega_a, omega_p, omega_c;
  int32_t detect_singletons, max_clust;
  double min_fold;
  uint32_t min_hamming, min_abund;
  int32_t use_quals, greedy;
  int32_t host_threads; /* threads for the host phases of dgpu_dada_batch; 0 = half the cores */
  int32_t transitions;  /* 1: also count transitions by quality after the final-subs pass
                           (DadaAux.transitions, src/dada.rs:609-673, src/error.rs:194-249) */
  int32_t lambda_fp32;  /* 1: decisions take lambda from its compensated FP32 log-sum,
                           except that any p-value within 1e3x of omega_a (times the
                           raws, as the bud tests it), omega_p (prior raws) or omega_c
                           (the final map) is repriced from the FP64 product; the
                           store's e_minmax bound stays FP64. Not in the reference:
                           a precision variant, compared against the FP64 default. */
} dgpu_dada_params;

/* Counters of one compare call (CompareTiming's denominators, src/cluster.rs:190-231). */
typedef struct {
  uint64_t screened, aligned, shrouded, stored;
  uint64_t gapless, vectorized, homo, endsfree;
} dgpu_counters;

/* Output layout of dgpu_dada / dgpu_dada_batch results (all caller-allocated;
 * sizes from dgpu_result_sizes). Cluster c's center sequence is
 * cl_seq[cl_seq_off[c] .. cl_seq_off[c+1]) (codes 1..4); its members are
 * mem_*[cl_mem_off[c] .. cl_mem_off[c+1]). map[r] = -1 when raw r was not
 * corrected to any cluster (src/dada.rs:525-533). counters (16 slots):
 * nalign, compare_calls, cmp_scanned (sum of nraw over compare calls),
 * screened, aligned, stored, gapless, vectorized, homo, endsfree,
 * shuffle_calls, shuffle_moves, nshroud, then the nanoseconds this sample's
 * host spent in shuffle, p-update and bud. times (6 slots, seconds): this
 * sample's compare calls (launch to results), the time from the start of the
 * clustering loop until this sample finished, this sample's host phases
 * (shuffle, p-update, bud), time the host waited on the device for this
 * sample's compare calls (a batched call counts for every sample it carries), time this
 * sample waited for a launch slot (ready to launched) and for a host thread
 * (results absorbed to host phase started). */
typedef struct {
  uint32_t* cl_reads;
  int32_t* cl_birth_type;
  uint32_t* cl_birth_from;
  double* cl_birth_pval;
  double* cl_birth_fold;
  double* cl_birth_e;
  uint32_t* cl_birth_hamming;
  uint32_t* cl_seq_off;
  uint8_t* cl_seq;
  uint32_t* cl_mem_off;
  uint32_t* mem_raw;
  uint32_t* mem_hamming;
  double* mem_lambda;
  double* mem_pval;
  int32_t* map;
  double* pvals;
  uint64_t* counters;
  double* times;
} dgpu_dada_out;

typedef struct dgpu_ctx dgpu_ctx;
typedef struct dgpu_result dgpu_result;
typedef struct dgpu_batch dgpu_batch;

/* Process-wide kernel accounting (for benchmarks). Index k: 0 profiles,
 * 1 screen, 2 align (ordered-k-mer distance, gapless or NW alignment and
 * lambda for the pairs that passed the screen), 3 store. screen_bytes =
 * algorithmic bytes of the screen: 4^k profile bytes per non-skipped compare
 * plus 16 bytes of per-raw metadata per compare. ms[] sums the device time
 * (CUDA events around each kernel on its stream) of the timed compare calls
 * only -- every N-th call while dgpu_stats_timing(N) is in force -- and the
 * timed_* fields count those calls, their screen bytes and compares. */
typedef struct {
  uint64_t launches[4];
  double ms[4];
  uint64_t rounds, compares, screened, screen_bytes;
  uint64_t timed_rounds, timed_screen_bytes, timed_compares;
  uint64_t h2d_bytes;  /* host-to-device bytes copied: uploads, lock flags, per-call task tables */
  double batch_ms[3];  /* wall time of dgpu_batch_run / dgpu_dada_batch runs: before the loop
                          (resets, sample state), the loop, after it (results, final-subs) */
  double prepare_ms[4]; /* wall time of dgpu_batch_prepare / dgpu_dada_batch preparation:
                           validation, encoding and pool set-up; upload and k-mer profiles;
                           of the latter, the launch slots' set-up and the wait for the copies
                           and the profile kernel */
} dgpu_kernel_stats;

const char* dgpu_last_error(void);
int dgpu_device_count(int* count);

/* ---- compare-level drop-in (one pool of uniques resident on one device) ---- */
int dgpu_ctx_create(int device, const dgpu_align_params* params, const double* err_mat, int ncol,
                    int use_quals, dgpu_ctx** out);
void dgpu_ctx_destroy(dgpu_ctx* ctx);
/* seqs: concatenated codes 1..4 (A,C,G,T); quals: rounded mean Phred per
 * position, same offsets, or NULL. Builds the k-mer profiles on the device. */
int dgpu_upload_raws(dgpu_ctx* ctx, int nraw, const uint8_t* seqs, const uint32_t* offs,
                     const uint32_t* lens, const uint8_t* quals, const uint32_t* reads);
int dgpu_set_locks(dgpu_ctx* ctx, const uint8_t* lock);
/* Reset every raw's running max expected abundance to -999 (B::new). */
int dgpu_reset_e_minmax(dgpu_ctx* ctx);
int dgpu_get_e_minmax(dgpu_ctx* ctx, double* out);
/* The map: per raw lambda, hamming (UINT32_MAX = shrouded or skipped), skipped flag. */
int dgpu_compare(dgpu_ctx* ctx, int center, double kdist_cutoff, int greedy, double* lambda_out,
                 uint32_t* hamming_out, uint8_t* skipped_out, dgpu_counters* cnt);
/* The aligner each raw took in the context's latest compare (raw_align_dp's
 * method choice, src/nwalign.rs:1315-1414): 0 none (skipped or shrouded),
 * 1 gapless, 2 vectorized, 3 homopolymer, 4 ends-free; nraw bytes. */
int dgpu_get_methods(dgpu_ctx* ctx, uint8_t* out);
/* Map + store: comps with lambda*total_reads > e_minmax, ascending raw index,
 * e_minmax updated on the device; self_out = the center's own lambda. */
int dgpu_compare_store(dgpu_ctx* ctx, int center, int cluster_i, double kdist_cutoff, int greedy,
                       uint32_t* comp_index, double* comp_lambda, uint32_t* comp_hamming,
                       int* nstored, double* self_out, dgpu_counters* cnt);

/* ---- full denoising ---- */
/* One sample (ASCII uniques, per-position Phred SUMS or NULL). */
int dgpu_dada(int device, const dgpu_dada_params* params, int nraw, const char* seqs,
              const uint32_t* offs, const uint32_t* lens, const uint32_t* abund, const uint8_t* prior,
              const uint32_t* qual_sums, const double* err_mat, int ncol, dgpu_result** out);
/* Many independent samples in one pass: sample s owns uniques
 * [sample_start[s], sample_start[s+1]) of the concatenated inputs. out[s]
 * receives one result per sample. */
int dgpu_dada_batch(int device, const dgpu_dada_params* params, int nsamples,
                    const uint32_t* sample_start, const char* seqs, const uint32_t* offs,
                    const uint32_t* lens, const uint32_t* abund, const uint8_t* prior,
                    const uint32_t* qual_sums, const double* err_mat, int ncol, dgpu_result** out);
/* The same work split in two: prepare validates, encodes and uploads the
 * samples and builds their k-mer profiles (the inputs become resident in HBM);
 * run executes the whole clustering loop on the resident inputs and may be
 * called repeatedly (each run starts from a fresh partition). out needs
 * nsamples slots. */
int dgpu_batch_prepare(int device, const dgpu_dada_params* params, int nsamples,
                       const uint32_t* sample_start, const char* seqs, const uint32_t* offs,
                       const uint32_t* lens, const uint32_t* abund, const uint8_t* prior,
                       const uint32_t* qual_sums, const double* err_mat, int ncol, dgpu_batch** out);
int dgpu_batch_run(dgpu_batch* batch, dgpu_result** out);
void dgpu_batch_free(dgpu_batch* batch);

/* ---- one sample over several GPUs ---- */
/* All-gather of fixed-size blocks among the ranks of a sharded run: every
 * rank passes `bytes` bytes in send; recv (world * bytes) receives rank r's
 * block at offset r * bytes. Returns 0, or nonzero when the exchange failed.
 * The callback must end with an error, not block, when a peer has gone (for
 * example through a process-group timeout). */
typedef int (*dgpu_allgather_fn)(void* user, const void* send, uint64_t bytes, void* recv);
/* dgpu_dada with the compare calls split over `world` ranks (one process or
 * thread per GPU, `device` being the rank's own). Every rank passes the same
 * inputs and parameters and runs the same clustering loop; a compare call
 * screens and aligns only the rank's contiguous share of the uniques
 * (balanced by bases) and the stored comps of all shares are all-gathered in
 * rank order, the ascending raw order of the one-device store
 * (src/cluster.rs:351-397). Two exchanges per compare call: a 56-byte head
 * (status, counters, the center's own lambda) and, when any share stored
 * comps, 24 bytes per comp of the largest share. Every rank's result equals
 * dgpu_dada's on the same inputs. A failure on any rank after the argument
 * checks fails every rank at the same exchange. Replaces, for one pooled
 * sample spanning GPUs, the per-raw map of b_compare_parallel
 * (src/cluster.rs:279-330), which the reference runs on one host's threads. */
int dgpu_dada_sharded(int device, const dgpu_dada_params* params, int nraw, const char* seqs,
                      const uint32_t* offs, const uint32_t* lens, const uint32_t* abund,
                      const uint8_t* prior, const uint32_t* qual_sums, const double* err_mat,
                      int ncol, int rank, int world, dgpu_allgather_fn gather, void* user,
                      dgpu_result** out);

/* Device memory reuse. No counterpart in the reference (its compare step holds
 * no device memory). A finished pool (dgpu_dada, dgpu_dada_batch,
 * dgpu_batch_free) keeps its device and pinned host blocks in a per-device
 * cache, at most 32 GiB of each kind per device, that the next call reuses.
 * This frees every cached block of `device` (all devices when device < 0) and
 * writes the bytes given back to *freed (may be NULL). */
int dgpu_cache_release(int device, uint64_t* freed);

/* ---- tuning table ----
 * The launch shape of the compare step per read-length class of a pool
 * (class 0: longest unique <= 200 nt, 1: <= 600 nt, 2: longer):
 * launch_slots         concurrent compare launches (streams) of a batch, 1..8
 * samples_per_launch   most samples one compare launch serves, 1..4096
 * dedicated_slots      slots reserved for the samples with the longest chains, 0..7
 * align_ctas_per_sm    resident CTAs of the alignment kernel per SM (4 pairs each), 1..4
 * screen_chunk_max     largest run of (center, unique) items one screen warp takes, 16 or 32
 * screen_blocks_per_sm screen blocks per SM in its single wave, 1..4
 * pivot_min_items      compare launches of at least this many (center, unique) items
 *                      exclude far uniques by the exact pivot bound without reading
 *                      their k-mer profiles (one extra small kernel); 0 = never
 * programmatic_launch  1: the alignment and store kernels are launched as programmatic
 *                      dependents of the kernel before them (scheduled while it drains);
 *                      0: ordinary stream order
 * The library loads DGPU_TUNING_FILE, else tuning.txt beside itself, at first
 * use (the autotuner, dada2_b200/autotune.py, writes that file); the
 * DGPU_LAUNCH_SLOTS, DGPU_BATCH_MAX and DGPU_DEDICATED_SLOTS environment
 * variables override it. A setting applies to pools created after it.
 * Results never depend on it. Replaces the reference's only scheduling knob,
 * the rayon grain DADA2_RS_PAR_GRAIN (src/cluster.rs:19-28). */
typedef struct {
  int32_t launch_slots, samples_per_launch, dedicated_slots, align_ctas_per_sm, screen_chunk_max,
      screen_blocks_per_sm, pivot_min_items, programmatic_launch;
} dgpu_tuning;
/* the setting a pool whose longest unique has max_len bases would use */
int dgpu_tuning_get(int max_len, dgpu_tuning* out);
int dgpu_tuning_set(int length_class, const dgpu_tuning* t);
int dgpu_tuning_load(const char* path);
int dgpu_tuning_save(const char* path);
/* back to the built-in table; no file is loaded afterwards */
int dgpu_tuning_reset(void);

int dgpu_stats_reset(void);
/* every = 0 stops the per-kernel timing; every = N >= 1 times every N-th
 * compare call (events cost a few microseconds per call). */
int dgpu_stats_timing(int every);
int dgpu_stats_read(dgpu_kernel_stats* out);
/* Latency (ms) of each compare call since the last reset, from launch to the
 * results being on the host; copies up to cap values, returns how many exist. */
int dgpu_stats_latencies(double* out, int cap);

/* sizes: [nclust, nraw, total members, total center-sequence bytes] */
int dgpu_result_sizes(const dgpu_result* res, int64_t* sizes);
int dgpu_result_fill(const dgpu_result* res, const dgpu_dada_out* out);
/* Transition counts of a run made with dgpu_dada_params.transitions = 1: the
 * 16 x ncol matrix (row 4 * center nt + raw nt, column = quality; ncol is the
 * sample's error-matrix width after extension, or 1 without qualities) is
 * copied to out (when non-null) and ncol returned; 0 when not computed.
 * Replaces transition_counts (src/error.rs:194-249). */
int dgpu_result_transitions(const dgpu_result* res, uint32_t* out);
void dgpu_result_free(dgpu_result* res);

/* Precision variant of compute_lambda (src/pval.rs:253-320): with enable = 1
 * every later compare of the context also forms ln(lambda) of each aligned
 * pair as a compensated FP32 sum of logf(err) beside the FP64 product (which
 * stays the one every decision uses). dgpu_get_loglambda32 copies the latest
 * compare's values (nraw floats; -inf for pairs not aligned). No counterpart
 * in the reference, which computes FP64 only. */
int dgpu_ctx_set_lambda32(dgpu_ctx* ctx, int enable);
int dgpu_get_loglambda32(dgpu_ctx* ctx, float* out);
/* calc_pA (src/pval.rs:208-241): the Poisson abundance p-value of a unique
 * with `reads` reads against an expected e_reads, conditioned on being seen
 * unless `prior`. */
double dgpu_calc_pA(uint32_t reads, double e_reads, int prior);

/* ---- denoising service ----
 * Requests (one sample each, the inputs of dgpu_dada) are submitted at any
 * time and served on `device` by a worker thread: pending requests of the
 * oldest request's length class (longest unique <= 200, <= 600 or longer nt)
 * are batched in arrival order while the estimated device-memory footprint of
 * every batch in flight fits `hbm_budget` bytes (0: half the device's free
 * memory) and denoised together like dgpu_dada_batch, so each result is
 * dgpu_dada's on that sample; a request completes as soon as its own sample
 * does. DGPU_SERVICE_WORKERS (default 3) batches run at once. The
 * input buffers stay the caller's and must remain valid until the ticket's
 * wait returns (they are read when the request is served; a batch packs
 * copies of its requests' uniques). dgpu_service_wait blocks until the ticket is
 * served and returns its result (free with dgpu_result_free) and its latency
 * from submit to completion. Destroying the service serves what is pending.
 * No counterpart in the reference, whose per-sample fan-out is
 * for_each_sample_concurrent (src/main.rs:4648-4697). */
/* With lambda_fp32: [0] p-values priced from the FP32 lambda, [1] of those
 * repriced from the FP64 product (the fallback). Zero otherwise. */
int dgpu_result_fp32_stats(const dgpu_result* res, uint64_t* out2);
/* Decision margins of the run: out3[0] the smallest |p - omega_a| /
 * min(p, omega_a) over the bud's tests of p * nraw against omega_a (+inf for
 * p = 0), out3[1] the same for the
 * prior raw's p against omega_p (both src/cluster.rs:1501-1640), out3[2] for
 * the final map's p against omega_c (src/dada.rs:525-533); +inf where no
 * such test ran. A margin far above 1e-12 shows that p-values differing by a
 * few ulps could not have changed any decision. No counterpart in the
 * reference (a diagnostic of this implementation). */
int dgpu_result_margins(const dgpu_result* res, double* out3);

/* ---- learn-errors ----
 * The error-model fit applied to an accumulated 16 x nq transition matrix
 * (row 4 * ref nt + query nt, column = quality score):
 *   DGPU_ERRFUN_LOESS   loess_errfun (src/error_models.rs:119-210): per
 *                       off-diagonal transition, LOESS (span 0.75, degree 2)
 *                       of log10((count + 1) / total of the source nucleotide)
 *                       on the quality score weighted by that total, surface
 *                       0 direct (the dada2-rs default) or 1 kd-tree
 *                       interpolation with `cell` (R's default, 0.2), flat
 *                       extrapolation, rates clamped to [min, max]
 *   DGPU_ERRFUN_NOQUAL  noqual_errfun (src/error_models.rs:212-261): one
 *                       rate per transition from counts summed over
 *                       qualities plus `pseudocount`
 *   DGPU_ERRFUN_BINNED  binned_qual_errfun (src/error_models.rs:263-396):
 *                       the observed rate at each of the `nbins` anchor
 *                       qualities `bins` (ascending), linear between
 *                       adjacent anchors, flat beyond the outer ones;
 *                       DGPU_E_INVALID when no column has an observation or
 *                       an observed quality lies outside the anchors
 *   DGPU_ERRFUN_PACBIO  pacbio_errfun (src/error_models.rs:408-462): with
 *                       nq = 94 (a Q93 column), LOESS over columns 0..92 and
 *                       (count + 1) / (source total + 4) for column 93;
 *                       otherwise LOESS
 *   DGPU_ERRFUN_EXTERNAL external_errfun (src/error_models.rs:650-780): the
 *                       command `cmd` (split on whitespace, no shell) runs
 *                       with two paths appended, a TSV of the transitions
 *                       to read and a TSV of the error matrix to write (R's
 *                       read.table layout: a header of a tab and 0..nq-1,
 *                       then rows A2A .. T2T); every value must be finite
 *                       and in [0, 1]; a failed command's standard error
 *                       is in the message
 * The diagonal of each nucleotide is 1 minus its three off-diagonals
 * (PacBio's column 93 and the external fit excepted). */
#define DGPU_ERRFUN_LOESS 0
#define DGPU_ERRFUN_NOQUAL 1
#define DGPU_ERRFUN_BINNED 2
#define DGPU_ERRFUN_PACBIO 3
#define DGPU_ERRFUN_EXTERNAL 4
typedef struct {
  int32_t kind;
  int32_t surface;  /* LOESS: 0 direct, 1 interpolate */
  double cell;      /* LOESS interpolate: kd-tree cell fraction (0.2) */
  double max_error_rate, min_error_rate;  /* clamp of the off-diagonal rates (0.25, 1e-7) */
  double pseudocount;                     /* NOQUAL (1.0) */
  const double* bins;                     /* BINNED: anchor qualities (NULL otherwise) */
  int32_t nbins;
  const char* cmd;                        /* EXTERNAL: the command line */
} dgpu_errfun;
/* err_out (16 x nq) = the fit of trans (16 x nq). Host only. */
int dgpu_errfun_apply(const dgpu_errfun* ef, const uint32_t* trans, int nq, double* err_out);

/* learn_errors (src/learn_errors.rs:739-1010): the self-consistent loop that
 * estimates the error model from samples. nq = the largest rounded mean
 * quality + 1 (src/learn_errors.rs:494-506). An init pass denoises every
 * sample with an all-ones error matrix and at most one cluster, counts
 * transitions, fits and forces the diagonal to 1 (src/learn_errors.rs:525-616);
 * then up to max_consist passes denoise all samples with the current matrix
 * (the batched GPU path), count each sample's transitions by realigning every
 * corrected unique to its center (build_trans_mat, src/learn_errors.rs:618-738;
 * counted on the device), sum them, fit, and stop once the fit equals bit for
 * bit any matrix used as input so far. Samples as in dgpu_dada_batch;
 * qual_sums are required (without qualities no transition is counted). The
 * dada parameters' error matrix is the loop's own. */
typedef struct dgpu_learn dgpu_learn;
int dgpu_learn_errors(int device, const dgpu_dada_params* params, const dgpu_errfun* errfun, int max_consist,
                      int nsamples, const uint32_t* sample_start, const char* seqs, const uint32_t* offs,
                      const uint32_t* lens, const uint32_t* abund, const uint32_t* qual_sums, dgpu_learn** out);
/* info[0] nq, [1] passes run (init pass excluded), [2] converged (0/1);
 * trans (16 x nq, may be NULL): the last pass's summed transitions; err_in /
 * err_out (16 x nq doubles, may be NULL): the matrix that pass used and the
 * fit of its transitions. */
int dgpu_learn_read(const dgpu_learn* l, int32_t* info, uint32_t* trans, double* err_in, double* err_out);
void dgpu_learn_free(dgpu_learn* l);

/* ---- ingest: FASTQ -> uniques ----
 * Dereplicates a FASTQ file (plain or gzip, four-line records) as
 * dereplicate does (src/derep.rs:43-240, ordering src/derep.rs:179-185):
 * uniques by read count descending, ties by sequence bytes ascending; per
 * unique the per-position SUM of (quality byte - phred_offset), stored as u32
 * (a negative sum becomes 0, one beyond u32 is DGPU_E_UNSUPPORTED); map[r] is
 * read r's unique. nthreads 0 = one per core. Host only: no device is used.
 * The outputs feed dgpu_dada / dgpu_dada_batch directly (counts as abund). */
typedef struct dgpu_derep dgpu_derep;
int dgpu_derep_fastq(const char* path, int phred_offset, int nthreads, dgpu_derep** out);
/* sizes[0] uniques, [1] reads, [2] total bytes of unique sequence */
int dgpu_derep_sizes(const dgpu_derep* d, int64_t* sizes);
/* Any output may be null. seqs: sizes[2] bytes; offs, lens, counts:
 * sizes[0] entries; qual_sums: sizes[2] entries (same offsets as seqs); map:
 * sizes[1] entries. */
int dgpu_derep_fill(const dgpu_derep* d, char* seqs, uint32_t* offs, uint32_t* lens, uint64_t* counts,
                    uint32_t* qual_sums, uint32_t* map);
void dgpu_derep_free(dgpu_derep* d);

typedef struct dgpu_service dgpu_service;
int dgpu_service_create(int device, const dgpu_dada_params* params, const double* err_mat, int ncol,
                        uint64_t hbm_budget, dgpu_service** out);
int dgpu_service_submit(dgpu_service* svc, int nraw, const char* seqs, const uint32_t* offs, const uint32_t* lens,
                        const uint32_t* abund, const uint8_t* prior, const uint32_t* qual_sums, uint64_t* ticket);
int dgpu_service_wait(dgpu_service* svc, uint64_t ticket, dgpu_result** out, double* latency_s);
/* While held (hold != 0) the service starts no new batch; requests submitted
 * meanwhile are batched together when it is released. */
int dgpu_service_hold(dgpu_service* svc, int hold);
int dgpu_service_stats(dgpu_service* svc, uint64_t* batches, uint64_t* served);
void dgpu_service_destroy(dgpu_service* svc);

/* ---- aligners alone (test entry) ----
 * which: 0 vectorized (compressed anti-diagonal i16, end_gap as given),
 *        1 ends-free with homopolymer gaps, 2 ends-free i32.
 * al0/al1 receive each pair's rows at al_off[p] (capacity len1+len2) in
 * left-to-right order; al_len[p] their length. */
int dgpu_align_debug(int device, int which, int npairs, const uint8_t* s1cat, const uint32_t* off1,
                     const uint32_t* len1, const uint8_t* s2cat, const uint32_t* off2,
                     const uint32_t* len2, const dgpu_align_params* params, int end_gap,
                     uint8_t* al0, uint8_t* al1, const uint32_t* al_off, uint32_t* al_len);

/* ---- aligners without device allocation ----
 * No counterpart in the reference. Same alignments as dgpu_align_debug, for
 * callers that cannot allocate device memory: a host whose device memory is
 * already reserved by its own pool allocator (cudaMalloc would fail or
 * fragment that pool), or a latency-bound pipeline that cannot afford the
 * device-wide synchronisation cudaFree implies. All pointers are
 * caller-owned and must be readable/writable by the current device (device
 * or managed memory); nothing is allocated. The aligners' scratch is a
 * 16 MiB static device array that every GPU loading this library holds until
 * exit. max_len bounds every sequence length (at most 3500 for which = 0);
 * lengths whose scratch for four concurrent alignments exceeds the array, or
 * whose shared-memory staging exceeds the device's per-block limit, are
 * rejected with DGPU_E_INVALID. A pair longer than max_len is refused on the
 * device: its outputs stay unwritten and the call returns DGPU_E_DEVICE (the
 * other pairs are aligned). The first call on a device looks up the array's
 * address (cudaGetSymbolAddress) and keeps it, so make that first call before
 * any stream capture, and do not use this entry point after cudaDeviceReset.
 * Every call shares the array: calls whose kernels overlap on one device race.
 * Runs on `stream` (a cudaStream_t; NULL = legacy default stream) and returns
 * after it finishes. */
int dgpu_align_pairs_noalloc(int which, int npairs, int max_len, const uint8_t* s1cat,
                             const uint32_t* off1, const uint32_t* len1, const uint8_t* s2cat,
                             const uint32_t* off2, const uint32_t* len2,
                             const dgpu_align_params* params, int end_gap, uint8_t* al0,
                             uint8_t* al1, const uint32_t* al_off, uint32_t* al_len,
                             void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DADA2_B200_H */

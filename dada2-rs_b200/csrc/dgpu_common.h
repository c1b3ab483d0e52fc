// Plain-data structures shared by the CUDA kernels and the C++ host driver.
#pragma once

#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <thread>

#include <cuda_runtime.h>

namespace dgpu {

// Alignment / screen parameters (AlignParams, src/nwalign.rs:63-90) plus the
// compare-loop switches the kernels read.
struct KParams {
  int32_t match, mismatch, gap, homo_gap;
  int32_t use_kmers, kmer_size, band, vectorized, gapless;
  int32_t use_quals, greedy;
  int32_t ncol;  // error-matrix columns
  int32_t lambda32;  // also form ln(lambda) as a compensated FP32 sum (precision report)
};

// Device view of a pool of uniques (one or more samples, concatenated).
struct PoolDev {
  const uint8_t* seq;     // 1..4 codes; raw g starts at off[g]
  const uint8_t* qual;    // rounded mean Phred, same offsets (nullptr: none)
  const uint32_t* off;
  const uint32_t* len;
  const uint8_t* kmer8;   // nraw x 4^k saturating u8 counts (k <= 7)
  const uint8_t* sat;     // per raw: some k-mer count reached 255
  // k = 8: each raw's present k-mers as ascending (index, saturating count)
  // pairs, kidx/kcnt[off[g] .. off[g] + knum[g])
  const uint16_t* kidx;
  const uint8_t* kcnt;
  const uint32_t* knum;
  const uint32_t* reads;
  const uint8_t* lock;
  double* e_minmax;
  const double* err;      // 16 x ncol
  // per-raw results of the latest compare launch
  double* res_lambda;
  uint32_t* res_ham;
  uint8_t* res_status;
  float* res_loglam32;  // with KParams::lambda32: FP32 ln(lambda) of aligned pairs, -inf otherwise
  // Pivot bound of the screen (k <= 7, the clustering loop only): per raw the
  // largest u8 k-mer dot with any center so far (piv_dot) and that center's
  // cluster (piv_cl, kNoPivot when none); per sample, cl_center[base + i] =
  // cluster i's center and cdot[base + i] = the current center's dot with it.
  uint32_t* piv_dot;
  uint32_t* piv_cl;
  uint32_t* cl_center;
  uint32_t* cdot;
  uint32_t nraw;
  uint32_t maxlen;
};

// One compare task: a new center against every raw of one sample.
struct TaskDev {
  uint32_t base;          // first global raw of the sample
  uint32_t n;             // raws in the sample
  uint32_t center;        // global raw index of the center
  uint32_t center_reads;
  double total_reads;     // B.reads of the sample
  double cutoff;          // kdist_cutoff for this call
  uint32_t out_off;       // first slot of this task's comp output
  uint32_t cluster;       // cluster index i (for the store's update_raw rule)
};

// The per-call values of a compare launch, at the head of the launch's table
// upload. A launch replayed from a captured CUDA graph keeps its kernel
// parameters fixed and takes these from device memory instead (CompareLaunch::
// hdr); the offsets are from the header's own address.
struct CallHeader {
  uint32_t ntask, total_items, screen_chunk, nstore_blocks;
  uint32_t pivot, cdot_ready, total_cl, pad;
  uint32_t o_tasks, o_pref, o_clp, o_map;
};
static_assert(sizeof(CallHeader) == 48, "the call header has a fixed layout");

// res_status layout: low 2 bits = outcome, next 3 bits = aligner.
enum : uint8_t { ST_ALIGNED = 0, ST_SKIPPED = 1, ST_SHROUDED = 2 };
enum : uint8_t { AM_NONE = 0, AM_GAPLESS = 1, AM_VECTORIZED = 2, AM_HOMO = 3, AM_ENDSFREE = 4 };

// Per-task counters written by the store kernel.
enum { TC_SCREENED = 0, TC_ALIGNED, TC_SHROUD, TC_STORED, TC_GAPLESS, TC_VECTORIZED, TC_HOMO,
       TC_ENDSFREE, TC_NCOUNTERS };

// Device error bits (OR-ed into the status word; the host turns them into codes).
enum : uint32_t {
  DERR_TRACEBACK = 1u << 0,   // invalid pointer reached (the reference panics here)
  DERR_GEOMETRY = 1u << 1,    // a pair exceeded the scratch bounds it was sized for
  DERR_BAND_RANGE = 1u << 2,  // vectorized band bookkeeping left the compressed matrix
  DERR_UNSUPPORTED = 1u << 3, // band wider than the row-major kernel supports
  DERR_LAMBDA = 1u << 4,      // a non-ACGT code reached the lambda product
};

// Scratch geometry for the NW kernels, sized by the host for a pool.
struct NwGeom {
  int32_t lmax;        // longest sequence
  int32_t vec_ncol;    // bound on the vectorized compressed width
  int32_t vec_nrow;    // 2*lmax+1
  int32_t rm_pairs;    // bound on offset pairs of the row-major band (ceil(W/2))
  int32_t nwarps;      // resident warps of the persistent NW kernels
  size_t vec_scratch;  // bytes per warp (pointer matrix)
  size_t rm_scratch;   // bytes per warp (pointer bit planes)
  int32_t forms;       // the aligner forms a compare launch can reach (kForms*)
};
// Aligner forms a compare launch can reach, fixed by the pool's geometry and
// parameters; k_align is compiled once per set, so a launch runs only the code
// it can use (a smaller kernel: fewer instruction-cache misses in the
// latency-bound late calls, and no register pressure from unused forms).
constexpr int32_t kFormsAll = 0;   // every form
constexpr int32_t kFormsVec1 = 1;  // gapless and the fast register form with one lane group
constexpr int32_t kFormsRm = 2;    // gapless and the row-major forms

// ---- shared-memory carving, used by kernels and by the host sizing code ----
constexpr int kScreenWarps = 8;   // warps per screen CTA
constexpr int kScreenSmemTasks = 128; // tasks whose table the screen keeps in shared memory
constexpr int kNwWarps = 4;       // warps per NW CTA
constexpr int kAlignCtasPerSm = 4; // resident align CTAs per SM (128 registers per thread)
constexpr int kStageBytes = 4096; // traceback staging per warp
constexpr uint32_t kNoPivot = 0xffffffffu;
constexpr int kRmStageRows = 128; // anti-diagonals of pointer planes the row-major traceback stages at once
constexpr int kStoreSpan = 2048;  // raws per store CTA (its own output segment)
constexpr int kStoreThreads = 256; // threads per store CTA
constexpr int kSeqPad = 160;      // guard bytes on each side of the aligners' shared-memory sequences

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~size_t(15); }
__host__ __device__ inline size_t err_smem_bytes(int ncol) { return align16(size_t(16) * size_t(ncol) * 8); }
__host__ __device__ inline size_t screen_smem_per_warp(uint32_t maxlen) {
  return align16(size_t(maxlen) * 2) + align16(maxlen);
}
__host__ __device__ inline int rm_kbound(int rm_pairs) {
  int k = (rm_pairs + 31) / 32, b = 1;
  while (b < k) b <<= 1;
  return b;
}
__host__ __device__ inline size_t nw_smem_per_warp_vec(const NwGeom& g) {
  return align16(g.lmax + 2 * kSeqPad) * 2 + align16(size_t(3) * g.vec_ncol * 2) + align16(size_t(g.vec_ncol) * 2) +
         align16(g.vec_ncol) + align16(kStageBytes) + align16(g.lmax) + align16(size_t(g.lmax) * 2) +
         align16(g.lmax);
}
__host__ __device__ inline size_t rm_stage_bytes(int kbound) { return align16(size_t(kRmStageRows) * 2 * kbound * 4); }
// The lambda indices (2 bytes per raw position) are built after the traceback
// is done with the staged window, so they share its bytes when they fit.
__host__ __device__ inline bool rm_fidx_in_stage(int lmax, int kbound) {
  return size_t(lmax) * 2 <= rm_stage_bytes(kbound);
}
__host__ __device__ inline size_t nw_smem_per_warp_rm(const NwGeom& g) {
  const int kb = rm_kbound(g.rm_pairs);
  return align16(g.lmax) * 2 + rm_stage_bytes(kb) + align16(g.lmax) +
         (rm_fidx_in_stage(g.lmax, kb) ? 0 : align16(size_t(g.lmax) * 2));
}
// The align kernel carves either layout from the same per-warp region, sized
// for the forms the geometry lets a pair take (a zero scratch size marks a
// form no pair of the launch can reach: the register form needs a vectorized
// launch without homopolymer gaps and both lengths <= 3500; every other pair
// is row-major).
__host__ __device__ inline size_t align_smem_per_warp(const NwGeom& g) {
  const size_t a = g.vec_scratch ? nw_smem_per_warp_vec(g) : 0, b = g.rm_scratch ? nw_smem_per_warp_rm(g) : 0;
  const size_t m = a > b ? a : b;
  return m > 16 ? m : 16;
}

// ---- launchers (dgpu_kernels.cu) ----
void launch_fill_f64(double* p, size_t n, double v, cudaStream_t st);
void launch_profiles(const uint8_t* seq, const uint32_t* off, const uint32_t* len, uint32_t nraw,
                     int k, uint8_t* kmer8, uint8_t* sat, cudaStream_t st);
// k = 8: sparse profiles (see PoolDev::kidx); lmax bounds every length.
void launch_profiles_sparse(const uint8_t* seq, const uint32_t* off, const uint32_t* len, uint32_t nraw,
                            uint32_t lmax, uint16_t* kidx, uint8_t* kcnt, uint32_t* knum, uint8_t* sat,
                            cudaStream_t st);
// Runs screen/gapless/lambda, both NW kernels and the ordered store for `ntask`
// tasks; `task_prefix` holds ntask+1 running raw counts.
struct CompareLaunch {
  PoolDev pool;
  KParams kp;
  const TaskDev* tasks;
  const uint32_t* task_prefix;
  uint32_t ntask;
  uint32_t total_items;
  uint32_t screen_chunk;    // items a k_screen warp takes at a time (4..32; set by launch_compare)
  uint32_t screen_chunk_max;  // tuning: the largest chunk launch_compare may pick (16 or 32)
  uint32_t screen_blocks_per_sm;  // tuning: k_screen blocks per SM in its one wave (1..4)
  // Pivot bound: with `pivot` the screen keeps each raw's pivot and records
  // each task's center as cl_center[base + cluster]; with `cdot_ready`
  // k_pivot_dots has filled cdot for clusters [0, cluster) of every task
  // (task_cl_prefix: prefix sums of the tasks' cluster indices) and the
  // screen excludes raws by the bound.
  uint32_t pivot, cdot_ready;
  uint32_t pdl;  // tuning: launch the align and store kernels as programmatic dependents
  const uint32_t* task_cl_prefix;
  uint32_t total_cl;
  uint32_t* queue_pass;     // nraw capacity: items that passed the screen
  uint32_t* queue_counts;   // 8 words; [4] = items pushed to queue_pass, [5] = profiles the
                            // screen read, [6] = the align warps' slot cursor
  uint8_t* nw_scratch;      // nwarps * max(vec_scratch, rm_scratch)
  NwGeom geom;
  uint32_t* err_word;
  // store outputs
  uint32_t* comp_index;
  double* comp_lambda;
  uint32_t* comp_ham;
  float* comp_ll32;         // with kp.lambda32: each stored comp's FP32 ln(lambda); else null
  double* task_self;        // ntask
  // store CTAs: CTA b covers raws [store_chunk[b]*kStoreSpan, +kStoreSpan) of
  // task store_task[b]; blk_counters[b] = its counters, TC_STORED its count
  const uint32_t* store_task;
  const uint32_t* store_chunk;
  uint32_t* blk_counters;
  uint32_t nstore_blocks;
  int do_store;
  // with do_store: the store's first CTA copies *err_word to err_host (mapped
  // host memory) and clears queue_counts for the launch context's next call
  uint32_t* err_host;
  // null: the fields above are this call's; else the launch is a graph
  // replay and ntask, total_items, screen_chunk, nstore_blocks, pivot,
  // cdot_ready, total_cl and the table pointers come from *hdr
  const CallHeader* hdr;
};
// ev (optional): 4 events recorded before the screen and after screen, align
// and store, for per-kernel device times.
void launch_compare(const CompareLaunch& L, cudaStream_t st, cudaEvent_t* ev = nullptr);
// The screen's chunk size for a call of `total` items (launch_compare's rule).
uint32_t compare_screen_chunk(uint32_t total, uint32_t screen_blocks_per_sm, uint32_t screen_chunk_max);
// Captures the compare sequence on `st` as a graph for replay with L.hdr set:
// `screen_grid` screen CTAs, k_pivot_dots when `pivot_dots`, k_align and
// `store_grid` store CTAs (spare screen warps find no chunk, spare store CTAs
// return at once). Returns 0 and sets *out (the caller instantiates it or
// updates an instantiated one and destroys it), or a CUDA error code.
int capture_compare_graph(const CompareLaunch& L, cudaStream_t st, uint32_t screen_grid, bool pivot_dots,
                          uint32_t store_grid, cudaGraph_t* out);

// Final-subs pass (src/dada.rs:609-673) feeding the transition counts
// (src/error.rs:194-249): item i realigns raw[i] against center[i]; counts go
// to out + sample[i] * 16 * tncol. Items are ordered by sample.
struct FinalSubsLaunch {
  PoolDev pool;
  KParams kp;  // the run's parameters with use_kmers = 0
  NwGeom geom;
  uint8_t* nw_scratch;
  const uint32_t* raw;
  const uint32_t* center;
  const uint32_t* sample;
  uint32_t nitems;
  int tncol;      // columns counted (the error matrix's, or 1 without qualities)
  int has_quals;  // count at the raw's quality (else column 0)
  uint32_t* out;
  unsigned long long* out64;  // non-null: counts go here (64-bit) instead of out
  uint32_t* err_word;
};
void launch_final_subs(const FinalSubsLaunch& F, cudaStream_t st);

// Alignment-only entry used by the parity tests: emits al0/al1 strings.
void launch_align_debug(int which, const uint8_t* s1cat, const uint32_t* off1, const uint32_t* len1,
                        const uint8_t* s2cat, const uint32_t* off2, const uint32_t* len2, uint32_t npairs,
                        KParams kp, int end_gap, const NwGeom& geom, uint8_t* scratch, uint8_t* al0,
                        uint8_t* al1, const uint32_t* aloff, uint32_t* alen, uint32_t* err_word,
                        cudaStream_t st);

// Records the message dgpu_last_error() returns on this thread.
void set_last_error(const char* msg);

// Host wait limit for a compare launch, in seconds: DGPU_WAIT_LIMIT_S, else
// 300. No launch of this library runs anywhere near that long (the largest
// workloads' launches take milliseconds), so reaching it means the device
// stopped making progress.
inline double wait_limit_s() {
  static const double limit = [] {
    const char* v = std::getenv("DGPU_WAIT_LIMIT_S");
    const double x = v ? std::atof(v) : 0.0;
    return x > 0.0 ? x : 300.0;
  }();
  return limit;
}

// Waits for queued device work by polling `query` (cudaStreamQuery on the
// stream) and yielding the thread between polls, for at most limit_s
// seconds. Returns cudaSuccess once the work is done, the first error other
// than cudaErrorNotReady that query reports, or cudaErrorTimeout when the work
// is still running at the limit; the work is then left queued, and the
// caller reports the failure instead of blocking for good.
template <class Query>
cudaError_t poll_with_limit(Query query, double limit_s) {
  const auto t0 = std::chrono::steady_clock::now();
  for (uint64_t k = 0;; ++k) {
    const cudaError_t q = query();
    if (q != cudaErrorNotReady) return q;
    if ((k & 63) == 63 &&
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit_s)
      return cudaErrorTimeout;
    std::this_thread::yield();
  }
}

}  // namespace dgpu

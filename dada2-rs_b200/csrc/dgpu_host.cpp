// Host side of the B200 compare step: device pools, the clustering loop that
// drives the compare kernels, and the C ABI declared in include/dada2_b200.h.
//
// The loop restates run_dada (src/dada.rs:749-1110): compare cluster 0 with the
// screen off, then bud -> compare -> shuffle -> p-update until nothing buds. The
// compare (screen, alignment, lambda, store) runs on the GPU; the serial phases
// (shuffle, p-update, bud) run here, one host thread per sample in batch mode.
#include <dlfcn.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cctype>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "dada2_b200.h"
#include "dgpu_common.h"

namespace dgpu {

static thread_local std::string g_err;

static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

void set_last_error(const char* msg) { g_err = msg; }

#define CUDA_TRY(x)                                                                     \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess) return fail(DGPU_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define TRY(x)            \
  do {                    \
    int r_ = (x);         \
    if (r_ != 0) return r_; \
  } while (0)

using Clock = std::chrono::steady_clock;
static double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

// Process-wide kernel accounting behind dgpu_stats_*.
struct GlobalStats {
  std::mutex mu;
  dgpu_kernel_stats s{};
  std::atomic<uint64_t> timing_every{0};  // time every N-th compare call (0: none)
  std::atomic<uint64_t> call_seq{0};
  std::vector<double> round_ms;  // latency of each compare call (launch to results on the host)
};
static GlobalStats g_stats;

// Host-to-device bytes the compare path copies (uploads, lock flags, task tables).
static void count_h2d(uint64_t bytes) {
  std::lock_guard<std::mutex> g(g_stats.mu);
  g_stats.s.h2d_bytes += bytes;
}

// ---------------------------------------------------------------------------
// Block cache. A finished pool gives its device and mapped-host blocks back
// here (after synchronizing its stream, so every block in the cache is idle)
// and the next pool takes blocks of about the size it asks for, so repeated
// calls on similar batches do not pay for cudaMalloc / cudaHostAlloc / free
// again. A block serves requests from half its size up to its size. The cache
// holds at most kCacheCap bytes per device and kind; dgpu_cache_release empties
// it, and a failed cudaMalloc empties it for that device and retries.
// ---------------------------------------------------------------------------
constexpr int kCacheDevs = 64;
constexpr size_t kCacheCap = size_t(32) << 30;

struct HostBlock {
  void* h;
  void* d;
};

struct BlockCache {
  std::mutex mu;
  std::multimap<size_t, void*> dev[kCacheDevs];
  std::multimap<size_t, HostBlock> host[kCacheDevs];
  size_t dev_bytes[kCacheDevs] = {};
  size_t host_bytes[kCacheDevs] = {};
};

static BlockCache& block_cache() {
  static BlockCache* c = new BlockCache;  // never destroyed: no CUDA calls at process exit
  return *c;
}

static size_t block_round(size_t b) {
  const size_t g = b >= (size_t(2) << 20) ? (size_t(2) << 20) : size_t(4096);
  return (b + g - 1) / g * g;
}

static int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

static void* cache_take_dev(int dev, size_t bytes, size_t* got) {
  if (dev < 0 || dev >= kCacheDevs) return nullptr;
  BlockCache& c = block_cache();
  std::lock_guard<std::mutex> g(c.mu);
  auto it = c.dev[dev].lower_bound(bytes);
  if (it == c.dev[dev].end() || it->first > 2 * bytes) return nullptr;
  void* p = it->second;
  *got = it->first;
  c.dev_bytes[dev] -= it->first;
  c.dev[dev].erase(it);
  return p;
}

static bool cache_put_dev(int dev, size_t bytes, void* p) {
  if (dev < 0 || dev >= kCacheDevs) return false;
  BlockCache& c = block_cache();
  std::lock_guard<std::mutex> g(c.mu);
  if (c.dev_bytes[dev] + bytes > kCacheCap) return false;
  c.dev[dev].emplace(bytes, p);
  c.dev_bytes[dev] += bytes;
  return true;
}

static bool cache_take_host(int dev, size_t bytes, size_t* got, HostBlock* out) {
  if (dev < 0 || dev >= kCacheDevs) return false;
  BlockCache& c = block_cache();
  std::lock_guard<std::mutex> g(c.mu);
  auto it = c.host[dev].lower_bound(bytes);
  if (it == c.host[dev].end() || it->first > 2 * bytes) return false;
  *out = it->second;
  *got = it->first;
  c.host_bytes[dev] -= it->first;
  c.host[dev].erase(it);
  return true;
}

static bool cache_put_host(int dev, size_t bytes, HostBlock b) {
  if (dev < 0 || dev >= kCacheDevs) return false;
  BlockCache& c = block_cache();
  std::lock_guard<std::mutex> g(c.mu);
  if (c.host_bytes[dev] + bytes > kCacheCap) return false;
  c.host[dev].emplace(bytes, b);
  c.host_bytes[dev] += bytes;
  return true;
}

// Frees every cached block of `dev` (all devices when dev < 0); returns the
// number of bytes released.
static size_t cache_release(int dev) {
  BlockCache& c = block_cache();
  std::lock_guard<std::mutex> g(c.mu);
  size_t freed = 0;
  int prev = current_device();
  for (int d = 0; d < kCacheDevs; ++d) {
    if (dev >= 0 && d != dev) continue;
    if (c.dev[d].empty() && c.host[d].empty()) continue;
    cudaSetDevice(d);
    for (auto& kv : c.dev[d]) cudaFree(kv.second);
    for (auto& kv : c.host[d]) cudaFreeHost(kv.second.h);
    freed += c.dev_bytes[d] + c.host_bytes[d];
    c.dev[d].clear();
    c.host[d].clear();
    c.dev_bytes[d] = c.host_bytes[d] = 0;
  }
  cudaSetDevice(prev);
  return freed;
}

// ---------------------------------------------------------------------------
// Buffers. release() frees at once (cudaFree waits for the device, so a block
// still read by queued work is safe); recycle() hands an idle block to the
// cache and is only called once the owner's stream has drained.
// ---------------------------------------------------------------------------
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  size_t bytes = 0;
  int dev = -1;
  int alloc(size_t count) {
    release();
    if (count == 0) count = 1;
    const size_t want = block_round(count * sizeof(T));
    const int d = current_device();
    size_t got = 0;
    void* q = cache_take_dev(d, want, &got);
    if (!q) {
      cudaError_t e = cudaMalloc(&q, want);
      if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        cache_release(d);
        e = cudaMalloc(&q, want);
      }
      if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DGPU_E_NOMEM, "cudaMalloc(" + std::to_string(count * sizeof(T)) + " bytes): " +
                                      cudaGetErrorString(e));
      }
      got = want;
    }
    p = static_cast<T*>(q);
    n = count;
    bytes = got;
    dev = d;
    return 0;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = bytes = 0;
  }
  void recycle() {
    if (p && !cache_put_dev(dev, bytes, p)) cudaFree(p);
    p = nullptr;
    n = bytes = 0;
  }
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
};

// Pinned host memory mapped into the device address space: the store kernel
// writes its small per-call outputs straight into it.
template <class T>
struct HBuf {
  T* h = nullptr;
  T* d = nullptr;
  size_t n = 0;
  size_t bytes = 0;
  int dev = -1;
  int alloc(size_t count) {
    release();
    if (count == 0) count = 1;
    const size_t want = block_round(count * sizeof(T));
    const int dv = current_device();
    size_t got = 0;
    HostBlock b{nullptr, nullptr};
    if (!cache_take_host(dv, want, &got, &b)) {
      cudaError_t e = cudaHostAlloc(&b.h, want, cudaHostAllocMapped);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DGPU_E_NOMEM, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
      }
      e = cudaHostGetDevicePointer(&b.d, b.h, 0);
      if (e != cudaSuccess) {
        cudaFreeHost(b.h);
        cudaGetLastError();
        return fail(DGPU_E_CUDA, std::string("cudaHostGetDevicePointer: ") + cudaGetErrorString(e));
      }
      got = want;
    }
    h = static_cast<T*>(b.h);
    d = static_cast<T*>(b.d);
    n = count;
    bytes = got;
    dev = dv;
    return 0;
  }
  void release() {
    if (h) cudaFreeHost(h);
    h = d = nullptr;
    n = bytes = 0;
  }
  void recycle() {
    if (h && !cache_put_host(dev, bytes, HostBlock{h, d})) cudaFreeHost(h);
    h = d = nullptr;
    n = bytes = 0;
  }
  HBuf() = default;
  HBuf(const HBuf&) = delete;
  HBuf& operator=(const HBuf&) = delete;
  ~HBuf() { release(); }
};

template <class... B>
static void recycle_all(B&... b) {
  (b.recycle(), ...);
}

// ---------------------------------------------------------------------------
// Device pool: the resident uniques of one or more samples
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Tuning table: the launch shape of the compare step per read-length class
// (class 0: longest unique <= 200 nt, 1: <= 600 nt, 2: longer). Filled by the
// autotuner (dada2_b200/autotune.py sweeps these knobs on synthetic workloads
// of each class and saves the fastest), loaded at first use from
// DGPU_TUNING_FILE or else tuning.txt beside this library, and set or saved
// through dgpu_tuning_*. The DGPU_LAUNCH_SLOTS / DGPU_BATCH_MAX /
// DGPU_DEDICATED_SLOTS environment variables still override it. Without a
// table the built-in values below apply (measured on the 40-sample
// 250/220-nt batch).
// ---------------------------------------------------------------------------
static const dgpu_tuning kTuneDefault = {6, 4, 1, kAlignCtasPerSm, 32, 4, 32768, 1};
static std::mutex g_tune_mu;
static dgpu_tuning g_tune[3] = {kTuneDefault, kTuneDefault, kTuneDefault};
static bool g_tune_loaded = false;

static int length_class(uint32_t lmax) { return lmax <= 200 ? 0 : (lmax <= 600 ? 1 : 2); }

static bool tuning_valid(const dgpu_tuning& t) {
  return t.launch_slots >= 1 && t.launch_slots <= 8 && t.samples_per_launch >= 1 && t.samples_per_launch <= 4096 &&
         t.dedicated_slots >= 0 && t.dedicated_slots <= 7 && t.align_ctas_per_sm >= 1 &&
         t.align_ctas_per_sm <= kAlignCtasPerSm && (t.screen_chunk_max == 16 || t.screen_chunk_max == 32) &&
         t.screen_blocks_per_sm >= 1 && t.screen_blocks_per_sm <= 4 && t.pivot_min_items >= 0 &&
         (t.programmatic_launch == 0 || t.programmatic_launch == 1);
}

// Text form: one line per class, "class C launch_slots A samples_per_launch B
// dedicated_slots D align_ctas_per_sm E screen_chunk_max F
// screen_blocks_per_sm G"; '#' starts a comment. Unknown keys are an error.
static int tuning_parse(const std::string& text, dgpu_tuning out[3], std::string* msg) {
  dgpu_tuning t[3] = {g_tune[0], g_tune[1], g_tune[2]};
  size_t pos = 0;
  int lineno = 0;
  while (pos < text.size()) {
    size_t e = text.find('\n', pos);
    if (e == std::string::npos) e = text.size();
    std::string line = text.substr(pos, e - pos);
    pos = e + 1;
    ++lineno;
    const size_t h = line.find('#');
    if (h != std::string::npos) line.resize(h);
    std::vector<std::string> tok;
    size_t q = 0;
    while (q < line.size()) {
      while (q < line.size() && std::isspace(static_cast<unsigned char>(line[q]))) ++q;
      size_t r = q;
      while (r < line.size() && !std::isspace(static_cast<unsigned char>(line[r]))) ++r;
      if (r > q) tok.push_back(line.substr(q, r - q));
      q = r;
    }
    if (tok.empty()) continue;
    if (tok.size() % 2 != 0 || tok[0] != "class") {
      *msg = "tuning line " + std::to_string(lineno) + ": expected 'class C key value ...'";
      return DGPU_E_INVALID;
    }
    const int c = std::atoi(tok[1].c_str());
    if (c < 0 || c > 2 || tok[1].find_first_not_of("0123456789") != std::string::npos) {
      *msg = "tuning line " + std::to_string(lineno) + ": class must be 0, 1 or 2";
      return DGPU_E_INVALID;
    }
    dgpu_tuning v = t[c];
    for (size_t k = 2; k + 1 < tok.size(); k += 2) {
      const int x = std::atoi(tok[k + 1].c_str());
      if (tok[k] == "launch_slots") v.launch_slots = x;
      else if (tok[k] == "samples_per_launch") v.samples_per_launch = x;
      else if (tok[k] == "dedicated_slots") v.dedicated_slots = x;
      else if (tok[k] == "align_ctas_per_sm") v.align_ctas_per_sm = x;
      else if (tok[k] == "screen_chunk_max") v.screen_chunk_max = x;
      else if (tok[k] == "screen_blocks_per_sm") v.screen_blocks_per_sm = x;
      else if (tok[k] == "pivot_min_items") v.pivot_min_items = x;
      else if (tok[k] == "programmatic_launch") v.programmatic_launch = x;
      else {
        *msg = "tuning line " + std::to_string(lineno) + ": unknown key " + tok[k];
        return DGPU_E_INVALID;
      }
    }
    if (!tuning_valid(v)) {
      *msg = "tuning line " + std::to_string(lineno) + ": value out of range";
      return DGPU_E_INVALID;
    }
    t[c] = v;
  }
  for (int c = 0; c < 3; ++c) out[c] = t[c];
  return 0;
}

static std::string tuning_format(const dgpu_tuning t[3]) {
  std::string o = "# compare-step launch shape per read-length class (0: <= 200 nt, 1: <= 600 nt, 2: longer)\n";
  for (int c = 0; c < 3; ++c)
    o += "class " + std::to_string(c) + " launch_slots " + std::to_string(t[c].launch_slots) +
         " samples_per_launch " + std::to_string(t[c].samples_per_launch) + " dedicated_slots " +
         std::to_string(t[c].dedicated_slots) + " align_ctas_per_sm " + std::to_string(t[c].align_ctas_per_sm) +
         " screen_chunk_max " + std::to_string(t[c].screen_chunk_max) + " screen_blocks_per_sm " +
         std::to_string(t[c].screen_blocks_per_sm) + " pivot_min_items " + std::to_string(t[c].pivot_min_items) +
         " programmatic_launch " + std::to_string(t[c].programmatic_launch) + "\n";
  return o;
}

// Under g_tune_mu.
static int tuning_load_file(const std::string& path, std::string* msg) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    *msg = "cannot open tuning file " + path;
    return DGPU_E_INVALID;
  }
  std::string text;
  char buf[4096];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
  std::fclose(f);
  dgpu_tuning t[3];
  const int rc = tuning_parse(text, t, msg);
  if (rc) return rc;
  for (int c = 0; c < 3; ++c) g_tune[c] = t[c];
  return 0;
}

// Under g_tune_mu: on first use, the table of DGPU_TUNING_FILE or of
// tuning.txt beside this library (a missing or malformed file leaves the
// built-in table).
static void tuning_first_use() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  std::string path;
  if (const char* e = std::getenv("DGPU_TUNING_FILE")) {
    path = e;
  } else {
    Dl_info info{};
    if (dladdr(reinterpret_cast<void*>(&tuning_first_use), &info) && info.dli_fname) {
      path = info.dli_fname;
      const size_t sl = path.rfind('/');
      path = (sl == std::string::npos ? std::string(".") : path.substr(0, sl)) + "/tuning.txt";
    }
  }
  if (path.empty()) return;
  if (FILE* f = std::fopen(path.c_str(), "rb")) {
    std::fclose(f);
    std::string msg;
    (void)tuning_load_file(path, &msg);
  }
}

static dgpu_tuning tuning_class(int c) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  tuning_first_use();
  return g_tune[c];
}
static dgpu_tuning tuning_for(uint32_t lmax) { return tuning_class(length_class(lmax)); }

// Compare calls replay captured CUDA graphs unless DGPU_COMPARE_GRAPHS=0.
static bool compare_graphs_on() {
  static const bool on = [] {
    const char* e = std::getenv("DGPU_COMPARE_GRAPHS");
    return !(e && e[0] == '0');
  }();
  return on;
}

// Launch slots dedicated to the longest chains: DGPU_DEDICATED_SLOTS (0..7) if
// set, else the tuning table's (1 built in).
static size_t dedicated_slots(uint32_t lmax) {
  if (const char* e = std::getenv("DGPU_DEDICATED_SLOTS")) {
    const int v = std::atoi(e);
    if (v >= 0 && v <= 7) return size_t(v);
  }
  return size_t(tuning_for(lmax).dedicated_slots);
}

struct Pool;

// One launch context: its own stream, queue, NW scratch, task tables and store
// bookkeeping, so that compares of different samples can be in flight at once.
// Results land in the pool's raw-indexed arrays, which concurrent launches
// never share: a sample has at most one compare pending.
// Compare graphs by variant (screen grid, store grid, k_pivot_dots), each
// with the fixed launch parameters it was captured for.
struct GraphSet {
  struct Entry {
    cudaGraphExec_t exec = nullptr;
    CompareLaunch key;
  };
  std::map<uint32_t, Entry> by_variant;
};
static std::mutex g_graph_mu;
static std::vector<GraphSet*> g_graph_free[64];  // per device; never freed (the execs outlive pools)
static GraphSet* graph_set_take(int dev) {
  std::lock_guard<std::mutex> g(g_graph_mu);
  std::vector<GraphSet*>& f = g_graph_free[dev & 63];
  if (f.empty()) return new GraphSet();
  GraphSet* s = f.back();
  f.pop_back();
  return s;
}
static void graph_set_return(int dev, GraphSet* s) {
  std::lock_guard<std::mutex> g(g_graph_mu);
  g_graph_free[dev & 63].push_back(s);
}

struct Slot {
  Pool* P = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  DBuf<uint32_t> queue_pass, queue_counts, err_dev;
  DBuf<uint8_t> scratch;
  DBuf<uint8_t> dpack;  // tasks | task prefix | store map of the current launch
  HBuf<uint8_t> hpack;  // its pinned staging copy (one upload per launch)
  HBuf<uint32_t> blk_counters, err_host;
  HBuf<double> task_self;
  HBuf<TaskDev> task_stage;
  std::vector<uint32_t> task_blk0;  // first store CTA of each task in the latest launch
  uint32_t ntask_cap = 0, nblk_cap = 0;
  size_t pack_cap = 0;
  // Instantiated compare graphs, checked out of a per-device free list for
  // the slot's lifetime and handed back after it (a new pool's slots update
  // them in place instead of instantiating again).
  GraphSet* gs = nullptr;
  bool graphs_failed = false;
  int dev = 0;  // the slot's device

  ~Slot() {
    if (st && cudaStreamSynchronize(st) == cudaSuccess && gs) graph_set_return(dev, gs);
    if (st && cudaStreamSynchronize(st) == cudaSuccess)  // every block is idle now
      recycle_all(queue_pass, queue_counts, err_dev, scratch, dpack, hpack, blk_counters, err_host, task_self,
                  task_stage);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }

  int init(Pool* pool, bool high_priority = false) {
    P = pool;
    CUDA_TRY(cudaGetDevice(&dev));
    int lo = 0, hi = 0;
    CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CUDA_TRY(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, high_priority ? hi : lo));
    for (auto& e : ev) CUDA_TRY(cudaEventCreate(&e));
    TRY(queue_counts.alloc(8));
    TRY(err_dev.alloc(1));
    TRY(err_host.alloc(2));  // [0] error flags, [1] profiles the screen read
    err_host.h[0] = 0;
    err_host.h[1] = 0;
    // both start at zero; every call leaves them at zero again
    CUDA_TRY(cudaMemsetAsync(queue_counts.p, 0, 32, st));
    CUDA_TRY(cudaMemsetAsync(err_dev.p, 0, 4, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return 0;
  }

  int ensure_tasks(uint32_t ntask) {
    if (ntask <= ntask_cap) return 0;
    uint32_t cap = std::max<uint32_t>(ntask, 64);
    TRY(task_self.alloc(cap));
    TRY(task_stage.alloc(cap));
    ntask_cap = cap;
    return 0;
  }

  int ensure_blocks(uint32_t nblk) {
    if (nblk <= nblk_cap) return 0;
    const uint32_t cap = std::max<uint32_t>(nblk, 256);
    TRY(blk_counters.alloc(size_t(cap) * TC_NCOUNTERS));
    nblk_cap = cap;
    return 0;
  }

  int ensure_pack(size_t bytes) {
    if (bytes <= pack_cap) return 0;
    const size_t cap = std::max<size_t>(bytes, 16384);
    TRY(hpack.alloc(cap));
    TRY(dpack.alloc(cap));
    pack_cap = cap;
    return 0;
  }

  template <class F>
  void for_each_stored(uint32_t t, F&& f) const;
  void task_counters(uint32_t t, uint32_t* out) const;
  int run_compare(uint32_t ntask, bool do_store, double* wait_s);
};

// Device pool: the resident uniques of one or more samples.
struct Pool {
  int device = 0;
  cudaStream_t st = nullptr;  // uploads and resets
  uint32_t nraw = 0, lmax = 0, lmin = 0;
  KParams kp{};
  NwGeom geom{};
  int sms = 148;
  // Compare calls replay captured graphs (Slot::run_compare): on for pools
  // that serve many batch runs (resident batches, learn-errors, compare
  // contexts), where the graphs' set-up is paid once; a one-shot denoising
  // launches directly.
  bool replay_graphs = false;
  // The largest length difference of two uniques that are ever compared (a
  // batch compares only within a sample); -1: any two uniques of the pool.
  // It bounds the aligners' band geometry.
  int64_t pair_spread = -1;
  int nslots = 1;
  DBuf<uint8_t> seq, qual, kmer8, sat, lock, status;
  DBuf<uint32_t> off, len, reads, ham, knum;
  DBuf<uint16_t> kidx;
  DBuf<uint8_t> kcnt;
  DBuf<double> e_minmax, err, lambda;
  DBuf<float> loglam32;
  DBuf<uint32_t> piv_dot, piv_cl, cl_center, cdot;  // the screen's pivot bound (PoolDev)
  bool pivot_on = false;  // the clustering loop runs here: keep pivots and use the bound
  // stored comps of each task, at the task's first raw (its sample's base)
  HBuf<uint32_t> comp_index, comp_ham;
  HBuf<double> comp_lambda;
  HBuf<float> comp_ll32;  // with kp.lambda32: FP32 ln(lambda) of each stored comp
  HBuf<uint8_t> lock_host;  // pinned host copy of every lock flag
  bool has_qual = false;
  std::vector<std::unique_ptr<Slot>> slots;

  ~Pool() {
    slots.clear();  // each slot drains its own stream first
    if (st && cudaStreamSynchronize(st) == cudaSuccess)
      recycle_all(seq, qual, kmer8, sat, lock, status, off, len, reads, ham, knum, kidx, kcnt, e_minmax, err, lambda, loglam32,
                  comp_index, comp_ham, comp_lambda, comp_ll32, lock_host, piv_dot, piv_cl, cl_center, cdot);
    if (st) cudaStreamDestroy(st);
  }

  // nslot launch contexts are made once the pool's geometry is known.
  int init(int dev, int nslot = 1) {
    device = dev;
    nslots = std::max(1, nslot);
    CUDA_TRY(cudaSetDevice(dev));
    CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return 0;
  }

  Slot& slot0() { return *slots[0]; }
  // seqs: codes 1..4 concatenated; quals_u8 may be null.
  int upload(uint32_t n, const uint8_t* seqs, const uint32_t* offs, const uint32_t* lens, const uint8_t* quals_u8,
             const uint32_t* rd, const KParams& params, const double* errm) {
    kp = params;
    nraw = n;
    lmax = 0;
    lmin = 0xffffffffu;
    uint64_t total = 0;
    for (uint32_t t = 0; t < n; ++t) {
      lmax = std::max(lmax, lens[t]);
      lmin = std::min(lmin, lens[t]);
      total += lens[t];
    }
    if (total >= 0xffffffffull) return fail(DGPU_E_UNSUPPORTED, "more than 4 GiB of sequence in one pool");
    has_qual = quals_u8 != nullptr;
    // Sequences already packed back to back (offs[t] = running length) go up
    // as they are; anything else is packed first.
    bool contiguous = true;
    {
      uint64_t w = 0;
      for (uint32_t t = 0; t < n && contiguous; ++t) {
        contiguous = offs[t] == w;
        w += lens[t];
      }
    }
    std::vector<uint32_t> o;
    std::vector<uint8_t> packed, qpacked;
    const uint8_t* seq_src = seqs;
    const uint8_t* qual_src = quals_u8;
    const uint32_t* off_src = offs;
    if (!contiguous) {
      o.resize(n);
      packed.resize(total ? total : 1);
      if (has_qual) qpacked.resize(total ? total : 1);
      uint64_t w = 0;
      for (uint32_t t = 0; t < n; ++t) {
        o[t] = uint32_t(w);
        std::memcpy(packed.data() + w, seqs + offs[t], lens[t]);
        if (has_qual) std::memcpy(qpacked.data() + w, quals_u8 + offs[t], lens[t]);
        w += lens[t];
      }
      seq_src = packed.data();
      qual_src = has_qual ? qpacked.data() : nullptr;
      off_src = o.data();
    }
    const size_t seq_bytes = total ? size_t(total) : 1;
    const size_t nk = size_t(1) << (2 * kp.kmer_size);
    TRY(seq.alloc(seq_bytes));
    TRY(off.alloc(n));
    TRY(len.alloc(n));
    TRY(reads.alloc(n));
    TRY(lock.alloc(n));
    TRY(status.alloc(n));
    TRY(ham.alloc(n));
    TRY(lambda.alloc(n));
    TRY(loglam32.alloc(n));
    TRY(e_minmax.alloc(n));
    TRY(err.alloc(size_t(16) * kp.ncol));
    const bool sparse = kp.use_kmers && kp.kmer_size >= 8;  // src/kmers.rs:213-221
    TRY(kmer8.alloc(kp.use_kmers && !sparse ? size_t(n) * nk : 1));
    TRY(kidx.alloc(sparse ? seq_bytes : 1));
    TRY(kcnt.alloc(sparse ? seq_bytes : 1));
    TRY(knum.alloc(sparse ? n : 1));
    TRY(sat.alloc(n));
    {
      const size_t pn = kp.use_kmers && !sparse ? size_t(n) : 1;
      TRY(piv_dot.alloc(pn));
      TRY(piv_cl.alloc(pn));
      TRY(cl_center.alloc(pn));
      TRY(cdot.alloc(pn));
    }
    TRY(comp_index.alloc(n));
    TRY(comp_ham.alloc(n));
    TRY(comp_lambda.alloc(n));
    if (kp.lambda32) TRY(comp_ll32.alloc(n));
    TRY(lock_host.alloc(n));
    std::memset(lock_host.h, 0, n);
    if (has_qual) {
      TRY(qual.alloc(seq_bytes));
      if (total) CUDA_TRY(cudaMemcpyAsync(qual.p, qual_src, size_t(total), cudaMemcpyHostToDevice, st));
    }
    if (total) CUDA_TRY(cudaMemcpyAsync(seq.p, seq_src, size_t(total), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(off.p, off_src, size_t(n) * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(len.p, lens, size_t(n) * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(reads.p, rd, size_t(n) * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(err.p, errm, size_t(16) * kp.ncol * 8, cudaMemcpyHostToDevice, st));
    count_h2d(uint64_t(total) * (has_qual ? 2 : 1) + uint64_t(n) * 12 + uint64_t(16) * kp.ncol * 8);
    CUDA_TRY(cudaMemsetAsync(lock.p, 0, n, st));
    TRY(reset_e_minmax());
    if (kp.use_kmers) {
      if (sparse)
        launch_profiles_sparse(seq.p, off.p, len.p, n, lmax, kidx.p, kcnt.p, knum.p, sat.p, st);
      else
        launch_profiles(seq.p, off.p, len.p, n, kp.kmer_size, kmer8.p, sat.p, st);
      std::lock_guard<std::mutex> g(g_stats.mu);
      g_stats.s.launches[0] += 1;
    }
    CUDA_TRY(cudaGetLastError());
    const auto tn0 = Clock::now();
    TRY(size_nw());
    const auto tn1 = Clock::now();
    CUDA_TRY(cudaStreamSynchronize(st));  // the staging vectors go out of scope
    {
      std::lock_guard<std::mutex> g(g_stats.mu);
      g_stats.s.prepare_ms[2] += 1e3 * secs(tn0, tn1);
      g_stats.s.prepare_ms[3] += 1e3 * secs(tn1, Clock::now());
    }
    return 0;
  }

  // Per-run device state: every e_minmax back to -999 (B::new,
  // src/containers.rs:342) and no raw with a pivot yet.
  int reset_e_minmax() {
    launch_fill_f64(e_minmax.p, nraw, -999.0, st);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemsetAsync(piv_cl.p, 0xff, piv_cl.n * 4, st));
    CUDA_TRY(cudaMemsetAsync(piv_dot.p, 0, piv_dot.n * 4, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return 0;
  }

  int size_nw() {
    const bool use_homo = kp.homo_gap != kp.gap && kp.homo_gap <= 0;
    const bool vec_possible = kp.vectorized && !use_homo && lmin <= 3500;
    const bool rm_possible = use_homo || !kp.vectorized || lmax > 3500;
    geom.lmax = int32_t(lmax);
    const int64_t bb = kp.band < 0 ? int64_t(lmax) : int64_t(kp.band);
    int64_t diff = int64_t(lmax) - int64_t(lmin);
    if (pair_spread >= 0 && pair_spread < diff) diff = pair_spread;
    geom.vec_ncol = int32_t(4 + (std::min<int64_t>(bb, lmax) + 1) / 2 + std::min<int64_t>(bb + diff, lmax) / 2);
    geom.vec_nrow = int32_t(2 * lmax + 1);
    int64_t W = kp.band < 0 ? int64_t(2 * lmax + 1) : std::min<int64_t>(2 * bb + diff + 1, 2 * int64_t(lmax) + 1);
    geom.rm_pairs = int32_t(std::min<int64_t>((W + 1) / 2, 512));
    const int kb = rm_kbound(geom.rm_pairs);
    // byte matrix for the shared-memory form, two u32 bit-planes per 32 columns
    // (at most 4 groups) for the register form
    geom.vec_scratch = vec_possible ? align16(size_t(geom.vec_nrow) * std::max<size_t>(size_t(geom.vec_ncol), 32)) : 0;
    geom.rm_scratch = rm_possible ? align16(size_t(2 * lmax + 1) * 2 * kb * 4) : 0;
    geom.nwarps = sms * tuning_for(lmax).align_ctas_per_sm * kNwWarps;
    // the forms k_align can reach (vec_align_any takes the fast register form
    // with one lane group for every pair when the compressed width is <= 32,
    // gaps are not positive and no sum can saturate i16)
    geom.forms = kFormsAll;
    if (rm_possible && !vec_possible) {
      geom.forms = kFormsRm;
    } else if (vec_possible && !rm_possible) {
      const int64_t pmax = std::max<int64_t>({int64_t(kp.match), int64_t(kp.mismatch), 0});
      if (geom.vec_ncol <= 32 && kp.gap <= 0 && pmax * (int64_t(lmax) + 1) <= 32767) geom.forms = kFormsVec1;
    }
    const size_t per = std::max<size_t>(std::max(geom.vec_scratch, geom.rm_scratch), 16);
    slots.clear();
    for (int k = 0; k < nslots; ++k) {
      slots.emplace_back(new Slot);
      Slot& L = *slots.back();
      TRY(L.init(this, nslots > 1 && size_t(k) < dedicated_slots(lmax)));  // the dedicated slots come first
      TRY(L.scratch.alloc(per * size_t(geom.nwarps)));
      TRY(L.queue_pass.alloc(nraw));
    }
    return 0;
  }

  PoolDev view() const {
    PoolDev v;
    v.seq = seq.p;
    v.qual = has_qual ? qual.p : nullptr;
    v.off = off.p;
    v.len = len.p;
    v.kmer8 = kmer8.p;
    v.sat = sat.p;
    v.kidx = kidx.p;
    v.kcnt = kcnt.p;
    v.knum = knum.p;
    v.reads = reads.p;
    v.lock = lock.p;
    v.e_minmax = e_minmax.p;
    v.err = err.p;
    v.res_lambda = lambda.p;
    v.res_ham = ham.p;
    v.res_status = status.p;
    v.res_loglam32 = loglam32.p;
    v.piv_dot = piv_dot.p;
    v.piv_cl = piv_cl.p;
    v.cl_center = cl_center.p;
    v.cdot = cdot.p;
    v.nraw = nraw;
    v.maxlen = lmax;
    return v;
  }

  int push_locks(uint32_t base, uint32_t n, cudaStream_t s) {
    CUDA_TRY(cudaMemcpyAsync(lock.p + base, lock_host.h + base, n, cudaMemcpyHostToDevice, s));
    count_h2d(n);
    return 0;
  }
};

// Stored comps of task t (latest launch), in ascending raw order.
template <class F>
void Slot::for_each_stored(uint32_t t, F&& f) const {
  const TaskDev& T = task_stage.h[t];
  const uint32_t nb = (T.n + kStoreSpan - 1) / kStoreSpan;
  for (uint32_t b = 0; b < nb; ++b) {
    const uint32_t cnt = blk_counters.h[size_t(task_blk0[t] + b) * TC_NCOUNTERS + TC_STORED];
    const uint32_t o = T.out_off + b * uint32_t(kStoreSpan);
    const float* ll = P->kp.lambda32 && P->comp_ll32.h ? P->comp_ll32.h + o : nullptr;
    for (uint32_t k = 0; k < cnt; ++k)
      f(P->comp_index.h[o + k], P->comp_lambda.h[o + k], P->comp_ham.h[o + k],
        ll ? ll[k] : std::numeric_limits<float>::quiet_NaN());
  }
}

// Counters of task t summed over its store CTAs.
void Slot::task_counters(uint32_t t, uint32_t* out) const {
  for (int k = 0; k < TC_NCOUNTERS; ++k) out[k] = 0;
  const uint32_t nb = (task_stage.h[t].n + kStoreSpan - 1) / kStoreSpan;
  for (uint32_t b = 0; b < nb; ++b)
    for (int k = 0; k < TC_NCOUNTERS; ++k) out[k] += blk_counters.h[size_t(task_blk0[t] + b) * TC_NCOUNTERS + k];
}

// Launches one compare over `ntask` tasks already in task_stage; waits for it.
// The launch's tables go up in one copy; with the store, the error flags come
// back through mapped memory and the queue counters are rearmed on the device.
int Slot::run_compare(uint32_t ntask, bool do_store, double* wait_s) {
  const auto t_call = Clock::now();
  TRY(ensure_tasks(ntask));
  const Pool& Q = *P;
  uint32_t total = 0, nblk = 0;
  task_blk0.assign(ntask, 0);
  for (uint32_t t = 0; t < ntask; ++t) {
    task_stage.h[t].out_off = task_stage.h[t].base;
    task_blk0[t] = nblk;
    nblk += (task_stage.h[t].n + kStoreSpan - 1) / kStoreSpan;
  }
  TRY(ensure_blocks(nblk));
  // header | tasks | task prefix | cluster prefix | store map
  const size_t o_tasks = align16(sizeof(CallHeader));
  const size_t o_pref = o_tasks + align16(sizeof(TaskDev) * ntask);
  const size_t o_clp = o_pref + align16(size_t(4) * (ntask + 1));
  const size_t o_map = o_clp + align16(size_t(4) * (ntask + 1));
  const size_t pack_bytes = o_map + align16(size_t(8) * std::max<uint32_t>(nblk, 1));
  TRY(ensure_pack(pack_bytes));
  std::memcpy(hpack.h + o_tasks, task_stage.h, sizeof(TaskDev) * ntask);
  uint32_t* pref = reinterpret_cast<uint32_t*>(hpack.h + o_pref);
  uint32_t* smap = reinterpret_cast<uint32_t*>(hpack.h + o_map);
  for (uint32_t t = 0; t < ntask; ++t) {
    pref[t] = total;
    total += task_stage.h[t].n;
    const uint32_t nb = (task_stage.h[t].n + kStoreSpan - 1) / kStoreSpan;
    for (uint32_t b = 0; b < nb; ++b) {
      smap[task_blk0[t] + b] = t;
      smap[nblk + task_blk0[t] + b] = b;
    }
  }
  pref[ntask] = total;
  // the pivot bound: clusters [0, cluster) of each task get a center dot
  uint32_t* clp = reinterpret_cast<uint32_t*>(hpack.h + o_clp);
  uint32_t total_cl = 0;
  const bool pivot = Q.pivot_on && Q.kp.use_kmers && Q.kp.kmer_size <= 7;
  for (uint32_t t = 0; t < ntask; ++t) {
    clp[t] = total_cl;
    const TaskDev& T = task_stage.h[t];
    if (pivot && T.cluster < T.n) total_cl += T.cluster;
  }
  clp[ntask] = total_cl;
  const uint32_t min_items = uint32_t(tuning_for(Q.lmax).pivot_min_items);
  const bool cdot_ready = pivot && total_cl > 0 && min_items > 0 && total >= min_items;
  const dgpu_tuning tu = tuning_for(Q.lmax);
  {
    CallHeader& H = *reinterpret_cast<CallHeader*>(hpack.h);
    H = CallHeader{};
    H.ntask = ntask;
    H.total_items = total;
    H.screen_chunk = compare_screen_chunk(total, uint32_t(tu.screen_blocks_per_sm), uint32_t(tu.screen_chunk_max));
    H.nstore_blocks = nblk;
    H.pivot = pivot ? 1u : 0u;
    H.cdot_ready = cdot_ready ? 1u : 0u;
    H.total_cl = cdot_ready ? total_cl : 0u;
    H.o_tasks = uint32_t(o_tasks);
    H.o_pref = uint32_t(o_pref);
    H.o_clp = uint32_t(o_clp);
    H.o_map = uint32_t(o_map);
  }
  CUDA_TRY(cudaMemcpyAsync(dpack.p, hpack.h, pack_bytes, cudaMemcpyHostToDevice, st));
  count_h2d(pack_bytes);
  CompareLaunch L;
  std::memset(&L, 0, sizeof L);  // padding too: graph_key compares the bytes
  L.pool = Q.view();
  L.kp = Q.kp;
  L.tasks = reinterpret_cast<const TaskDev*>(dpack.p + o_tasks);
  L.task_prefix = reinterpret_cast<const uint32_t*>(dpack.p + o_pref);
  L.ntask = ntask;
  L.total_items = total;
  L.queue_pass = queue_pass.p;
  L.queue_counts = queue_counts.p;
  L.nw_scratch = scratch.p;
  L.geom = Q.geom;
  L.err_word = err_dev.p;
  L.comp_index = Q.comp_index.d;
  L.comp_lambda = Q.comp_lambda.d;
  L.comp_ham = Q.comp_ham.d;
  L.comp_ll32 = Q.kp.lambda32 && Q.comp_ll32.h ? Q.comp_ll32.d : nullptr;
  L.task_self = task_self.d;
  L.store_task = reinterpret_cast<const uint32_t*>(dpack.p + o_map);
  L.store_chunk = L.store_task + nblk;
  L.blk_counters = blk_counters.d;
  L.nstore_blocks = nblk;
  L.do_store = do_store ? 1 : 0;
  L.err_host = err_host.d;
  {
    L.screen_chunk_max = uint32_t(tu.screen_chunk_max);
    L.screen_blocks_per_sm = uint32_t(tu.screen_blocks_per_sm);
    L.pdl = uint32_t(tu.programmatic_launch);
  }
  L.pivot = pivot ? 1u : 0u;
  L.cdot_ready = cdot_ready ? 1u : 0u;
  L.task_cl_prefix = reinterpret_cast<const uint32_t*>(dpack.p + o_clp);
  L.total_cl = cdot_ready ? total_cl : 0u;
  const uint64_t every = g_stats.timing_every.load();
  const bool timing = every != 0 && g_stats.call_seq.fetch_add(1) % every == 0;
  bool launched = false;
  if (do_store && !timing && total > 0 && Q.replay_graphs && compare_graphs_on() && !graphs_failed) {
    // Replay a captured graph of the launch sequence: one submission instead
    // of three or four, which the launch slots' threads otherwise contend
    // for in the driver. Its kernels take this call's values from the
    // header just uploaded; the store grid is rounded up (spare CTAs return).
    CompareLaunch K = L;
    K.ntask = K.total_items = K.screen_chunk = K.nstore_blocks = 0;
    K.pivot = K.cdot_ready = K.total_cl = 0;
    K.tasks = nullptr;
    K.task_prefix = K.task_cl_prefix = K.store_task = K.store_chunk = nullptr;
    K.hdr = reinterpret_cast<const CallHeader*>(dpack.p);
    if (!gs) gs = graph_set_take(dev);
    // the screen's grid as launch_compare sizes it, rounded up to a power of
    // two (at least 64, at most the one wave); the store grid to 8 x 4^j
    const CallHeader& H = *reinterpret_cast<const CallHeader*>(hpack.h);
    const uint32_t bps = (tu.screen_blocks_per_sm >= 1 && tu.screen_blocks_per_sm <= 4) ? uint32_t(tu.screen_blocks_per_sm) : 4u;
    const uint32_t wave = uint32_t(Q.sms) * bps;
    const uint32_t need = uint32_t((uint64_t(total) + uint64_t(kScreenWarps) * H.screen_chunk - 1) /
                                   (uint64_t(kScreenWarps) * H.screen_chunk));
    uint32_t sgrid = 64;
    while (sgrid < need && sgrid < wave) sgrid *= 2;
    sgrid = std::min(sgrid, wave);
    uint32_t grid = 8;
    while (grid < nblk) grid *= 4;
    const uint32_t key = (sgrid << 20) ^ (grid << 1) ^ (cdot_ready ? 1u : 0u);
    GraphSet::Entry& E = gs->by_variant[key];
    if (!E.exec || std::memcmp(&E.key, &K, sizeof K) != 0) {
      cudaGraph_t g = nullptr;
      bool ok = capture_compare_graph(K, st, sgrid, cdot_ready, grid, &g) == 0 && g;
      if (ok && E.exec) {  // same shape, new parameters: update in place
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(E.exec, g, &info) != cudaSuccess) {
          (void)cudaGetLastError();
          cudaGraphExecDestroy(E.exec);
          E.exec = nullptr;
        }
      }
      if (ok && !E.exec) ok = cudaGraphInstantiate(&E.exec, g, 0) == cudaSuccess;
      if (g) cudaGraphDestroy(g);
      if (ok) {
        E.key = K;
      } else {
        (void)cudaGetLastError();
        if (E.exec) cudaGraphExecDestroy(E.exec);
        gs->by_variant.erase(key);
        graphs_failed = true;  // direct launches from here on
      }
    }
    if (!graphs_failed) {
      CUDA_TRY(cudaGraphLaunch(gs->by_variant[key].exec, st));
      launched = true;
    }
  }
  if (!launched) launch_compare(L, st, timing ? ev : nullptr);
  CUDA_TRY(cudaGetLastError());
  if (!do_store) {  // no store kernel to rearm the queue or report the flags
    CUDA_TRY(cudaMemcpyAsync(err_host.h, err_dev.p, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(err_host.h + 1, queue_counts.p + 5, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemsetAsync(queue_counts.p, 0, 32, st));
  }
  auto t0 = Clock::now();
  // Poll and yield rather than block in the driver's spin: the launch slots'
  // threads share the cores with the host phases they wait for (on B200 with
  // 16 host cores the 40-sample step went from 79-82 ms to 75-78 ms).
  const cudaError_t q = poll_with_limit([&] { return cudaStreamQuery(st); }, wait_limit_s());
  if (q == cudaErrorTimeout)
    return fail(DGPU_E_CUDA, "compare launch still running after the wait limit (DGPU_WAIT_LIMIT_S, default 300 s); "
                             "the context must not be reused");
  CUDA_TRY(q);
  const auto t1 = Clock::now();
  if (wait_s) *wait_s += secs(t0, t1);
  {
    float ms[3] = {0, 0, 0};
    if (timing)
      for (int k = 0; k < 3; ++k) CUDA_TRY(cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]));
    uint64_t screened = 0;
    if (do_store)
      for (uint32_t b = 0; b < nblk; ++b) screened += blk_counters.h[size_t(b) * TC_NCOUNTERS + TC_SCREENED];
    std::lock_guard<std::mutex> g(g_stats.mu);
    dgpu_kernel_stats& S = g_stats.s;
    S.launches[1] += 1;
    S.launches[2] += 1;
    if (do_store) S.launches[3] += 1;
    for (int k = 0; k < 3; ++k) S.ms[k + 1] += ms[k];
    S.rounds += 1;
    S.compares += total;
    S.screened += screened;
    // algorithmic screen bytes: the 4^k profile of every raw whose profile the
    // screen read (screened raws less those the pivot bound excluded), or
    // for k = 8 the sparse list of every screened raw (3 bytes per present
    // k-mer, at most L - k + 1); 16 B of metadata per compare, 8 more for the
    // pivot when the loop keeps pivots; and both profiles of each center dot
    const uint64_t prof = Q.kp.kmer_size >= 8 ? uint64_t(3) * (Q.lmax - uint32_t(Q.kp.kmer_size) + 1)
                                              : (uint64_t(1) << (2 * Q.kp.kmer_size));
    const uint64_t nread = Q.kp.kmer_size >= 8 ? screened : uint64_t(err_host.h[1]);
    const uint64_t sb = nread * prof + uint64_t(total) * (pivot ? 24u : 16u) +
                        (cdot_ready ? uint64_t(total_cl) * 2u * prof : 0u);
    S.screen_bytes += sb;
    if (timing) {
      S.timed_rounds += 1;
      S.timed_screen_bytes += sb;
      S.timed_compares += total;
    }
    if (g_stats.round_ms.size() < (size_t(1) << 20)) g_stats.round_ms.push_back(1e3 * secs(t_call, t1));
  }
  const uint32_t ew = *reinterpret_cast<volatile uint32_t*>(err_host.h);
  if (ew) {
    std::string what;
    if (ew & DERR_TRACEBACK) what += " invalid traceback pointer;";
    if (ew & DERR_GEOMETRY) what += " alignment exceeded its scratch bounds;";
    if (ew & DERR_BAND_RANGE) what += " vectorized band left the compressed matrix;";
    if (ew & DERR_UNSUPPORTED) what += " band wider than 1024 offsets on the row-major aligner;";
    if (ew & DERR_LAMBDA) what += " non-ACGT code or quality beyond the error matrix in lambda;";
    err_host.h[0] = 0;
    err_host.h[1] = 0;
    CUDA_TRY(cudaMemsetAsync(err_dev.p, 0, 4, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return fail(ew & DERR_UNSUPPORTED ? DGPU_E_UNSUPPORTED : DGPU_E_DEVICE, "device error:" + what);
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Fork-join helpers for the large loops inside one sample's host phases. The
// calling thread always works on its own loop, so a busy pool only means less
// help, never a wait on unstarted work.
// ---------------------------------------------------------------------------
class Helpers {
 public:
  static Helpers& get() {
    static Helpers h(std::max(1, int(std::thread::hardware_concurrency()) / 2));
    return h;
  }
  // fn(chunk_index, lo, hi) over [0, n) in chunks of `grain`.
  void parallel_for(size_t n, size_t grain, const std::function<void(size_t, size_t, size_t)>& fn) {
    const size_t nch = (n + grain - 1) / grain;
    if (nch <= 1 || th_.empty()) {
      for (size_t c = 0; c < nch; ++c) fn(c, c * grain, std::min(n, (c + 1) * grain));
      return;
    }
    auto task = std::make_shared<Task>();
    task->fn = &fn;
    task->n = n;
    task->grain = grain;
    task->nch = nch;
    {
      std::lock_guard<std::mutex> g(mu_);
      q_.push_back(task);
    }
    cv_.notify_all();
    run(*task);
    while (task->done.load(std::memory_order_acquire) < nch) std::this_thread::yield();
  }
  ~Helpers() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }

 private:
  struct Task {
    const std::function<void(size_t, size_t, size_t)>* fn = nullptr;
    size_t n = 0, grain = 1, nch = 0;
    std::atomic<size_t> next{0}, done{0};
  };
  explicit Helpers(int n) {
    for (int t = 0; t < n; ++t) th_.emplace_back([this] { loop(); });
  }
  static void run(Task& t) {
    for (;;) {
      const size_t c = t.next.fetch_add(1);
      if (c >= t.nch) break;
      (*t.fn)(c, c * t.grain, std::min(t.n, (c + 1) * t.grain));
      t.done.fetch_add(1, std::memory_order_release);
    }
  }
  void loop() {
    for (;;) {
      std::shared_ptr<Task> t;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return stop_ || !q_.empty(); });
        if (stop_) return;
        t = q_.front();
        if (t->next.load() >= t->nch) {
          q_.pop_front();
          continue;
        }
      }
      run(*t);
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::shared_ptr<Task>> q_;
  bool stop_ = false;
};

static constexpr size_t kParMin = 8192;   // loops shorter than this stay serial
static constexpr size_t kParGrain = 2048;
static constexpr size_t kParMinRepriced = 16384;  // repriced members worth splitting a reprice for
static constexpr size_t kRepriceGrain = 256;   // members per reprice chunk

// ---------------------------------------------------------------------------
// Clustering state of one sample (containers.rs B/Bi/Raw, SoA)
// ---------------------------------------------------------------------------
struct Comp {
  uint32_t i = 0, index = 0;
  double lambda = 0.0;
  uint32_t hamming = 0;
};
struct BudCand {
  double p;
  uint32_t reads;
  uint32_t r;
  uint32_t raw;
};
// A raw's candidate cluster (index_add_cluster, src/cluster.rs:731-739). A
// sample keeps all of them in one pool, each raw's as a list in the order
// they were added (ascending cluster index), so the loop makes no per-raw
// allocations.
struct Cand {
  uint32_t ci;
  uint32_t hamming;
  uint32_t next;  // the raw's next candidate in the pool, or kNoCand
  double lambda;
};
static constexpr uint32_t kNoCand = 0xffffffffu;
// One bit per member position: set where the member at that position has
// the property. Updated with the member list, so scans can skip the rest.
struct PosBits {
  std::vector<uint64_t> w;
  std::vector<uint64_t> sum;  // bit k set iff w[k] != 0, so sparse scans skip empty words
  bool get(size_t r) const { return (r >> 6) < w.size() && ((w[r >> 6] >> (r & 63)) & 1u); }
  void put(size_t r, bool v) {
    const size_t k = r >> 6;
    if (k >= w.size()) {
      if (!v) return;
      w.resize(k + 1, 0);
      sum.resize((w.size() + 63) >> 6, 0);
    }
    const uint64_t m = uint64_t(1) << (r & 63);
    w[k] = v ? (w[k] | m) : (w[k] & ~m);
    const uint64_t sm = uint64_t(1) << (k & 63);
    sum[k >> 6] = w[k] ? (sum[k >> 6] | sm) : (sum[k >> 6] & ~sm);
  }
  void clear() {
    std::fill(w.begin(), w.end(), uint64_t(0));
    std::fill(sum.begin(), sum.end(), uint64_t(0));
  }
  // f(r) for every position in [lo, hi) set here and not in ex, ascending
  template <class F>
  void each_excluding(const PosBits& ex, size_t lo, size_t hi, F&& f) const {
    hi = std::min(hi, w.size() * 64);
    for (size_t k = lo >> 6; k * 64 < hi; ++k) {
      uint64_t x = w[k] & ~(k < ex.w.size() ? ex.w[k] : uint64_t(0));
      if (k * 64 < lo) x &= ~uint64_t(0) << (lo & 63);
      while (x) {
        const size_t r = k * 64 + size_t(__builtin_ctzll(x));
        if (r >= hi) return;
        f(r);
        x &= x - 1;
      }
    }
  }
  // f(r) for every set position in [lo, hi), ascending (nonempty words only)
  template <class F>
  void each(size_t lo, size_t hi, F&& f) const {
    hi = std::min(hi, w.size() * 64);
    if (lo >= hi) return;
    const size_t k0 = lo >> 6, k1 = (hi - 1) >> 6;
    for (size_t sk = k0 >> 6; sk <= (k1 >> 6); ++sk) {
      uint64_t y = sum[sk];
      if (sk == (k0 >> 6)) y &= ~uint64_t(0) << (k0 & 63);
      while (y) {
        const size_t k = sk * 64 + size_t(__builtin_ctzll(y));
        y &= y - 1;
        if (k > k1) return;
        uint64_t x = w[k];
        if (k == k0) x &= ~uint64_t(0) << (lo & 63);
        while (x) {
          const size_t r = k * 64 + size_t(__builtin_ctzll(x));
          if (r >= hi) return;
          f(r);
          x &= x - 1;
        }
      }
    }
  }
};

// What a reprice reads of a member, kept beside the member list (position-
// indexed) so the scans run through memory in order: the lambda and hamming of
// the raw's comp to its cluster's center, its reads, and its prior in the top
// bit of hp.
struct MemberInfo {
  double lambda;
  uint32_t reads;
  uint32_t hp;
  uint32_t hamming() const { return hp & 0x7fffffffu; }
  bool prior() const { return (hp >> 31) != 0; }
};

struct Cluster {
  int64_t center = -1;
  std::vector<uint32_t> raws;
  std::vector<MemberInfo> info;  // info[r] describes raws[r]
  PosBits var;    // members that are repriced (not fixed_p)
  PosBits multi;  // members with two or more candidate clusters
  // Members known to price at exactly 0.0 for as long as the cluster's reads
  // stay at or below z_reads (non-prior bud candidates; see pA_floor), by
  // reads descending then position: the reprice skips them and takes the
  // first as its candidate among them. zbits marks their positions (and
  // zcount counts them); zheap is a min-heap on (UINT32_MAX - reads,
  // position, raw) whose entries count only while that position is marked
  // and still holds that raw, so a member leaves the set by clearing its bit.
  std::vector<std::array<uint32_t, 3>> zheap;
  PosBits zbits;
  uint32_t zcount = 0;
  uint32_t z_reads = 0;
  uint32_t reads = 0;
  uint32_t nvar = 0;  // members whose p is repriced (not fixed at 1.0)
  bool update_e = true, check_locks = true;
  double self_ = 0.0;
  int32_t birth_type = 0;
  uint32_t birth_from = 0;
  double birth_pval = 0.0, birth_fold = 1.0, birth_e = 0.0;
  Comp birth_comp;
  std::vector<Comp> comp;
  std::vector<double> comp64;  // with DadaConf::fp32: the FP64 lambda of each comp
};

struct RunStats {
  uint64_t compare_calls = 0, cmp_scanned = 0, screened = 0, aligned = 0, stored = 0;
  uint64_t gapless = 0, vectorized = 0, homo = 0, endsfree = 0, shuffle_calls = 0, shuffle_moves = 0;
  double t_compare = 0, t_total = 0, t_host = 0, t_wait = 0;
  double t_done = -1;  // from the start of the loop until this sample finished
  double t_slot_wait = 0, t_job_wait = 0;  // ready -> launched; results -> host phase started
  Clock::time_point t_mark{};              // when the sample last became ready / got its results
  uint64_t ns_shuffle = 0, ns_pupdate = 0, ns_bud = 0;  // host phases, nanoseconds
};

struct DadaConf {
  double omega_a, omega_p, omega_c, min_fold, kdist_cutoff;
  bool detect_singletons, greedy;
  uint32_t min_hamming, min_abund;
  size_t max_clust;
  bool fp32 = false;  // decisions from the FP32 lambda, FP64 near the thresholds
};

struct SampleState {
  uint32_t n = 0, base = 0;
  uint32_t total_reads = 0;
  const uint32_t* reads = nullptr;  // n entries
  const uint8_t* prior = nullptr;   // n entries
  uint8_t* lock = nullptr;          // n entries, pinned (Pool::lock_host + base)
  std::vector<Comp> rcomp;
  std::vector<double> p;
  std::vector<uint32_t> raw_cluster;
  std::vector<uint32_t> raw_pos;  // position of each raw in its cluster's member list
  std::vector<uint32_t> center_raw;  // each cluster's center (compact, for the shuffle's scans)
  // each cluster's bud cache (src/pval.rs:91-123), kept compact for the bud
  // scan: bm_flags bit 0 = a candidate, bit 1 = a prior candidate
  std::vector<BudCand> bm_c, bmp_c;
  std::vector<uint8_t> bm_flags;
  std::vector<std::pair<uint64_t, uint32_t>> mv_buf;  // move_changed's work list
  std::vector<Cluster> clusters;
  std::vector<Cand> cand_pool;
  std::vector<uint32_t> cand_head, cand_tail;  // per raw: first and last candidate in cand_pool
  std::vector<uint32_t> ncand;   // cand[raw].size(), kept flat for the shuffle scans
  std::vector<uint8_t> fixed_p;  // get_pA answers 1.0 whatever the cluster (src/pval.rs:383)
  uint64_t nalign = 0, nshroud = 0;
  RunStats stats;
  bool lock_dirty = false, done = false;
  int64_t pending = -1;  // cluster whose compare is queued
  // shuffle carry (src/cluster.rs:848-866)
  std::vector<Comp> compmax;
  std::vector<double> emax;
  std::vector<uint32_t> reads_used, dirty_list, reads_fell_list;
  std::vector<uint32_t> changed_raws;  // raws whose best cluster changed since the last move pass
  std::vector<uint32_t> touched_list;  // clusters whose member list changed since the last pass A2
  std::vector<uint8_t> touched;
  std::vector<uint8_t> changed_mark;
  std::vector<uint8_t> in_affected, dirty_cluster, reads_fell;
  std::vector<uint32_t> affected;
  bool built = false;
  const DadaConf* conf = nullptr;

  void init(uint32_t n_, uint32_t base_, const uint32_t* rd, const uint8_t* pr, uint8_t* lk, const DadaConf* c) {
    n = n_;
    base = base_;
    reads = rd;
    prior = pr;
    lock = lk;
    conf = c;
    total_reads = 0;
    for (uint32_t t = 0; t < n; ++t) total_reads += reads[t];
    rcomp.assign(n, Comp());
    p.assign(n, 0.0);
    // A singleton without a prior gets p = 1.0 from get_pA for any cluster
    // (unless singletons are detected), so it is set once here and never
    // repriced. Such a raw never buds: the bud scan starts from p = 1.0 (the
    // p of cluster 0's center, whose own comparison has hamming 0) and the
    // center's reads, and a candidate replaces that only with a smaller p or
    // an equal p and more reads.
    fixed_p.assign(n, 0);
    if (!conf->detect_singletons)
      for (uint32_t t = 0; t < n; ++t)
        if (reads[t] == 1 && !prior[t]) {
          fixed_p[t] = 1;
          p[t] = 1.0;
        }
    raw_cluster.assign(n, 0);
    raw_pos.resize(n);
    cand_pool.clear();
    cand_pool.reserve(size_t(n) + n / 2);
    cand_head.assign(n, kNoCand);
    cand_tail.assign(n, kNoCand);
    ncand.assign(n, 0);
    changed_mark.assign(n, 0);
    clusters.clear();
    center_raw.clear();
    bm_c.clear();
    bmp_c.clear();
    bm_flags.clear();
    Cluster c0;
    c0.birth_e = double(total_reads);
    c0.raws.resize(n);
    c0.info.resize(n);
    for (uint32_t t = 0; t < n; ++t) {
      c0.raws[t] = t;
      raw_pos[t] = t;
      c0.info[t] = member_info(t);
      if (!fixed_p[t]) c0.var.put(t, true);
    }
    c0.reads = total_reads;
    for (uint32_t t = 0; t < n; ++t) c0.nvar += fixed_p[t] ? 0u : 1u;
    clusters.push_back(std::move(c0));
    upd_list.assign(1, 0u);
    assign_center(0);
  }

  void assign_center(size_t i) {  // src/containers.rs:450-463 (last maximum wins)
    Cluster& c = clusters[i];
    if (c.raws.empty()) return;
    uint32_t best = c.raws[0];
    for (uint32_t r : c.raws)
      if (reads[r] >= reads[best]) best = r;
    c.center = best;
    if (center_raw.size() <= i) center_raw.resize(i + 1, UINT32_MAX);
    center_raw[i] = best;
  }

  MemberInfo member_info(uint32_t raw) const {
    return MemberInfo{rcomp[raw].lambda, reads[raw], (rcomp[raw].hamming & 0x7fffffffu) | (prior[raw] ? 0x80000000u : 0u)};
  }
  // rcomp[raw] = cp, and the copy beside the raw's place in its cluster
  void set_rcomp(uint32_t raw, const Comp& cp) {
    rcomp[raw] = cp;
    Cluster& c = clusters[raw_cluster[raw]];
    c.info[raw_pos[raw]] = member_info(raw);
    zero_drop(c, raw_pos[raw]);  // its comp changed: no longer known to price at zero
  }
  static bool zero_valid(const Cluster& c, const std::array<uint32_t, 3>& e) {
    return c.zbits.get(e[1]) && e[1] < c.raws.size() && c.raws[e[1]] == e[2];
  }
  void zero_add(Cluster& c, size_t r, uint32_t raw) {
    if (!c.zbits.get(r)) ++c.zcount;
    c.zbits.put(r, true);
    c.zheap.push_back({UINT32_MAX - reads[raw], uint32_t(r), raw});
    std::push_heap(c.zheap.begin(), c.zheap.end(), std::greater<>());
  }
  // The zero set's first member (most reads, then lowest position), dropping
  // stale heap entries; false when the set is empty.
  bool zero_first(Cluster& c, uint32_t* zr, uint32_t* zpos) {
    if (c.zcount == 0) {
      c.zheap.clear();
      return false;
    }
    if (c.zheap.size() > 2 * size_t(c.zcount) + 4096) {  // mostly stale: rebuild
      std::vector<std::array<uint32_t, 3>> keep;
      keep.reserve(c.zcount);
      for (const auto& e : c.zheap)
        if (zero_valid(c, e)) keep.push_back(e);
      c.zheap.swap(keep);
      std::make_heap(c.zheap.begin(), c.zheap.end(), std::greater<>());
    }
    while (!c.zheap.empty() && !zero_valid(c, c.zheap.front())) {
      std::pop_heap(c.zheap.begin(), c.zheap.end(), std::greater<>());
      c.zheap.pop_back();
    }
    if (c.zheap.empty()) return false;
    *zr = UINT32_MAX - c.zheap.front()[0];
    *zpos = c.zheap.front()[1];
    return true;
  }
  void zero_drop(Cluster& c, size_t r) {
    if (!c.zbits.get(r)) return;
    c.zbits.put(r, false);
    --c.zcount;
  }

  // Frees the per-raw state; batch_run calls it for all samples in parallel
  // rather than leaving hundreds of thousands of small frees to one thread.
  void release() {
    std::vector<Cand>().swap(cand_pool);
    std::vector<uint32_t>().swap(cand_head);
    std::vector<uint32_t>().swap(cand_tail);
    std::vector<Cluster>().swap(clusters);
    std::vector<Comp>().swap(rcomp);
    std::vector<Comp>().swap(compmax);
    std::vector<double>().swap(emax);
    std::vector<double>().swap(p);
    std::vector<uint32_t>().swap(raw_cluster);
    std::vector<uint32_t>().swap(raw_pos);
    std::vector<uint32_t>().swap(ncand);
    std::vector<uint8_t>().swap(fixed_p);
  }

  void add_cand(uint32_t raw, uint32_t ci, double lambda, uint32_t hamming) {
    const uint32_t q = uint32_t(cand_pool.size());
    cand_pool.push_back(Cand{ci, hamming, kNoCand, lambda});
    if (cand_tail[raw] == kNoCand)
      cand_head[raw] = q;
    else
      cand_pool[cand_tail[raw]].next = q;
    cand_tail[raw] = q;
  }

  // clusters whose p-values need repricing: update_e set, listed once
  std::vector<uint32_t> upd_list;
  void mark_update(size_t ci) {
    Cluster& c = clusters[ci];
    if (!c.update_e) {
      c.update_e = true;
      upd_list.push_back(uint32_t(ci));
    }
  }

  void touch(size_t ci) {
    if (ci >= touched.size()) touched.resize(std::max(ci + 1, clusters.size()), 0);
    if (!touched[ci]) {
      touched[ci] = 1;
      touched_list.push_back(uint32_t(ci));
    }
  }

  void add_raw(size_t ci, uint32_t raw) {  // src/containers.rs:403-415
    touch(ci);
    raw_cluster[raw] = uint32_t(ci);
    Cluster& c = clusters[ci];
    const size_t pos = c.raws.size();
    c.info.push_back(member_info(raw));
    raw_pos[raw] = uint32_t(pos);
    c.var.put(pos, !fixed_p[raw]);
    c.multi.put(pos, ncand[raw] > 1);
    clusters[ci].raws.push_back(raw);
    clusters[ci].reads += reads[raw];
    clusters[ci].nvar += fixed_p[raw] ? 0u : 1u;
    mark_update(ci);
  }

  uint32_t pop_raw(size_t ci, size_t r) {  // src/containers.rs:424-435 (swap_remove)
    touch(ci);
    std::vector<uint32_t>& v = clusters[ci].raws;
    Cluster& c = clusters[ci];
    uint32_t raw = v[r];
    const size_t last = v.size() - 1;
    zero_drop(c, r);
    if (last != r && c.zbits.get(last)) {  // the last member moves to r
      c.zbits.put(last, false);
      --c.zcount;
      if (r != 0) zero_add(c, r, v[last]);  // position 0 is never a bud candidate
    }
    v[r] = v.back();
    v.pop_back();
    c.info[r] = c.info.back();
    c.info.pop_back();
    raw_pos[v.size() > r ? v[r] : raw] = uint32_t(r);
    c.var.put(r, c.var.get(last));
    c.multi.put(r, c.multi.get(last));
    c.var.put(last, false);
    c.multi.put(last, false);
    clusters[ci].reads -= reads[raw];
    clusters[ci].nvar -= fixed_p[raw] ? 0u : 1u;
    mark_update(ci);
    return raw;
  }

  TaskDev task_for(size_t ci, double cutoff) const {
    TaskDev T{};
    T.base = base;
    T.n = n;
    T.center = base + uint32_t(clusters[ci].center);
    T.center_reads = reads[clusters[ci].center];
    T.total_reads = double(total_reads);
    T.cutoff = cutoff;
    T.cluster = uint32_t(ci);
    return T;
  }

  // The store's host half: comps from the device into cluster ci (src/cluster.rs:351-397).
  void absorb(size_t ci, const Slot& P, uint32_t t) {
    uint32_t ctr[TC_NCOUNTERS];
    P.task_counters(t, ctr);
    absorb_from(ci, ctr, P.task_self.h[t], [&](auto&& f) { P.for_each_stored(t, f); });
  }

  // absorb for comps from any source: ctr = the call's counters (TC_STORED =
  // the number of comps), self = the center's own lambda, and each(f) calls
  // f(index, lambda, hamming, FP32 ln lambda) for every stored comp in
  // ascending raw order.
  template <class Each>
  void absorb_from(size_t ci, const uint32_t* ctr, double self, Each&& each) {
    const uint32_t ns = ctr[TC_STORED];
    nalign += ctr[TC_SCREENED];
    nshroud += ctr[TC_SHROUD];
    stats.compare_calls++;
    stats.cmp_scanned += n;
    stats.screened += ctr[TC_SCREENED];
    stats.aligned += ctr[TC_ALIGNED];
    stats.stored += ns;
    stats.gapless += ctr[TC_GAPLESS];
    stats.vectorized += ctr[TC_VECTORIZED];
    stats.homo += ctr[TC_HOMO];
    stats.endsfree += ctr[TC_ENDSFREE];
    Cluster& c = clusters[ci];
    c.self_ = self;
    c.comp.clear();
    c.comp.reserve(ns);
    const uint32_t center = uint32_t(c.center);
    c.comp64.clear();
    const bool fp32 = conf->fp32;
    each([&](uint32_t idx, double lam, uint32_t ham, float ll32) {
      // with fp32 the decisions take exp of the FP32 log-sum; the FP64
      // product is kept beside for the threshold fallback
      const double ld = !fp32 || lam == 0.0 ? lam : std::exp(double(ll32));
      const Comp cp{uint32_t(ci), idx, ld, ham};
      c.comp.push_back(cp);
      if (fp32) c.comp64.push_back(lam);
      if (ci == 0 || cp.index == center) set_rcomp(cp.index, cp);
    });
    for (const Comp& cp : c.comp) {  // index_add_cluster
      const uint32_t raw = cp.index;
      add_cand(raw, uint32_t(ci), cp.lambda, cp.hamming);
      // A raw with one candidate keeps its emax implicit (see shuffle_converge);
      // on gaining a second it gets the value the eager updates would hold.
      if (++ncand[raw] == 2) {
        clusters[raw_cluster[raw]].multi.put(raw_pos[raw], true);
        if (built) emax[raw] = compmax[raw].lambda * double(reads_used[compmax[raw].i]);
      }
    }
  }

  // ---- pval.rs ----
  // Bud candidate comparison of the cache scan: smaller p, then more reads;
  // a scan in ascending position keeps the first of equals.
  static bool better(const BudCand& c, const BudCand& m) {
    return c.p < m.p || (c.p == m.p && c.reads > m.reads);
  }

  struct BudAcc {
    bool have = false, havep = false;
    BudCand bm{}, bmp{};
    std::vector<uint32_t> newz;  // positions found to price at zero for good (see pA_floor)
  };

  // get_pA, answering 0.0 at once where calc_pA's log-space tail
  // (upper_tail_direct, reached when gamma_lr's exponent ax is below -709.78
  // and k >= e) is sure to underflow: its log is ln P(X = k) plus the log of
  // a sum below 1 / (1 - e / (k + 1)), and ln P(X = k) = ax - ln k to within
  // rounding; a margin of 1 in the log keeps the test on the safe side.
  double get_pA_quick(uint32_t rd, bool pr, double lambda, uint32_t hamming, uint32_t bi_reads) const {
    if (!(rd == 1 && !pr && !conf->detect_singletons) && hamming != 0 && lambda != 0.0) {
      const double e = lambda * double(bi_reads);
      const double a = double(rd);
      if (e > 0.0 && e < 0.5 * (a + 1.0)) {
        const double ax = a * std::log(e) - e - lgamma_of(a);
        if (ax < -709.78271289338399 && ax - std::log(a) - std::log1p(-e / (a + 1.0)) + 1.0 < -745.2) return 0.0;
      }
    }
    return get_pA(rd, pr, lambda, hamming, bi_reads);
  }

  // A floor under get_pA's value that costs one log and one exp (0.0 when
  // there is none). get_pA's shortcuts are answered exactly. Otherwise p is at
  // least P(X = k) for X ~ Poisson(e), k = rd: the series form of gamma_lr
  // returns exp(ax)/a times a sum of positive terms starting at 1, the
  // continued fraction (e > 1 and e > k) returns at least P(X >= k) less an
  // absolute rounding of about 1e-15, and the conditioning divides by a norm
  // of at most 1. The floor is that P(X = k) = exp(ax)/a, from gamma_lr's own
  // exponent, lowered by 1e-9 relative; it is kept only while it is normal,
  // and in the continued-fraction range only while it is at least 1e-5, so it
  // stays below the computed p whatever its rounding.
  //
  // *zero is set where get_pA is sure to answer exactly 0.0 (then the floor
  // is that answer): get_pA's lambda == 0, or calc_pA's log-space tail
  // underflowing (the test of get_pA_quick, loosened so it needs no log:
  // ax <= k * ex * ln 2 - e - lnGamma(k) for e = m * 2^ex, m in [0.5, 1);
  // -ln k <= 0; -ln(1 - r) <= 2r for r = e / (k + 1) < 1/2).
  //
  // *forever is set where that 0.0 holds for every smaller bi_reads too:
  // lambda == 0, or the underflow test with e added to its left side (as
  // bi_reads falls, e falls, ex does not grow and -e grows by less than e).
  double pA_floor(uint32_t rd, bool pr, double lambda, uint32_t hamming, uint32_t bi_reads, bool* zero,
                  bool* forever) const {
    *zero = false;
    *forever = false;
    if (rd == 1 && !pr && !conf->detect_singletons) return 1.0;
    if (hamming == 0) return 1.0;
    if (lambda == 0.0) {
      *zero = true;
      *forever = true;
      return 0.0;
    }
    const double e = lambda * double(bi_reads);
    if (!(e > 0.0)) return 1.0;
    const double a = double(rd);
    // the Poisson median is at least e - ln 2, so P(X >= k) >= 1/2 for any
    // k <= e - ln 2 (that range is the continued fraction's or gamma_lr's 1.0)
    if (a <= e - 0.7) return 0.49;
    uint64_t bits;
    std::memcpy(&bits, &e, 8);
    const int ex = int((bits >> 52) & 0x7ffu) - 1022;  // e < 2^ex (also for subnormal e)
    const std::vector<double>& lgt = lgamma_table();
    const double lg = rd < lgt.size() ? lgt[rd] : lgamma_of(a);
    const double ax_hi = a * double(ex) * 0.6931471805599453 - e - lg;
    if (ax_hi < -711.0) {  // below gamma_lr's underflow limit: no floor above 0
      const double r = e / (a + 1.0);
      *zero = r < 0.5 && ax_hi + 2.0 * r + 1.0 < -745.2;
      *forever = r < 0.5 && ax_hi + e + 2.0 * r + 1.0 < -745.2;
      return 0.0;
    }
    const double ax = a * std::log(e) - e - lgamma_of(a);
    if (ax < -709.78271289338399) return a < e ? 1.0 : 0.0;  // gamma_lr answers 1.0, then p >= 1.0
    const double lb = std::exp(ax) / a;
    if (!(lb >= 1e-300)) return 0.0;
    if (e > 1.0 && e > a && lb < 1e-5) return 0.0;
    return lb * (1.0 - 1e-9);
  }

  // ---- decision margins ----
  // The smallest relative distance |p - omega| / min(p, omega) of any
  // p-value that a threshold test of the loop compared: the bud's p * nraw
  // against omega_a and the prior raw's p against omega_p
  // (src/cluster.rs:1501-1640), and the final map's p against omega_c
  // (src/dada.rs:525-533). It is symmetric (p = omega / 2 and p = 2 omega
  // both give 1) and +inf for p = 0. A margin far above 1e-12 means that
  // ulp-level differences in the p-values cannot change a decision. +inf when
  // no test of that kind ran.
  double margin[3] = {std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
                      std::numeric_limits<double>::infinity()};
  static double rel_margin(double pv, double omega) {
    const double lo = std::min(pv, omega);
    return lo > 0.0 ? std::fabs(pv - omega) / lo : std::numeric_limits<double>::infinity();
  }

  // ---- FP32 lambda decisions (DadaConf::fp32) ----
  std::atomic<uint64_t> fp32_evals{0}, fp32_fallbacks{0};
  static bool near_threshold(double pv, double omega) { return pv >= omega * 1e-3 && pv <= omega * 1e3; }
  // The FP64 lambda of raw's comp to its cluster's center: the comps of a
  // cluster are in ascending raw order.
  double lambda64_of(uint32_t raw) const {
    const Comp& rc = rcomp[raw];
    const Cluster& c = clusters[rc.i];
    auto it = std::lower_bound(c.comp.begin(), c.comp.end(), raw,
                               [](const Comp& x, uint32_t v) { return x.index < v; });
    if (it == c.comp.end() || it->index != raw || c.comp64.empty()) return rc.lambda;
    return c.comp64[size_t(it - c.comp.begin())];
  }
  // get_pA of a member with the FP32 lambda, repriced from the FP64 product
  // where the bud would test it within 1e3x of omega_a (p times the raws) or,
  // for a prior raw, of omega_p.
  double price_fp32(uint32_t raw, uint32_t bi_reads) {
    const DadaConf& C = *conf;
    const bool pr = prior[raw] != 0;
    double pv = get_pA(reads[raw], pr, rcomp[raw].lambda, rcomp[raw].hamming, bi_reads);
    fp32_evals.fetch_add(1, std::memory_order_relaxed);
    if (near_threshold(pv * double(n), C.omega_a) || (pr && near_threshold(pv, C.omega_p))) {
      pv = get_pA(reads[raw], pr, lambda64_of(raw), rcomp[raw].hamming, bi_reads);
      fp32_fallbacks.fetch_add(1, std::memory_order_relaxed);
    }
    return pv;
  }
  // The plain scan (every member priced), for the FP32 decisions.
  void reprice_range_fp32(const Cluster& bi, size_t lo, size_t hi, BudAcc& acc) {
    const DadaConf& C = *conf;
    const uint32_t bi_reads = bi.reads;
    bi.var.each(lo, hi, [&](size_t r) {
      const uint32_t raw = bi.raws[r];
      const double pv = price_fp32(raw, bi_reads);
      p[raw] = pv;
      if (r == 0) return;
      if (reads[raw] < C.min_abund || rcomp[raw].hamming < C.min_hamming) return;
      if (!(C.min_fold <= 1.0 || double(reads[raw]) >= C.min_fold * rcomp[raw].lambda * double(bi_reads))) return;
      const BudCand cd{pv, reads[raw], uint32_t(r), raw};
      if (!acc.have || better(cd, acc.bm)) {
        acc.bm = cd;
        acc.have = true;
      }
      if (prior[raw] && (!acc.havep || better(cd, acc.bmp))) {
        acc.bmp = cd;
        acc.havep = true;
      }
    });
  }

  // Members [lo, hi) of cluster bi: reprice and fold into a local cache. Only
  // the bud candidates (src/pval.rs:91-123) and cluster 0's center (the bud
  // scan's starting p) read these p-values; the final pass prices every member
  // again. So a candidate whose floor lies above the exact p of the candidate
  // with the lowest floor (above both, for a prior raw) can be neither cache
  // entry and is not priced: the cache is the one a full scan builds.
  //
  // With a zero set, zr / zpos are its first member's reads and position (else
  // zr = 0): a non-prior member with fewer reads, or as many at a later
  // position, can beat that p = 0.0 candidate neither on p nor on the ties,
  // so it is not visited.
  void reprice_range(const Cluster& bi, size_t lo, size_t hi, BudAcc& acc, uint32_t zr = 0,
                     uint32_t zpos = 0) {
    if (conf->fp32) {
      reprice_range_fp32(bi, lo, hi, acc);
      return;
    }
    const DadaConf& C = *conf;
    const uint32_t bi_reads = bi.reads;
    const int64_t ic = clusters[0].center;
    const MemberInfo* info = bi.info.data();
    auto eligible = [&](size_t r) {
      if (r == 0) return false;
      const MemberInfo& m = info[r];
      if (m.reads < C.min_abund || m.hamming() < C.min_hamming) return false;
      return C.min_fold <= 1.0 || double(m.reads) >= C.min_fold * m.lambda * double(bi_reads);
    };
    auto price = [&](size_t r) {
      const MemberInfo& m = info[r];
      return get_pA_quick(m.reads, m.prior(), m.lambda, m.hamming(), bi_reads);
    };
    // pass 1: floors, and the exact p of the lowest-floor candidates
    // (a candidate known to price at exactly 0.0 sets its threshold to 0.0)
    thread_local std::vector<uint32_t> pos;
    thread_local std::vector<double> floor_of;
    thread_local std::vector<uint8_t> zero_of;
    pos.clear();
    if (zr == 0) {
      bi.var.each_excluding(bi.zbits, lo, hi, [&](size_t r) { pos.push_back(uint32_t(r)); });
    } else {
      bi.var.each_excluding(bi.zbits, lo, hi, [&](size_t r) {
        const MemberInfo& m = info[r];
        if (m.prior() || m.reads > zr || (m.reads == zr && r < zpos)) pos.push_back(uint32_t(r));
      });
    }
    floor_of.resize(pos.size());
    zero_of.resize(pos.size());
    double fmin = std::numeric_limits<double>::infinity(), fminp = fmin;
    size_t amin = 0, aminp = 0;
    bool any = false, anyp = false, zmin = false, zminp = false;
    for (size_t i = 0; i < pos.size(); ++i) {
      const size_t r = pos[i];
      if (!eligible(r)) continue;
      const MemberInfo& m = info[r];
      bool z = false, fz = false;
      const double f = pA_floor(m.reads, m.prior(), m.lambda, m.hamming(), bi_reads, &z, &fz);
      floor_of[i] = f;
      zero_of[i] = z;
      if (fz && !m.prior()) acc.newz.push_back(uint32_t(r));
      if (!zmin && (!any || f < fmin || z)) {
        fmin = f;
        amin = r;
        any = true;
        zmin = z;
      }
      if (m.prior() && !zminp && (!anyp || f < fminp || z)) {
        fminp = f;
        aminp = r;
        anyp = true;
        zminp = z;
      }
    }
    const double t = zmin ? 0.0 : (any ? price(amin) : 0.0);
    const double tp = zminp ? 0.0 : (anyp ? price(aminp) : 0.0);
    // pass 2: exact p where it can decide, folded in ascending position
    for (size_t i = 0; i < pos.size(); ++i) {
      const size_t r = pos[i];
      const uint32_t raw = bi.raws[r];
      if (!eligible(r)) {
        if (int64_t(raw) == ic) p[raw] = price(r);
        continue;
      }
      const MemberInfo& m = info[r];
      const double f = floor_of[i];
      const bool pr = m.prior();
      if (f > t && (!pr || f > tp)) continue;
      // nor can it replace the entries this scan holds so far (p >= f)
      auto held = [&](bool have, const BudCand& b) {
        return have && (f > b.p || (f >= b.p && m.reads <= b.reads));
      };
      if (held(acc.have, acc.bm) && (!pr || held(acc.havep, acc.bmp))) continue;
      const double pv = zero_of[i] ? 0.0 : price(r);
      p[raw] = pv;
      const BudCand cd{pv, m.reads, uint32_t(r), raw};
      if (!acc.have || better(cd, acc.bm)) {
        acc.bm = cd;
        acc.have = true;
      }
      if (pr && (!acc.havep || better(cd, acc.bmp))) {
        acc.bmp = cd;
        acc.havep = true;
      }
    }
  }

  void p_update() {  // src/pval.rs:45-130
    const DadaConf& C = *conf;
    bm_c.resize(clusters.size());
    bmp_c.resize(clusters.size());
    bm_flags.resize(clusters.size(), 0);
    // only the listed clusters can have update_e or check_locks set
    std::sort(upd_list.begin(), upd_list.end());
    for (const uint32_t i : upd_list) {
      Cluster& bi = clusters[i];
      if (bi.update_e) {
        const size_t nm = bi.raws.size();
        if (bi.zcount && bi.reads > bi.z_reads) {  // the zero set holds only while reads do not grow
          bi.zheap.clear();
          bi.zcount = 0;
          bi.zbits.clear();
        }
        BudAcc acc;
        uint32_t zr = 0, zpos = 0;  // the zero set's first member, if any
        zero_first(bi, &zr, &zpos);
        const size_t grain = kRepriceGrain;
        // members the scan prices (the zero set is skipped); a short scan
        // stays on this thread, since waking the helpers costs more
        const size_t to_scan = bi.nvar > bi.zcount ? bi.nvar - bi.zcount : 0;
        if (to_scan < kParMinRepriced || nm < 2 * grain) {
          reprice_range(bi, 0, nm, acc, zr, zpos);
        } else {
          // chunk-local caches folded in chunk order: the same first-of-equals
          // winner as one ascending scan
          std::vector<BudAcc> part((nm + grain - 1) / grain);
          Helpers::get().parallel_for(nm, grain, [&](size_t c, size_t lo, size_t hi) {
            reprice_range(bi, lo, hi, part[c], zr, zpos);
          });
          for (const BudAcc& a : part) {
            if (a.have && (!acc.have || better(a.bm, acc.bm))) {
              acc.bm = a.bm;
              acc.have = true;
            }
            if (a.havep && (!acc.havep || better(a.bmp, acc.bmp))) {
              acc.bmp = a.bmp;
              acc.havep = true;
            }
            acc.newz.insert(acc.newz.end(), a.newz.begin(), a.newz.end());
          }
        }
        if (!acc.newz.empty()) {
          for (uint32_t r : acc.newz) zero_add(bi, r, bi.raws[r]);
          bi.z_reads = bi.reads;
        }
        uint32_t zr2 = 0, zp2 = 0;
        if (zero_first(bi, &zr2, &zp2)) {
          // the zero set's first (most reads, then lowest position) is its
          // candidate; against the scanned ones p = 0.0 ties break on reads,
          // then on position (the scan keeps the first of equals)
          const BudCand zc{0.0, zr2, zp2, bi.raws[zp2]};
          if (!acc.have || zc.p < acc.bm.p ||
              (zc.p == acc.bm.p && (zc.reads > acc.bm.reads || (zc.reads == acc.bm.reads && zc.r < acc.bm.r)))) {
            acc.bm = zc;
            acc.have = true;
          }
        }
        bm_c[i] = acc.bm;
        bmp_c[i] = acc.bmp;
        bm_flags[i] = uint8_t((acc.have ? 1 : 0) | (acc.havep ? 2 : 0));
        bi.update_e = false;
      }
      if (C.greedy && bi.check_locks) {
        const int64_t center = bi.center;
        const uint32_t cr = center >= 0 ? reads[center] : 0;
        for (uint32_t raw : bi.raws) {
          const bool l = double(cr) * rcomp[raw].lambda > double(reads[raw]) || int64_t(raw) == center;
          if (l && !lock[raw]) {
            lock[raw] = 1;
            lock_dirty = true;
          }
        }
        bi.check_locks = false;
      }
    }
    upd_list.clear();
  }

  double get_pA(uint32_t rd, bool pr, double lambda, uint32_t hamming, uint32_t bi_reads) const {  // src/pval.rs:376-398
    if (rd == 1 && !pr && !conf->detect_singletons) return 1.0;
    if (hamming == 0) return 1.0;
    if (lambda == 0.0) return 0.0;
    return calc_pA(rd, lambda * double(bi_reads), pr || conf->detect_singletons);
  }

  // lnGamma as statrs 0.18.0's ln_gamma computes it (the function behind
  // Poisson::sf): the Lanczos approximation with G. R. Pugh's parameters
  // ("An Analysis of the Lanczos Gamma Approximation", 2004, p. 116),
  // r = 10.900511 and eleven coefficients, for x >= 0.5:
  //   ln(d_0 + sum_{k=1..10} d_k / ((x + k) - 1)) + ln(2 sqrt(e/pi))
  //     + (x - 0.5) ln(((x - 0.5) + r) / e),
  // summed left to right. Read counts are >= 1, so the x < 0.5 reflection
  // is never needed. It differs from the C library's lgamma by ulps.
  static double ln_gamma_lanczos(double x) {
    static const double kD[11] = {
        2.48574089138753565546e-5,  1.05142378581721974210,     -3.45687097222016235469,
        4.51227709466894823700,     -2.98285225323576655721,    1.05639711577126713077,
        -1.95428773191645869583e-1, 1.70970543404441224307e-2,  -5.71926117404305781283e-4,
        4.63399473359905636708e-6,  -2.71994908488607703910e-9};
    double s = kD[0];
    for (int k = 1; k <= 10; ++k) s = s + kD[k] / (x + double(k) - 1.0);
    return std::log(s) + 0.6207822376352452 + (x - 0.5) * std::log((x - 0.5 + 10.900511) / 2.718281828459045);
  }
  // lnGamma of the integer read counts, filled once with the same function
  // on the same argument, so every value is the one computed on demand.
  static const std::vector<double>& lgamma_table() {
    static const std::vector<double> table = [] {
      std::vector<double> t(size_t(1) << 16);
      for (size_t k = 1; k < t.size(); ++k) t[k] = ln_gamma_lanczos(double(k));
      return t;
    }();
    return table;
  }
  static double lgamma_of(double a) {
    const std::vector<double>& table = lgamma_table();
    if (a >= 1.0 && a < double(table.size()) && a == std::floor(a)) return table[size_t(a)];
    return ln_gamma_lanczos(a);
  }

  // Regularised lower incomplete gamma, statrs 0.18.0's Poisson::sf kernel,
  // following the published Cephes igam/igamc method (series when x <= 1 or
  // x <= a, Legendre continued fraction otherwise). Like statrs it first
  // answers 0.0 for x within 10 * 2^-53 of zero (its default accuracy).
  static double gamma_lr(double a, double x) {
    const double eps = 1e-15, big = 4503599627370496.0, big_inv = 2.22044604925031308085e-16;
    if (std::isnan(a) || std::isnan(x)) return std::numeric_limits<double>::quiet_NaN();
    if (std::fabs(a) < 1.1102230246251565e-15) return 1.0;
    if (std::fabs(x) < 1.1102230246251565e-15) return 0.0;
    const double ax = a * std::log(x) - x - lgamma_of(a);
    if (ax < -709.78271289338399) return a < x ? 1.0 : 0.0;
    if (x <= 1.0 || x <= a) {
      double r = a, c = 1.0, ans = 1.0;
      for (;;) {
        r += 1.0;
        c *= x / r;
        ans += c;
        if (c / ans <= eps) break;
      }
      return std::exp(ax) * ans / a;
    }
    double y = 1.0 - a, z = x + y + 1.0, c = 0.0;
    double p3 = 1.0, q3 = x, p2 = x + 1.0, q2 = z * x, ans = p2 / q2;
    for (;;) {
      y += 1.0;
      z += 2.0;
      c += 1.0;
      const double yc = y * c;
      const double pn = p2 * z - p3 * yc, qn = q2 * z - q3 * yc;
      p3 = p2;
      p2 = pn;
      q3 = q2;
      q2 = qn;
      if (std::fabs(pn) > big) {
        p3 *= big_inv;
        p2 *= big_inv;
        q3 *= big_inv;
        q2 *= big_inv;
      }
      if (qn != 0.0) {
        const double nx = pn / qn, er = std::fabs((ans - nx) / nx);
        ans = nx;
        if (er <= eps) break;
      }
    }
    return 1.0 - std::exp(ax) * ans;
  }

  // ln(k!) as the left-to-right sum log(1) + ... + log(k) of src/pval.rs:333;
  // the table holds the running sums of that same loop.
  static double log_factorial(uint32_t rd) {
    static const std::vector<double> table = [] {
      std::vector<double> t(size_t(1) << 16);
      double acc = 0.0;
      t[0] = 0.0;
      for (size_t k = 1; k < t.size(); ++k) t[k] = acc += std::log(double(k));
      return t;
    }();
    if (rd < table.size()) return table[rd];
    double acc = table.back();
    for (uint32_t t = uint32_t(table.size()); t <= rd; ++t) acc += std::log(double(t));
    return acc;
  }

  static double upper_tail_direct(uint32_t rd, double lambda) {  // src/pval.rs:329-353
    const double k = double(rd);
    const double log_kfact = log_factorial(rd);
    const double log_leading = -lambda + k * std::log(lambda) - log_kfact;
    double sum = 1.0, term = 1.0;
    for (uint32_t j = 1; j < 10000u; ++j) {
      term *= lambda / (k + double(j));
      if (!std::isfinite(term) || term <= 0.0) break;
      const double ns = sum + term;
      if (ns == sum) break;
      sum = ns;
    }
    return std::exp(log_leading + std::log(sum));
  }

  static double calc_pA(uint32_t rd, double e, bool pr) {  // src/pval.rs:208-241
    if (!(e > 0.0)) return 1.0;
    double pv = gamma_lr(double(rd - 1) + 1.0, e);
    if (pv == 0.0 && e > 0.0) pv = upper_tail_direct(rd, e);
    if (pr) return pv;
    double norm = 1.0 - std::exp(-e);
    if (norm < 1e-7) norm = e - 0.5 * e * e;
    return pv / norm;
  }

  // ---- cluster.rs: bud ----
  int64_t bud() {  // src/cluster.rs:1501-1640
    const DadaConf& C = *conf;
    const uint32_t ic = uint32_t(clusters[0].center);
    bool have = false, havep = false;
    BudCand m{}, mp{};
    size_t mci = 0, mpci = 0;
    double min_p = p[ic], min_pp = p[ic];
    uint32_t min_r = reads[ic], min_rp = reads[ic];
    for (size_t ci = 0; ci < bm_flags.size(); ++ci) {
      const uint8_t fl = bm_flags[ci];
      if (!fl) continue;
      const BudCand& bm = bm_c[ci];
      if ((fl & 1) && (bm.p < min_p || (bm.p == min_p && bm.reads > min_r))) {
        have = true;
        m = bm;
        mci = ci;
        min_p = bm.p;
        min_r = bm.reads;
      }
      const BudCand& bmp = bmp_c[ci];
      if ((fl & 2) && (bmp.p < min_pp || (bmp.p == min_pp && bmp.reads > min_rp))) {
        havep = true;
        mp = bmp;
        mpci = ci;
        min_pp = bmp.p;
        min_rp = bmp.reads;
      }
    }
    const double p_a = min_p * double(n);
    if (have) margin[0] = std::min(margin[0], rel_margin(p_a, C.omega_a));
    if (p_a < C.omega_a && have) return bud_tail(mci, m.r, m.raw, p_a, 1);
    if (havep) margin[1] = std::min(margin[1], rel_margin(min_pp, C.omega_p));
    if (min_pp < C.omega_p && havep) return bud_tail(mpci, mp.r, mp.raw, min_pp, 2);
    return -1;
  }

  int64_t bud_tail(size_t ci, uint32_t r, uint32_t raw, double pval, int32_t type) {
    const double expected = rcomp[raw].lambda * double(clusters[ci].reads);
    const Comp bc = rcomp[raw];
    const double fold = double(reads[raw]) / std::max(expected, std::numeric_limits<double>::min());
    pop_raw(ci, r);
    Cluster nb;
    nb.birth_type = type;
    if (type == 1) nb.birth_from = uint32_t(ci);
    nb.birth_pval = pval;
    nb.birth_fold = fold;
    nb.birth_e = expected;
    nb.birth_comp = bc;
    clusters.push_back(std::move(nb));
    const size_t nci = clusters.size() - 1;
    upd_list.push_back(uint32_t(nci));  // born with update_e and check_locks set
    add_raw(nci, raw);
    assign_center(nci);
    return int64_t(nci);
  }

  // ---- cluster.rs: shuffle ----
  size_t move_pass(size_t ci) {  // src/cluster.rs:748-767
    size_t moves = 0;
    size_t r = clusters[ci].raws.size();
    while (r > 0) {
      --r;
      const uint32_t raw = clusters[ci].raws[r];
      const uint32_t best = compmax[raw].i;
      if (best != ci) {
        if (clusters[ci].center == int64_t(raw)) continue;
        pop_raw(ci, r);
        rcomp[raw] = compmax[raw];
        add_raw(best, raw);
        ++moves;
      }
    }
    return moves;
  }

  // src/cluster.rs:792-810. The dirty mark is an atomic test-and-set so the
  // parallel passes below can share it; `out` receives clusters newly marked.
  // A reconcile's output: clusters that hold a raw whose best changed (each
  // once) and those raws.
  struct DirtyOut {
    std::vector<uint32_t> clusters, raws;
  };
  void record_change_to(uint32_t raw, uint32_t new_ci, DirtyOut& out) {
    if (new_ci == compmax[raw].i) return;
    const uint32_t cur = raw_cluster[raw];
    out.raws.push_back(raw);
    if (!__atomic_exchange_n(&dirty_cluster[cur], uint8_t(1), __ATOMIC_RELAXED)) out.clusters.push_back(cur);
  }

  // Pass A2 over one changed cluster's comps [lo, hi) (src/cluster.rs:1177-1224).
  void reconcile_a2(uint32_t ci, double rf, size_t lo, size_t hi, DirtyOut& dirty_out) {
    const std::vector<Comp>& cv = clusters[ci].comp;
    for (size_t k = lo; k < hi; ++k) {
      const Comp& cp = cv[k];
      const uint32_t raw = cp.index;
      if (in_affected[raw]) continue;
      const double e = cp.lambda * rf;
      if (compmax[raw].i == ci) {
        emax[raw] = e;
      } else if (e > emax[raw] || (e == emax[raw] && ci < compmax[raw].i)) {
        emax[raw] = e;
        record_change_to(raw, ci, dirty_out);
        compmax[raw] = cp;
      }
    }
  }

  // Pass B for affected raws [lo, hi): full candidate rescan (src/cluster.rs:1230-1247).
  void reconcile_b(size_t lo, size_t hi, DirtyOut& dirty_out) {
    for (size_t k = lo; k < hi; ++k) {
      const uint32_t raw = affected[k];
      double be = -std::numeric_limits<double>::infinity();
      Comp best;
      for (uint32_t q = cand_head[raw]; q != kNoCand; q = cand_pool[q].next) {
        const Cand& c = cand_pool[q];
        const double e = c.lambda * double(clusters[c.ci].reads);
        if (e > be) {
          be = e;
          best = Comp{c.ci, raw, c.lambda, c.hamming};
        }
      }
      if (best.i != compmax[raw].i) record_change_to(raw, best.i, dirty_out);
      compmax[raw] = best;
      emax[raw] = be;
      in_affected[raw] = 0;
    }
  }

  // Runs fn over [0, n) serially or, for long loops, in parallel chunks whose
  // newly dirtied clusters are appended in chunk order.
  template <class F>
  void par_dirty(size_t n, F&& fn) {
    auto merge = [&](const DirtyOut& d) {
      dirty_list.insert(dirty_list.end(), d.clusters.begin(), d.clusters.end());
      changed_raws.insert(changed_raws.end(), d.raws.begin(), d.raws.end());
    };
    if (n < kParMin) {
      DirtyOut d;
      fn(size_t(0), n, d);
      merge(d);
      return;
    }
    std::vector<DirtyOut> loc((n + kParGrain - 1) / kParGrain);
    Helpers::get().parallel_for(n, kParGrain, [&](size_t c, size_t lo, size_t hi) { fn(lo, hi, loc[c]); });
    for (const DirtyOut& d : loc) merge(d);
  }

  // The move passes of the dirty clusters in ascending order, visiting only
  // the raws whose best cluster changed since the last move pass: after a move
  // pass every raw but a center sits in its best cluster and the best changes
  // only in a reconcile, so these are the only raws a full backward scan would
  // move. Each cluster's movers go in descending position, the full scan's
  // order; a swap_remove brings in the last member, which is never a pending
  // mover, and appends to later clusters leave their positions alone, so the
  // pops and appends are exactly the full passes'.
  size_t move_changed() {
    std::vector<std::pair<uint64_t, uint32_t>>& mv = mv_buf;  // (cluster << 32 | ~position, raw)
    mv.clear();
    for (uint32_t raw : changed_raws) {
      if (changed_mark[raw]) continue;
      changed_mark[raw] = 1;
      const uint32_t ci = raw_cluster[raw];
      if (compmax[raw].i != ci && clusters[ci].center != int64_t(raw))
        mv.push_back({(uint64_t(ci) << 32) | uint64_t(0xffffffffu - raw_pos[raw]), raw});
    }
    for (uint32_t raw : changed_raws) changed_mark[raw] = 0;
    std::sort(mv.begin(), mv.end());
    for (const auto& m : mv) {
      const uint32_t raw = m.second;
      pop_raw(size_t(m.first >> 32), raw_pos[raw]);
      rcomp[raw] = compmax[raw];
      add_raw(compmax[raw].i, raw);
    }
    return mv.size();
  }

  void grow_to(size_t nc) {
    reads_used.resize(nc, 0);
    dirty_cluster.resize(nc, 0);
    reads_fell.resize(nc, 0);
  }

  // src/cluster.rs:908-1320 with the default arms (carry, prune, incremental reconcile).
  void shuffle_converge(size_t max_shuffle) {
    const bool carried = built;
    if (!carried) {
      compmax.assign(n, Comp());
      emax.assign(n, -std::numeric_limits<double>::infinity());
      reads_used.clear();
      dirty_cluster.clear();
      reads_fell.clear();
      grow_to(clusters.size());
      for (const Cluster& bi : clusters) {
        const double cr = double(bi.reads);
        for (const Comp& cp : bi.comp) {
          const double e = cp.lambda * cr;
          if (e > emax[cp.index]) {
            emax[cp.index] = e;
            compmax[cp.index] = cp;
          }
        }
      }
      for (size_t ci = 0; ci < clusters.size(); ++ci) reads_used[ci] = clusters[ci].reads;
      for (uint32_t ci : touched_list) touched[ci] = 0;
      touched_list.clear();
      built = true;
    } else {
      grow_to(clusters.size());
    }
    in_affected.resize(n, 0);
    bool after_reconcile = false, skip_move = carried;
    size_t nshuffle = 0;
    for (;;) {
      if (skip_move) {
        skip_move = false;
        ++nshuffle;
      } else {
        size_t moves = 0;
        if (after_reconcile) {
          moves += move_changed();
        } else {
          for (size_t ci = 0; ci < clusters.size(); ++ci) moves += move_pass(ci);
        }
        changed_raws.clear();
        for (uint32_t ci : dirty_list) dirty_cluster[ci] = 0;
        dirty_list.clear();
        dirty_cluster.resize(clusters.size(), 0);
        stats.shuffle_moves += moves;
        ++nshuffle;
        if (moves == 0 || nshuffle >= max_shuffle) break;
      }
      // Only clusters whose member list changed since the last pass A2 can
      // hold reads other than reads_used (A2 brings every other one level).
      reads_fell.resize(clusters.size(), 0);
      std::sort(touched_list.begin(), touched_list.end());
      for (uint32_t ci : touched_list) {
        if (ci < reads_used.size() && clusters[ci].reads < reads_used[ci] && !reads_fell[ci]) {
          reads_fell[ci] = 1;
          reads_fell_list.push_back(uint32_t(ci));
        }
      }
      // A raw with a single candidate cannot change cluster, and its emax is
      // read only once it has a second candidate (pass A2 reads it through
      // another cluster's comps, which it then has). Its emax is therefore left
      // implicit: the eager updates would hold lambda * reads_used[its cluster],
      // the reads as of the last reconcile, and index_add_cluster writes that
      // value when the second candidate arrives. So pass A1 queues only raws
      // with two or more candidates, and pass B's rescan of a single-candidate
      // raw (which would leave it in place) is skipped.
      // Pass A1: raws whose best cluster lost reads are queued for a rescan.
      // Every pass here follows a move pass (or the carried state, which ended
      // with one), after which each raw sits in its best cluster unless it is
      // a center; so the raws whose best is ci are ci's members plus centers
      // of other clusters, the same set as ci's comps with best ci. Pass B
      // rescans each queued raw on its own and the dirty list is sorted before
      // use, so the queue order does not matter. Long member lists are split
      // across threads.
      for (uint32_t ci : reads_fell_list) {
        const Cluster& cc = clusters[ci];
        cc.multi.each(0, cc.raws.size(), [&](size_t k) {  // members with ncand > 1
          const uint32_t raw = cc.raws[k];
          if (compmax[raw].i == ci && !in_affected[raw]) {
            in_affected[raw] = 1;
            affected.push_back(raw);
          }
        });
      }
      // the centers of other clusters whose best is a cluster that lost reads
      if (!reads_fell_list.empty())
        for (size_t cj = 0; cj < center_raw.size(); ++cj) {
          const uint32_t raw = center_raw[cj];
          if (raw == UINT32_MAX) continue;
          const uint32_t bi = compmax[raw].i;
          if (bi != cj && reads_fell[bi] && !in_affected[raw]) {
            in_affected[raw] = 1;
            affected.push_back(raw);
          }
        }
      // Pass A2: changed clusters in ascending order. A cluster whose reads
      // fell changes nothing here: every raw whose best it is was queued by A1
      // and is skipped, and for any other raw e = lambda * reads only dropped
      // below an emax that already held it (ties already went to the smaller
      // index), so its scan is left out.
      for (uint32_t ci : touched_list) {
        const uint32_t nr = clusters[ci].reads;
        if (nr == reads_used[ci]) continue;
        if (nr < reads_used[ci]) {
          reads_used[ci] = nr;
          continue;
        }
        const double rf = double(nr);
        par_dirty(clusters[ci].comp.size(), [&](size_t lo, size_t hi, DirtyOut& out) {
          reconcile_a2(uint32_t(ci), rf, lo, hi, out);
        });
        reads_used[ci] = nr;
      }
      for (uint32_t ci : touched_list) touched[ci] = 0;
      touched_list.clear();
      // Pass B: full rescans of the queued raws.
      par_dirty(affected.size(), [&](size_t lo, size_t hi, DirtyOut& out) { reconcile_b(lo, hi, out); });
      affected.clear();
      for (uint32_t ci : reads_fell_list) reads_fell[ci] = 0;
      reads_fell_list.clear();
      after_reconcile = true;
    }
    stats.shuffle_calls += nshuffle;
  }

  // After the compare of cluster ci has been absorbed: the serial tail of one
  // loop iteration, then the next bud. Returns the next cluster to compare or -1.
  int64_t advance(size_t ci) {
    const auto t0 = Clock::now();
    if (ci > 0) shuffle_converge(10);  // MAX_SHUFFLE, src/dada.rs:39
    const auto t1 = Clock::now();
    p_update();
    const auto t2 = Clock::now();
    stats.ns_shuffle += uint64_t(std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count());
    stats.ns_pupdate += uint64_t(std::chrono::duration_cast<std::chrono::nanoseconds>(t2 - t1).count());
    if (clusters.size() >= conf->max_clust) return -1;
    const int64_t next = bud();
    stats.ns_bud += uint64_t(std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now() - t2).count());
    return next;
  }
};

// ---------------------------------------------------------------------------
// Simple persistent worker pool for the per-sample host phases
// ---------------------------------------------------------------------------
class Workers {
 public:
  explicit Workers(int n) {
    for (int t = 0; t < n; ++t) th_.emplace_back([this] { loop(); });
  }
  ~Workers() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  void run(size_t n, const std::function<void(size_t)>& fn) {
    if (th_.empty() || n <= 1) {
      for (size_t t = 0; t < n; ++t) fn(t);
      return;
    }
    {
      std::lock_guard<std::mutex> g(mu_);
      fn_ = &fn;
      n_ = n;
      next_.store(0);
      pending_ = th_.size();
      ++gen_;
    }
    cv_.notify_all();
    for (;;) {  // the caller works too
      size_t t = next_.fetch_add(1);
      if (t >= n) break;
      fn(t);
    }
    std::unique_lock<std::mutex> g(mu_);
    done_.wait(g, [this] { return pending_ == 0; });
  }

 private:
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      std::unique_lock<std::mutex> g(mu_);
      cv_.wait(g, [&] { return stop_ || gen_ != seen; });
      if (stop_) return;
      seen = gen_;
      const std::function<void(size_t)>* fn = fn_;
      const size_t n = n_;
      g.unlock();
      for (;;) {
        size_t t = next_.fetch_add(1);
        if (t >= n) break;
        (*fn)(t);
      }
      g.lock();
      if (--pending_ == 0) done_.notify_all();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  const std::function<void(size_t)>* fn_ = nullptr;
  size_t n_ = 0, pending_ = 0;
  std::atomic<size_t> next_{0};
  uint64_t gen_ = 0;
  bool stop_ = false;
};

// Asynchronous job queue: the host phases of a sample run here while the GPU
// works on other samples' compares.
// Host-phase jobs, highest priority first (first come first among equals).
class JobQueue {
 public:
  explicit JobQueue(int n) {
    for (int t = 0; t < n; ++t) th_.emplace_back([this] { loop(); });
  }
  ~JobQueue() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  bool inline_mode() const { return th_.empty(); }
  void submit(std::function<void()> fn, int64_t priority = 0) {
    if (th_.empty()) {
      fn();
      return;
    }
    {
      std::lock_guard<std::mutex> g(mu_);
      q_.emplace(-priority, std::move(fn));
    }
    cv_.notify_one();
  }

 private:
  void loop() {
    for (;;) {
      std::function<void()> fn;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return stop_ || !q_.empty(); });
        if (q_.empty()) return;
        fn = std::move(q_.begin()->second);
        q_.erase(q_.begin());
      }
      fn();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::multimap<int64_t, std::function<void()>> q_;
  bool stop_ = false;
};

// ---------------------------------------------------------------------------
// Inputs: validation and encoding (src/dada.rs:248-418)
// ---------------------------------------------------------------------------
// A batch of samples encoded for the pool: codes 1..4 and rounded mean
// qualities of every unique back to back (sample after sample, input order),
// with per-unique offsets, lengths, reads and priors. The byte buffers belong
// to the caller (pinned host memory for an upload).
struct EncodedView {
  uint8_t* seq = nullptr;
  uint8_t* qual = nullptr;  // null when the input has no qualities
  std::vector<uint32_t> off, len, reads;
  std::vector<uint8_t> prior;
  std::vector<uint32_t> uqmax;  // per unique: its largest round(sum / max(reads, 1))
  uint32_t qmax = 0;
};

// Structural checks of dada_uniques_cached (src/dada.rs:248-317) for each
// sample, in the order the reference applies them; returns the index of the
// first failing sample (nsamples if none) with its code and message. Also
// returns the total sequence bytes.
static int check_samples(int nsamples, const uint32_t* sample_start, const uint32_t* lens, int k, uint64_t* total,
                         int* rc, std::string* msg) {
  *total = 0;
  for (int s = 0; s < nsamples; ++s) {
    const uint32_t lo = sample_start[s], hi = sample_start[s + 1];
    const std::string tag = "sample " + std::to_string(s) + ": ";
    if (hi == lo) {
      *rc = DGPU_E_INVALID;
      *msg = tag + "Zero input sequences.";
      return s;
    }
    uint32_t maxlen = 0, minlen = 0xffffffffu;
    for (uint32_t t = lo; t < hi; ++t) {
      maxlen = std::max(maxlen, lens[t]);
      minlen = std::min(minlen, lens[t]);
      *total += lens[t];
    }
    if (maxlen >= 9999) {
      *rc = DGPU_E_INVALID;
      *msg = tag + "Input sequences exceed the maximum allowed length (9999).";
      return s;
    }
    if (k < 3 || k > 8) {
      *rc = DGPU_E_INVALID;
      *msg = tag + "kmer_size out of supported range (3..=8).";
      return s;
    }
    if (minlen <= uint32_t(k)) {
      *rc = DGPU_E_INVALID;
      *msg = tag + "All input sequences must be longer than the k-mer size.";
      return s;
    }
  }
  return nsamples;
}

// nt code of an input character: A/C/G/T/U in either case -> 1..4, else 0
static const std::array<uint8_t, 256> kNtCode = [] {
  std::array<uint8_t, 256> t{};
  t['A'] = t['a'] = 1;
  t['C'] = t['c'] = 2;
  t['G'] = t['g'] = 3;
  t['T'] = t['t'] = t['U'] = t['u'] = 4;
  return t;
}();

// Encodes uniques [sample_start[0], sample_start[nsamples]) into E (seq, qual
// sized by the caller), in parallel chunks of uniques. Bases map A/C/G/T/U
// (either case) to 1..4; qualities are round(sum / reads) saturated to u8
// (src/containers.rs:128-137) and qmax the largest round(sum / max(reads, 1))
// (src/dada.rs:337-346). On a non-ACGT base the first one in input order is
// reported, as a sequential scan would: *bad_unique / *bad_pos (else
// bad_unique = UINT32_MAX).
static void encode_uniques(uint32_t t0, uint32_t t1, const char* seqs, const uint32_t* offs, const uint32_t* lens,
                           const uint32_t* abund, const uint8_t* prior, const uint32_t* qsums, EncodedView& E,
                           uint32_t* bad_unique, uint32_t* bad_pos) {
  const uint32_t n = t1 - t0;
  E.off.resize(n);
  E.len.resize(n);
  E.reads.resize(n);
  E.prior.assign(n, 0);
  E.uqmax.assign(n, 0);
  uint64_t w = 0;
  for (uint32_t r = 0; r < n; ++r) {
    E.off[r] = uint32_t(w);
    E.len[r] = lens[t0 + r];
    E.reads[r] = abund[t0 + r];
    E.prior[r] = prior ? prior[t0 + r] : 0;
    w += lens[t0 + r];
  }
  constexpr uint32_t kChunk = 512;
  const uint32_t nch = (n + kChunk - 1) / kChunk;
  std::vector<uint32_t> ch_bad(nch, 0xffffffffu), ch_pos(nch, 0), ch_qmax(nch, 0);
  std::atomic<uint32_t> next{0};
  auto work = [&] {
    for (uint32_t c; (c = next.fetch_add(1)) < nch;) {
      const uint32_t r0 = c * kChunk, r1 = std::min(n, r0 + kChunk);
      uint32_t qm_max = 0;
      for (uint32_t r = r0; r < r1; ++r) {
        const uint32_t t = t0 + r;
        const char* sq = seqs + offs[t];
        uint8_t* out = E.seq + E.off[r];
        bool bad = false;
        for (uint32_t p = 0; p < lens[t]; ++p) {
          const uint8_t code = kNtCode[static_cast<unsigned char>(sq[p])];
          if (!code) {
            ch_bad[c] = r;
            ch_pos[c] = p;
            bad = true;
            break;
          }
          out[p] = code;
        }
        if (bad) break;  // later uniques of this chunk cannot be the first failure
        if (E.qual) {
          // quality = round(sum / reads) half away from zero as u8
          // (src/containers.rs:128-137); uqmax takes the unclamped value with
          // reads floored at 1. For 0 <= x = sum / reads < 2^32, x + 0.5 is
          // exact and its truncation is that rounding; and x is never within
          // 1 / (2 reads) of a half-integer without being one, far above the
          // division's rounding, so this equals rounding the exact quotient.
          const uint32_t reads = abund[t];
          const double cq = double(std::max<uint32_t>(reads, 1));
          const uint32_t* qs = qsums + offs[t];
          uint8_t* qo = E.qual + E.off[r];
          uint32_t qm_u = 0;
          for (uint32_t p = 0; p < lens[t]; ++p) {
            const uint32_t q = uint32_t(double(qs[p]) / cq + 0.5);
            qm_u = std::max(qm_u, q);
            // reads == 0: sum / 0 is +inf (-> 255) for a positive sum, NaN (-> 0) for 0
            qo[p] = reads ? uint8_t(std::min<uint32_t>(q, 255u)) : (qs[p] ? 255 : 0);
          }
          E.uqmax[r] = qm_u;
          qm_max = std::max(qm_max, qm_u);
        }
      }
      ch_qmax[c] = qm_max;
    }
  };
  const uint32_t nt = std::max(1u, std::min(nch, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  for (uint32_t t = 1; t < nt; ++t) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
  *bad_unique = 0xffffffffu;
  *bad_pos = 0;
  E.qmax = 0;
  for (uint32_t c = 0; c < nch; ++c) {
    if (ch_bad[c] != 0xffffffffu) {
      *bad_unique = ch_bad[c];
      *bad_pos = ch_pos[c];
      return;
    }
    E.qmax = std::max(E.qmax, ch_qmax[c]);
  }
}

// Repeat the last learned column up to qmax (src/dada.rs:337-384).
static std::vector<double> extend_err(const double* errm, int ncol, uint32_t qmax, int& new_ncol) {
  new_ncol = ncol;
  if (int64_t(qmax) < ncol) return std::vector<double>(errm, errm + 16 * size_t(ncol));
  new_ncol = int(qmax) + 1;
  std::vector<double> ext(16 * size_t(new_ncol));
  for (int t = 0; t < 16; ++t) {
    for (int q = 0; q < ncol; ++q) ext[size_t(t) * new_ncol + q] = errm[size_t(t) * ncol + q];
    for (int q = ncol; q < new_ncol; ++q) ext[size_t(t) * new_ncol + q] = errm[size_t(t) * ncol + ncol - 1];
  }
  return ext;
}

static KParams to_kparams(const dgpu_align_params& a, int use_quals, int greedy, int ncol) {
  KParams k{};
  k.match = a.match_score;
  k.mismatch = a.mismatch;
  k.gap = a.gap_p;
  k.homo_gap = a.homo_gap_p;
  k.use_kmers = a.use_kmers ? 1 : 0;
  k.kmer_size = a.kmer_size;
  k.band = a.band;
  k.vectorized = a.vectorized ? 1 : 0;
  k.gapless = a.gapless ? 1 : 0;
  k.use_quals = use_quals ? 1 : 0;
  k.greedy = greedy ? 1 : 0;
  k.ncol = ncol;
  return k;
}

}  // namespace dgpu

// ---------------------------------------------------------------------------
// Results
// ---------------------------------------------------------------------------
struct dgpu_result {
  uint32_t nraw = 0;
  std::vector<uint32_t> cl_reads, cl_birth_from, cl_birth_hamming, cl_seq_off, cl_mem_off, mem_raw, mem_hamming;
  std::vector<int32_t> cl_birth_type, map;
  std::vector<double> cl_birth_pval, cl_birth_fold, cl_birth_e, mem_lambda, mem_pval, pvals;
  std::vector<uint8_t> cl_seq;
  uint64_t counters[16] = {0};
  double times[6] = {0};
  uint64_t fp32[2] = {0, 0};          // FP32-lambda p-values, FP64 fallbacks among them
  double margin[3] = {0, 0, 0};       // decision margins against omega_a, omega_p, omega_c
  std::vector<uint32_t> transitions;  // 16 x tncol when requested
  int tncol = 0;
};

namespace dgpu {

// The codes of one sample's uniques: raw r at seq + off[r], len[r] bytes.
struct SampleSeqs {
  const uint8_t* seq;
  const uint32_t* off;
  const uint32_t* len;
};

// Final p-values, the map and the cluster summaries (src/dada.rs:502-564).
static dgpu_result* finish(SampleState& S, const SampleSeqs& in) {
  dgpu_result* R = new dgpu_result();
  const uint32_t n = S.n;
  R->nraw = n;
  R->pvals.assign(n, 0.0);
  R->map.assign(n, -1);
  std::vector<uint8_t> correct(n, 0);
  // every raw once, with its cluster; priced independently (in parallel
  // chunks for a large sample)
  std::vector<uint32_t> mem_ci(n, 0), order;
  order.reserve(n);
  for (size_t ci = 0; ci < S.clusters.size(); ++ci)
    for (uint32_t raw : S.clusters[ci].raws) {
      mem_ci[raw] = uint32_t(ci);
      order.push_back(raw);
    }
  std::mutex margin_mu;
  double margin_c = std::numeric_limits<double>::infinity();
  auto price = [&](size_t lo, size_t hi) {
    double mc = std::numeric_limits<double>::infinity();
    for (size_t k = lo; k < hi; ++k) {
      const uint32_t raw = order[k];
      const Cluster& c = S.clusters[mem_ci[raw]];
      double pv;
      bool ok;
      if (int64_t(raw) == c.center) {
        pv = 1.0;
        ok = true;
      } else {
        pv = SampleState::calc_pA(S.reads[raw], S.rcomp[raw].lambda * double(c.reads), true);
        if (S.conf->fp32) {  // the map decision near omega_c from the FP64 product
          S.fp32_evals.fetch_add(1, std::memory_order_relaxed);
          if (SampleState::near_threshold(pv, S.conf->omega_c)) {
            pv = SampleState::calc_pA(S.reads[raw], S.lambda64_of(raw) * double(c.reads), true);
            S.fp32_fallbacks.fetch_add(1, std::memory_order_relaxed);
          }
        }
        ok = pv >= S.conf->omega_c;
        mc = std::min(mc, SampleState::rel_margin(pv, S.conf->omega_c));
      }
      S.p[raw] = pv;
      correct[raw] = ok;
      R->pvals[raw] = pv;
    }
    std::lock_guard<std::mutex> lk(margin_mu);
    margin_c = std::min(margin_c, mc);
  };
  if (order.size() < kParMin)
    price(0, order.size());
  else
    Helpers::get().parallel_for(order.size(), kParGrain, [&](size_t, size_t lo, size_t hi) { price(lo, hi); });
  for (size_t ci = 0; ci < S.clusters.size(); ++ci)
    for (uint32_t raw : S.clusters[ci].raws)
      if (correct[raw]) R->map[raw] = int32_t(ci);
  uint32_t so = 0, mo = 0;
  for (const Cluster& c : S.clusters) {
    R->cl_reads.push_back(c.reads);
    R->cl_birth_type.push_back(c.birth_type);
    R->cl_birth_from.push_back(c.birth_from);
    R->cl_birth_pval.push_back(c.birth_pval);
    R->cl_birth_fold.push_back(c.birth_fold);
    R->cl_birth_e.push_back(c.birth_e);
    R->cl_birth_hamming.push_back(c.birth_comp.hamming);
    R->cl_seq_off.push_back(so);
    if (c.center >= 0) {
      const uint32_t ce = uint32_t(c.center);
      R->cl_seq.insert(R->cl_seq.end(), in.seq + in.off[ce], in.seq + in.off[ce] + in.len[ce]);
      so += in.len[ce];
    }
    R->cl_mem_off.push_back(mo);
    for (uint32_t raw : c.raws) {
      R->mem_raw.push_back(raw);
      R->mem_hamming.push_back(S.rcomp[raw].hamming);
      R->mem_lambda.push_back(S.rcomp[raw].lambda);
      R->mem_pval.push_back(S.p[raw]);
    }
    mo += uint32_t(c.raws.size());
  }
  R->cl_seq_off.push_back(so);
  R->cl_mem_off.push_back(mo);
  const RunStats& st = S.stats;
  const uint64_t c[16] = {S.nalign, st.compare_calls, st.cmp_scanned, st.screened, st.aligned, st.stored,
                          st.gapless, st.vectorized, st.homo, st.endsfree, st.shuffle_calls, st.shuffle_moves,
                          S.nshroud, st.ns_shuffle, st.ns_pupdate, st.ns_bud};
  std::copy(c, c + 16, R->counters);
  R->times[0] = st.t_compare;
  R->times[1] = st.t_total;
  R->times[2] = st.t_host;
  R->times[3] = st.t_wait;
  R->times[4] = st.t_slot_wait;
  R->times[5] = st.t_job_wait;
  R->fp32[0] = S.fp32_evals.load();
  R->fp32[1] = S.fp32_fallbacks.load();
  R->margin[0] = S.margin[0];
  R->margin[1] = S.margin[1];
  R->margin[2] = margin_c;
  return R;
}

// The clustering loop over any number of samples resident in one pool.
// Samples advance independently. Each launch slot has a worker that takes
// every sample whose next cluster is ready, runs one compare launch over them
// and hands each sample's host phases (shuffle, p-update, bud) to the job
// queue; with several slots a sample that becomes ready while a launch is in
// flight goes out at once on another slot. A sample's own sequence of steps is
// exactly run_dada's.
static size_t batch_max_samples(uint32_t lmax);

// on_finish (may be empty) is called for each sample as soon as its loop ends,
// from the host thread that ran its last phase.
static int run_samples(Pool& P, std::vector<SampleState>& S, const dgpu_align_params& ap, int host_threads,
                       const std::function<void(size_t)>& on_finish = {}) {
  const size_t ns = S.size();
  const size_t batch_max = batch_max_samples(P.lmax);
  std::mutex mu;
  std::condition_variable cv;
  std::vector<size_t> ready;
  size_t finished = 0;
  for (size_t s = 0; s < ns; ++s) {
    S[s].pending = 0;  // cluster 0 first, with the screen off
    S[s].stats.t_mark = Clock::now();
    ready.push_back(s);
  }
  int rc = 0;
  std::string err_msg;
  std::atomic<int64_t> host_ns{0};
  // With several slots, the kd unfinished samples with the most uniques (the
  // longest chains) have a slot each, with a high-priority stream, to
  // themselves: they never wait for a slot and their kernels are scheduled
  // ahead of the others'. The other slots serve the rest, largest first.
  const size_t nw_all = std::min(P.slots.size(), ns);
  const size_t kd = nw_all > 1 ? std::min(dedicated_slots(P.lmax), nw_all - 1) : 0;
  std::vector<uint8_t> is_done(ns, 0), is_crit(ns, 0);
  std::vector<size_t> crit(kd, SIZE_MAX);  // crit[i]: the sample slot i serves
  auto pick_critical = [&] {  // under mu: the kd largest unfinished samples
    for (size_t& c : crit) c = SIZE_MAX;
    std::fill(is_crit.begin(), is_crit.end(), 0);
    for (size_t i = 0; i < kd; ++i) {
      size_t best = SIZE_MAX;
      for (size_t s = 0; s < ns; ++s)
        if (!is_done[s] && !is_crit[s] && (best == SIZE_MAX || S[s].n > S[best].n)) best = s;
      if (best == SIZE_MAX) break;
      crit[i] = best;
      is_crit[best] = 1;
    }
  };
  pick_critical();
  auto t_start = Clock::now();
  {
    JobQueue jobs(host_threads > 1 ? host_threads : 0);
    auto worker = [&](Slot& L) {
      size_t my = SIZE_MAX;  // the dedicated position of this slot, if any
      for (size_t i = 0; i < kd; ++i)
        if (&L == P.slots[i].get()) my = i;
      const bool mine = my != SIZE_MAX;
      auto has_work = [&] {  // under mu
        if (mine) return crit[my] != SIZE_MAX && std::find(ready.begin(), ready.end(), crit[my]) != ready.end();
        for (size_t s : ready)
          if (!is_crit[s]) return true;
        return false;
      };
      if (cudaSetDevice(P.device) != cudaSuccess) {
        std::lock_guard<std::mutex> g(mu);
        if (!rc) {
          rc = DGPU_E_CUDA;
          err_msg = "cudaSetDevice failed in a launch worker";
        }
        cv.notify_all();
        return;
      }
      std::vector<size_t> batch;
      double my_wait = 0.0;
      for (;;) {
        batch.clear();
        {
          std::unique_lock<std::mutex> lk(mu);
          cv.wait(lk, [&] { return has_work() || finished == ns || rc != 0; });
          if (rc != 0 || !has_work()) break;
          if (mine) {
            ready.erase(std::find(ready.begin(), ready.end(), crit[my]));
            batch.push_back(crit[my]);
          } else {
            std::vector<size_t> held;
            for (size_t k = 0; k < ready.size();) {
              if (is_crit[ready[k]]) {
                held.push_back(ready[k]);
                ready.erase(ready.begin() + long(k));
              } else {
                ++k;
              }
            }
            if (ready.size() <= batch_max) {
              batch.swap(ready);
            } else {
              // the largest samples (the longest chains) go first
              std::stable_sort(ready.begin(), ready.end(), [&](size_t x, size_t y) { return S[x].n > S[y].n; });
              batch.assign(ready.begin(), ready.begin() + batch_max);
              ready.erase(ready.begin(), ready.begin() + batch_max);
              if (!ready.empty()) cv.notify_all();
            }
            ready.insert(ready.end(), held.begin(), held.end());
          }
        }
        std::sort(batch.begin(), batch.end());
        {
          const auto now = Clock::now();
          for (size_t sidx : batch) S[sidx].stats.t_slot_wait += secs(S[sidx].stats.t_mark, now);
        }
        int r = L.ensure_tasks(uint32_t(batch.size()));
        for (size_t a = 0; a < batch.size() && !r; ++a) {
          SampleState& ss = S[batch[a]];
          const size_t ci = size_t(ss.pending);
          L.task_stage.h[a] = ss.task_for(ci, ci == 0 ? 1.0 : ap.kdist_cutoff);  // init_params, src/dada.rs:835-838
          if (ss.lock_dirty) {
            r = P.push_locks(ss.base, ss.n, L.st);
            ss.lock_dirty = false;
          }
        }
        const auto tc = Clock::now();
        const double w0 = my_wait;
        if (!r) r = L.run_compare(uint32_t(batch.size()), true, &my_wait);
        if (r) {
          std::lock_guard<std::mutex> g(mu);
          if (!rc) {
            rc = r;
            err_msg = g_err;
          }
          cv.notify_all();
          break;
        }
        const double tcmp = secs(tc, Clock::now());
        // each sample's host phase is queued as soon as its own results are
        // absorbed, the largest samples (the longest chains) first
        std::vector<uint32_t> order(batch.size());
        for (size_t a = 0; a < batch.size(); ++a) order[a] = uint32_t(a);
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return S[batch[x]].n > S[batch[y]].n; });
        for (uint32_t a : order) {
          const size_t sidx = batch[a];
          SampleState& sa = S[sidx];
          sa.absorb(size_t(sa.pending), L, a);
          sa.stats.t_compare += tcmp;
          sa.stats.t_wait += my_wait - w0;  // the device wait of the calls that carried this sample
          sa.stats.t_mark = Clock::now();
          auto host_phase = [&, sidx] {
            SampleState& ss = S[sidx];
            auto th = Clock::now();
            ss.stats.t_job_wait += secs(ss.stats.t_mark, th);
            ss.pending = ss.advance(size_t(ss.pending));
            const double dh = secs(th, Clock::now());
            ss.stats.t_host += dh;
            host_ns += int64_t(1e9 * dh);
            if (ss.pending < 0 && on_finish) {
              ss.stats.t_done = secs(t_start, Clock::now());
              ss.stats.t_total = ss.stats.t_done;
              on_finish(sidx);
            }
            std::lock_guard<std::mutex> g(mu);
            if (ss.pending >= 0) {
              ss.stats.t_mark = Clock::now();
              ready.push_back(sidx);
            } else {
              ++finished;
              if (!on_finish) ss.stats.t_done = secs(t_start, Clock::now());
              is_done[sidx] = 1;
              if (is_crit[sidx]) pick_critical();
            }
            cv.notify_all();
          };
          // the dedicated slot runs its sample's host phase itself and goes
          // straight on to the next compare: no hand-off between threads
          if (mine)
            host_phase();
          else
            jobs.submit(host_phase, int64_t(S[sidx].n));  // larger samples have the longer chains: serve them first
        }
      }
    };
    const size_t nw = std::min(P.slots.size(), ns);
    std::vector<std::thread> th;
    for (size_t k = 1; k < nw; ++k) th.emplace_back(worker, std::ref(*P.slots[k]));
    worker(*P.slots[0]);
    for (auto& t : th) t.join();
  }  // the job queue drains its queued host phases here
  const double total = secs(t_start, Clock::now());
  for (auto& ss : S) {
    ss.stats.t_total = ss.stats.t_done >= 0 ? ss.stats.t_done : total;
  }
  if (rc) return fail(rc, err_msg);
  return 0;
}

// Most samples one compare launch covers: DGPU_BATCH_MAX (1..4096) if set,
// else the tuning table's (4 built in). Small launches finish sooner, and the
// largest ready samples (the longest chains of dependent rounds) are served
// first.
static size_t batch_max_samples(uint32_t lmax) {
  if (const char* e = std::getenv("DGPU_BATCH_MAX")) {
    const long v = std::atol(e);
    if (v >= 1 && v <= 4096) return size_t(v);
  }
  return size_t(tuning_for(lmax).samples_per_launch);
}

// Launch slots for a batch of nsamples: DGPU_LAUNCH_SLOTS (1..8) if set, else
// the tuning table's (6 built in: on B200 the 40-sample batch stepped in
// 84-86 ms with 6, 87-88 with 4 and 96-101 with 3); never more than there are
// samples.
static int launch_slots(int nsamples, uint32_t lmax) {
  int k = tuning_for(lmax).launch_slots;
  if (const char* e = std::getenv("DGPU_LAUNCH_SLOTS")) {
    const int v = std::atoi(e);
    if (v >= 1 && v <= 8) k = v;
  }
  return std::max(1, std::min(k, nsamples));
}

// A prepared batch: encoded samples resident on one device.
struct Batch {
  Pool pool;
  HBuf<uint8_t> seq_h, qual_h;  // pinned encoded codes / qualities of every unique
  EncodedView E;
  std::vector<uint32_t> bases, counts;  // first raw and number of raws of each sample
  DadaConf conf{};
  std::vector<DadaConf> confs;
  dgpu_align_params align{};
  int host_threads = 1;
  bool transitions = false;  // run the final-subs pass after the loop
  int learn_nq = 0;          // > 0: that pass counts build_trans_mat's matrix (learn-errors)
  int ncol_in = 0;           // the caller's error-matrix width (before extension)
  ~Batch() {  // Pool::upload waited for its copies, so the staging blocks are idle
    seq_h.recycle();
    qual_h.recycle();
  }
};

static int batch_prepare(Batch& B, int device, const dgpu_dada_params* prm, int nsamples, const uint32_t* sample_start,
                         const char* seqs, const uint32_t* offs, const uint32_t* lens, const uint32_t* abund,
                         const uint8_t* prior, const uint32_t* qsums, const double* errm, int ncol) {
  const auto tp0 = Clock::now();
  if (!prm || !seqs || !offs || !lens || !abund || !errm || nsamples <= 0 || !sample_start)
    return fail(DGPU_E_INVALID, "null argument or no samples");
  if (ncol <= 0) return fail(DGPU_E_INVALID, "Error matrix length does not match 16 x ncol.");
  const int k = prm->align.kmer_size;
  for (int s = 0; s < nsamples; ++s)
    if (sample_start[s + 1] < sample_start[s]) return fail(DGPU_E_INVALID, "sample_start must be non-decreasing");
  // The reference validates sample after sample: the first sample that fails
  // a structural check or holds a non-ACGT base reports.
  uint64_t total = 0;
  int src = 0;
  std::string smsg;
  const int first_bad = check_samples(nsamples, sample_start, lens, k, &total, &src, &smsg);
  if (total >= 0xffffffffull) return fail(DGPU_E_UNSUPPORTED, "more than 4 GiB of sequence in one pool");
  uint32_t lmax_all = 0;
  for (uint32_t t = sample_start[0]; t < sample_start[nsamples]; ++t) lmax_all = std::max(lmax_all, lens[t]);
  TRY(B.pool.init(device, launch_slots(nsamples, lmax_all)));
  const int ns_ok = first_bad;  // samples [0, ns_ok) passed the structural checks
  uint64_t ok_bytes = 0;
  for (uint32_t t = sample_start[0]; t < sample_start[ns_ok]; ++t) ok_bytes += lens[t];
  TRY(B.seq_h.alloc(size_t(ok_bytes ? ok_bytes : 1)));
  if (qsums) TRY(B.qual_h.alloc(size_t(ok_bytes ? ok_bytes : 1)));
  B.E.seq = B.seq_h.h;
  B.E.qual = qsums ? B.qual_h.h : nullptr;
  uint32_t bad_t = 0, bad_p = 0;
  encode_uniques(sample_start[0], sample_start[ns_ok], seqs, offs, lens, abund, prior, qsums, B.E, &bad_t, &bad_p);
  if (bad_t != 0xffffffffu) {
    const uint32_t t = sample_start[0] + bad_t;
    int s = 0;
    while (sample_start[s + 1] <= t) ++s;
    return fail(DGPU_E_INVALID, "sample " + std::to_string(s) + ": Sequence " + std::to_string(t - sample_start[s]) +
                                    " contains a non-ACGT base at position " + std::to_string(bad_p) + ".");
  }
  if (first_bad < nsamples) return fail(src, smsg);
  B.bases.resize(size_t(nsamples));
  B.counts.resize(size_t(nsamples));
  for (int s = 0; s < nsamples; ++s) {
    B.bases[size_t(s)] = sample_start[s] - sample_start[0];
    B.counts[size_t(s)] = sample_start[s + 1] - sample_start[s];
  }
  int ncol2 = ncol;
  std::vector<double> err = qsums ? extend_err(errm, ncol, B.E.qmax, ncol2)
                                  : std::vector<double>(errm, errm + 16 * size_t(ncol));
  KParams kp = to_kparams(prm->align, prm->use_quals, prm->greedy, ncol2);
  kp.lambda32 = prm->lambda_fp32 ? 1 : 0;
  const auto tp1 = Clock::now();
  {  // uniques are compared only within their sample
    int64_t spread = 0;
    for (int s = 0; s < nsamples; ++s) {
      uint32_t lo = 0xffffffffu, hi = 0;
      for (uint32_t t = B.bases[size_t(s)]; t < B.bases[size_t(s)] + B.counts[size_t(s)]; ++t) {
        lo = std::min(lo, B.E.len[t]);
        hi = std::max(hi, B.E.len[t]);
      }
      if (hi >= lo) spread = std::max<int64_t>(spread, int64_t(hi) - int64_t(lo));
    }
    B.pool.pair_spread = spread;
  }
  TRY(B.pool.upload(uint32_t(B.E.off.size()), B.E.seq, B.E.off.data(), B.E.len.data(), B.E.qual, B.E.reads.data(), kp,
                    err.data()));
  {
    std::lock_guard<std::mutex> g(g_stats.mu);
    g_stats.s.prepare_ms[0] += 1e3 * secs(tp0, tp1);
    g_stats.s.prepare_ms[1] += 1e3 * secs(tp1, Clock::now());
  }
  B.conf.omega_a = prm->omega_a;
  B.conf.omega_p = prm->omega_p;
  B.conf.omega_c = prm->omega_c;
  B.conf.min_fold = prm->min_fold;
  B.conf.kdist_cutoff = prm->align.kdist_cutoff;
  B.conf.detect_singletons = prm->detect_singletons != 0;
  B.conf.greedy = prm->greedy != 0;
  B.conf.fp32 = prm->lambda_fp32 != 0;
  B.conf.min_hamming = prm->min_hamming;
  B.conf.min_abund = prm->min_abund;
  B.confs.assign(static_cast<size_t>(nsamples), B.conf);
  for (int s = 0; s < nsamples; ++s)
    B.confs[size_t(s)].max_clust = prm->max_clust == 0 ? B.counts[size_t(s)] : size_t(prm->max_clust);
  B.align = prm->align;
  B.transitions = prm->transitions != 0;
  B.ncol_in = ncol;
  // Host phases of different samples share the cores with the intra-sample
  // helpers (half the cores) and the launch workers, so by default they get
  // the other half.
  int threads = prm->host_threads;
  if (threads <= 0) threads = int(std::max(1u, std::thread::hardware_concurrency() / 2));
  B.host_threads = std::min(threads, nsamples);
  return 0;
}

// The final-subs pass and transition counts of every sample (DadaAux.transitions,
// src/dada.rs:609-673, src/error.rs:194-249): each correct member (map != -1,
// centers included) realigned against its cluster's center with the k-mer
// screen off, on the device; counts land in each sample's result with the
// sample's own error-matrix width (extended to its qmax + 1 when that is
// larger), or one column without qualities.
static int final_subs(Batch& B, std::vector<SampleState>& S, dgpu_result** out) {
  Pool& P = B.pool;
  const size_t ns = B.counts.size();
  std::vector<uint32_t> raw, center, sample;
  for (size_t s = 0; s < ns; ++s) {
    const dgpu_result* R = out[s];
    for (const Cluster& c : S[s].clusters) {
      if (c.center < 0) continue;
      for (uint32_t r : c.raws) {
        if (R->map[r] < 0) continue;
        raw.push_back(B.bases[s] + r);
        center.push_back(B.bases[s] + uint32_t(c.center));
        sample.push_back(uint32_t(s));
      }
    }
  }
  const bool has_q = B.E.qual != nullptr;
  // learn-errors (build_trans_mat, src/learn_errors.rs:618-738) counts every
  // sample at one width nq = the largest rounded quality + 1, so no quality
  // is clamped, and saturates each sample's counts at u32; without qualities
  // it counts nothing
  const bool learn = B.learn_nq > 0;
  if (learn && !has_q) raw.clear();
  const int tncol = learn ? B.learn_nq : (has_q ? P.kp.ncol : 1);
  const size_t nbins = size_t(16) * size_t(tncol);
  const uint32_t nitems = uint32_t(raw.size());
  DBuf<uint32_t> items, counts, err;
  DBuf<unsigned long long> counts64;
  TRY(items.alloc(size_t(3) * std::max<uint32_t>(nitems, 1)));
  TRY(counts.alloc(learn ? 1 : ns * nbins));
  if (learn) TRY(counts64.alloc(ns * nbins));
  TRY(err.alloc(1));
  CUDA_TRY(cudaMemcpyAsync(items.p, raw.data(), size_t(4) * nitems, cudaMemcpyHostToDevice, P.st));
  CUDA_TRY(cudaMemcpyAsync(items.p + nitems, center.data(), size_t(4) * nitems, cudaMemcpyHostToDevice, P.st));
  CUDA_TRY(cudaMemcpyAsync(items.p + 2 * size_t(nitems), sample.data(), size_t(4) * nitems, cudaMemcpyHostToDevice,
                           P.st));
  count_h2d(uint64_t(12) * nitems);
  if (learn) CUDA_TRY(cudaMemsetAsync(counts64.p, 0, ns * nbins * 8, P.st));
  else CUDA_TRY(cudaMemsetAsync(counts.p, 0, ns * nbins * 4, P.st));
  CUDA_TRY(cudaMemsetAsync(err.p, 0, 4, P.st));
  FinalSubsLaunch F{};
  F.pool = P.view();
  F.kp = P.kp;
  F.kp.use_kmers = 0;  // src/dada.rs:611-615: no k-mer screen, cutoff 1.0
  F.geom = P.geom;
  F.nw_scratch = P.slot0().scratch.p;
  F.raw = items.p;
  F.center = items.p + nitems;
  F.sample = items.p + 2 * size_t(nitems);
  F.nitems = nitems;
  F.tncol = tncol;
  F.has_quals = has_q ? 1 : 0;
  F.out = counts.p;
  F.out64 = learn ? counts64.p : nullptr;
  F.err_word = err.p;
  launch_final_subs(F, P.st);
  CUDA_TRY(cudaGetLastError());
  std::vector<uint32_t> host(ns * nbins);
  std::vector<unsigned long long> host64(learn ? ns * nbins : 0);
  uint32_t ew = 0;
  if (learn)
    CUDA_TRY(cudaMemcpyAsync(host64.data(), counts64.p, host64.size() * 8, cudaMemcpyDeviceToHost, P.st));
  else
    CUDA_TRY(cudaMemcpyAsync(host.data(), counts.p, host.size() * 4, cudaMemcpyDeviceToHost, P.st));
  CUDA_TRY(cudaMemcpyAsync(&ew, err.p, 4, cudaMemcpyDeviceToHost, P.st));
  CUDA_TRY(cudaStreamSynchronize(P.st));
  recycle_all(items, counts, counts64, err);
  if (ew) return fail(ew & DERR_UNSUPPORTED ? DGPU_E_UNSUPPORTED : DGPU_E_DEVICE, "device error in the final-subs pass");
  if (learn) {
    for (size_t s = 0; s < ns; ++s) {
      dgpu_result* R = out[s];
      R->tncol = tncol;
      R->transitions.resize(nbins);
      for (size_t b = 0; b < nbins; ++b)
        R->transitions[b] = uint32_t(std::min<unsigned long long>(host64[s * nbins + b], 0xffffffffull));
    }
    return 0;
  }
  for (size_t s = 0; s < ns; ++s) {
    int nc = 1;
    if (has_q) {
      uint32_t qm = 0;
      for (uint32_t r = 0; r < B.counts[s]; ++r) qm = std::max(qm, B.E.uqmax[B.bases[s] + r]);
      nc = int64_t(qm) >= B.ncol_in ? int(qm) + 1 : B.ncol_in;  // src/dada.rs:337-384, per sample
    }
    dgpu_result* R = out[s];
    R->tncol = nc;
    R->transitions.assign(size_t(16) * nc, 0u);
    for (int t = 0; t < 16; ++t)
      for (int q = 0; q < nc && q < tncol; ++q)
        R->transitions[size_t(t) * nc + q] = host[s * nbins + size_t(t) * tncol + q];
  }
  return 0;
}

// on_done (may be empty) receives each sample's result as soon as that sample
// is finished, while others still run; the result then belongs to on_done's
// owner and out[s] stays null. With transition counts requested every result
// goes out at the end, after the final-subs pass.
// fn(s) for every sample s < ns, on up to one thread per core.
template <class F>
static void for_samples(size_t ns, F&& fn) {
  std::atomic<size_t> next{0};
  auto work = [&] {
    for (size_t s; (s = next.fetch_add(1)) < ns;) fn(s);
  };
  const size_t nt = std::min<size_t>(ns, std::max(1u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  for (size_t t = 1; t < nt; ++t) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
}

static int batch_run(Batch& B, dgpu_result** out, const std::function<void(size_t, dgpu_result*)>& on_done = {}) {
  const size_t ns = B.counts.size();
  Pool& P = B.pool;
  const auto tb0 = Clock::now();
  CUDA_TRY(cudaSetDevice(P.device));
  P.pivot_on = true;  // cluster indices are the loop's own: the screen may keep pivots
  TRY(P.reset_e_minmax());
  std::memset(P.lock_host.h, 0, P.nraw);
  CUDA_TRY(cudaMemsetAsync(P.lock.p, 0, P.nraw, P.st));
  CUDA_TRY(cudaStreamSynchronize(P.st));  // the launch slots run on their own streams
  std::vector<SampleState> S(ns);
  for_samples(ns, [&](size_t s) {
    S[s].init(B.counts[s], B.bases[s], B.E.reads.data() + B.bases[s], B.E.prior.data() + B.bases[s],
              P.lock_host.h + B.bases[s], &B.confs[s]);
  });
  const bool early = on_done && !B.transitions;
  std::vector<uint8_t> released(ns, 0);
  std::function<void(size_t)> on_finish;
  if (early)
    on_finish = [&](size_t s) {
      dgpu_result* R = finish(S[s], SampleSeqs{B.E.seq, B.E.off.data() + B.bases[s], B.E.len.data() + B.bases[s]});
      released[s] = 1;
      on_done(s, R);
    };
  const auto tb1 = Clock::now();
  TRY(run_samples(P, S, B.align, B.host_threads, on_finish));
  const auto tb2 = Clock::now();
  // final p-values and result tables, samples in parallel
  for_samples(ns, [&](size_t s) {
    if (!released[s])
      out[s] = finish(S[s], SampleSeqs{B.E.seq, B.E.off.data() + B.bases[s], B.E.len.data() + B.bases[s]});
  });
  const int rc = B.transitions ? final_subs(B, S, out) : 0;
  for_samples(ns, [&](size_t s) { S[s].release(); });
  {
    std::lock_guard<std::mutex> g(g_stats.mu);
    g_stats.s.batch_ms[0] += 1e3 * secs(tb0, tb1);
    g_stats.s.batch_ms[1] += 1e3 * secs(tb1, tb2);
    g_stats.s.batch_ms[2] += 1e3 * secs(tb2, Clock::now());
  }
  if (rc) return rc;
  if (on_done && !early)
    for (size_t s = 0; s < ns; ++s) {
      on_done(s, out[s]);
      out[s] = nullptr;
    }
  return 0;
}

// dgpu_dada_batch with each sample's result handed to on_done as soon as it
// is ready (the denoising service's entry). Samples whose result was not
// handed over when this fails have none.
int dada_batch_each(int device, const dgpu_dada_params* params, int nsamples, const uint32_t* sample_start,
                    const char* seqs, const uint32_t* offs, const uint32_t* lens, const uint32_t* abund,
                    const uint8_t* prior, const uint32_t* qual_sums, const double* err_mat, int ncol,
                    const std::function<void(size_t, dgpu_result*)>& on_done) {
  Batch b;
  TRY(batch_prepare(b, device, params, nsamples, sample_start, seqs, offs, lens, abund, prior, qual_sums, err_mat,
                    ncol));
  std::vector<dgpu_result*> out(size_t(nsamples), nullptr);
  const int rc = batch_run(b, out.data(), on_done);
  for (dgpu_result* r : out) delete r;
  return rc;
}

// ---------------------------------------------------------------------------
// One sample sharded over ranks (one process or thread per GPU)
// ---------------------------------------------------------------------------
// Every rank holds the whole sample and runs the same clustering loop; a
// compare call screens and aligns only the rank's contiguous share of the
// uniques, and the stored comps of all shares are gathered in rank order,
// which is the ascending raw order of a single-device store
// (src/cluster.rs:351-397). The host phases are deterministic, so every rank
// takes the same next center and the same number of exchanges.

// One rank's outcome of one compare call (or of the setup, with err alone).
struct ShardHead {
  int32_t err;        // 0, or the rank's DGPU_E_* code
  uint32_t ns;        // comps stored from the rank's share
  uint32_t has_self;  // the center lies in the rank's share
  uint32_t pad;
  double self;        // the center's own lambda, with has_self
  uint32_t ctr[TC_NCOUNTERS];
};
struct ShardComp {
  uint32_t index, hamming;
  double lambda;
  float ll32;
  uint32_t pad;
};
static_assert(sizeof(ShardHead) == 56 && sizeof(ShardComp) == 24, "exchange records have a fixed layout");

// All-gather of fixed-size blocks: send `bytes` bytes, receive world * bytes
// with rank r's block at r * bytes; nonzero when the exchange failed.
using ShardGather = std::function<int(const void* send, uint64_t bytes, void* recv)>;

// Shares of the uniques [0, n), contiguous and balanced by bases (the work of
// a compare grows with the raw's length); world + 1 bounds.
static std::vector<uint32_t> shard_bounds(const uint32_t* lens, uint32_t n, int world) {
  uint64_t tot = 0;
  for (uint32_t t = 0; t < n; ++t) tot += lens[t];
  std::vector<uint32_t> b(size_t(world) + 1, n);
  b[0] = 0;
  int r = 1;
  uint64_t acc = 0;
  for (uint32_t t = 0; t < n && r < world; ++t) {
    acc += lens[t];
    while (r < world && acc * uint64_t(world) >= tot * uint64_t(r)) b[size_t(r++)] = t + 1;
  }
  return b;
}

// The heads of every rank; fails on every rank alike when any rank failed.
static int shard_heads(const ShardHead& mine, int world, const ShardGather& gather, std::vector<ShardHead>& heads) {
  heads.assign(size_t(world), ShardHead{});
  if (gather(&mine, sizeof(ShardHead), heads.data())) return fail(DGPU_E_INVALID, "shard exchange failed");
  if (mine.err) return mine.err;  // this rank's own message stands
  for (int r = 0; r < world; ++r)
    if (heads[size_t(r)].err)
      return fail(heads[size_t(r)].err, "rank " + std::to_string(r) + " of the sharded run failed");
  return 0;
}

// One compare call's exchange: gathers every rank's head and comps and folds
// them into S in rank order. Every rank calls it once per compare call, its
// own call failed or not, so that the ranks stay in step.
static int shard_exchange(SampleState& S, size_t ci, const ShardHead& mine, const std::vector<ShardComp>& local,
                          int world, const ShardGather& gather) {
  std::vector<ShardHead> heads;
  ShardHead head = mine;
  if (!head.err && local.size() != head.ns)  // reported in the head, so every rank stops here
    head.err = fail(DGPU_E_INVALID, "shard comps do not match the head");
  TRY(shard_heads(head, world, gather, heads));
  uint32_t maxns = 0;
  for (const ShardHead& h : heads) maxns = std::max(maxns, h.ns);
  std::vector<ShardComp> all(size_t(world) * maxns);
  if (maxns) {
    std::vector<ShardComp> send(maxns, ShardComp{});
    std::copy(local.begin(), local.end(), send.begin());
    if (gather(send.data(), uint64_t(maxns) * sizeof(ShardComp), all.data()))
      return fail(DGPU_E_INVALID, "shard exchange failed");
  }
  uint32_t ctr[TC_NCOUNTERS] = {};
  double self = 0.0;
  for (const ShardHead& h : heads) {
    for (int k = 0; k < TC_NCOUNTERS; ++k) ctr[k] += h.ctr[k];
    if (h.has_self) self = h.self;
  }
  S.absorb_from(ci, ctr, self, [&](auto&& f) {
    for (int r = 0; r < world; ++r)
      for (uint32_t k = 0; k < heads[size_t(r)].ns; ++k) {
        const ShardComp& c = all[size_t(r) * maxns + k];
        f(c.index, c.lambda, c.hamming, c.ll32);
      }
  });
  return 0;
}

// This rank's compare of cluster ci's center against the uniques [lo, hi).
static int shard_compare(Pool& P, SampleState& S, size_t ci, double cutoff, uint32_t lo, uint32_t hi, ShardHead& h,
                         std::vector<ShardComp>& local) {
  h = ShardHead{};
  local.clear();
  Slot& L = P.slot0();
  if (S.lock_dirty) {
    TRY(P.push_locks(S.base, S.n, L.st));
    S.lock_dirty = false;
  }
  if (lo == hi) return 0;
  TRY(L.ensure_tasks(1));
  TaskDev T = S.task_for(ci, cutoff);
  T.base = S.base + lo;
  T.n = hi - lo;
  L.task_stage.h[0] = T;
  TRY(L.run_compare(1, true, nullptr));
  L.task_counters(0, h.ctr);
  h.ns = h.ctr[TC_STORED];
  h.has_self = T.center >= T.base && T.center - T.base < T.n ? 1u : 0u;
  h.self = h.has_self ? L.task_self.h[0] : 0.0;
  local.reserve(h.ns);
  L.for_each_stored(0, [&](uint32_t idx, double lam, uint32_t ham, float ll) {
    local.push_back(ShardComp{lo + idx, ham, lam, ll, 0u});
  });
  return 0;
}

// The clustering loop of the batch's one sample with the compares sharded;
// prep_rc = this rank's batch_prepare outcome, exchanged first so that a rank
// that could not prepare stops the others before their first compare.
static int shard_run(Batch& B, int prep_rc, int rank, int world, const ShardGather& gather, dgpu_result** out) {
  Pool& P = B.pool;
  const auto t0 = Clock::now();
  std::vector<SampleState> S(1);
  SampleState& s = S[0];
  ShardHead setup{};
  setup.err = prep_rc ? prep_rc : [&]() -> int {
    CUDA_TRY(cudaSetDevice(P.device));
    P.pivot_on = false;  // a share's task base is not its sample's: no pivots
    TRY(P.reset_e_minmax());
    std::memset(P.lock_host.h, 0, P.nraw);
    CUDA_TRY(cudaMemsetAsync(P.lock.p, 0, P.nraw, P.st));
    CUDA_TRY(cudaStreamSynchronize(P.st));
    return 0;
  }();
  std::vector<ShardHead> heads;
  TRY(shard_heads(setup, world, gather, heads));
  s.init(B.counts[0], B.bases[0], B.E.reads.data(), B.E.prior.data(), P.lock_host.h, &B.confs[0]);
  const std::vector<uint32_t> bounds = shard_bounds(B.E.len.data(), s.n, world);
  const uint32_t lo = bounds[size_t(rank)], hi = bounds[size_t(rank) + 1];
  ShardHead h{};
  std::vector<ShardComp> local;
  for (int64_t ci = 0; ci >= 0;) {
    const auto tc = Clock::now();
    const int rc = shard_compare(P, s, size_t(ci), ci == 0 ? 1.0 : B.align.kdist_cutoff, lo, hi, h, local);
    if (rc) {
      h = ShardHead{rc, 0, 0, 0, 0.0, {}};
      local.clear();
    }
    TRY(shard_exchange(s, size_t(ci), h, local, world, gather));
    const auto th = Clock::now();
    s.stats.t_compare += secs(tc, th);
    ci = s.advance(size_t(ci));
    s.stats.t_host += secs(th, Clock::now());
  }
  s.stats.t_done = s.stats.t_total = secs(t0, Clock::now());
  out[0] = finish(s, SampleSeqs{B.E.seq, B.E.off.data(), B.E.len.data()});
  const int rc = B.transitions ? final_subs(B, S, out) : 0;
  s.release();
  return rc;
}

}  // namespace dgpu

// ---------------------------------------------------------------------------
// Compare-level context
// ---------------------------------------------------------------------------
struct dgpu_batch {
  dgpu::Batch b;
};

struct dgpu_ctx {
  dgpu::Pool pool;
  dgpu::KParams kp{};
  std::vector<double> err;
  std::vector<uint32_t> reads;
  bool uploaded = false;
};

using namespace dgpu;

struct dgpu_learn {
  int32_t nq = 0, passes = 0, converged = 0;
  std::vector<uint32_t> trans;
  std::vector<double> err_in, err_out;
};

namespace dgpu {
int errfun_apply(const dgpu_errfun& ef, const uint32_t* trans, int nq, double* err, std::string* msg);

// One learn-errors pass over the prepared samples: denoise them all with
// `err` (16 x nq) and at most max_clust clusters each (0: the parameters'
// own), count each sample's transitions as build_trans_mat does and sum them
// (accumulate_trans, src/error_models.rs:495-515, wrapping u32 additions).
static int learn_pass(Batch& B, const std::vector<double>& err, size_t max_clust, int nq,
                      std::vector<uint32_t>& acc) {
  Pool& P = B.pool;
  CUDA_TRY(cudaSetDevice(P.device));
  CUDA_TRY(cudaMemcpy(P.err.p, err.data(), err.size() * 8, cudaMemcpyHostToDevice));
  count_h2d(err.size() * 8);
  const size_t ns = B.counts.size();
  std::vector<size_t> keep(ns);
  for (size_t s = 0; s < ns; ++s) {
    keep[s] = B.confs[s].max_clust;
    if (max_clust) B.confs[s].max_clust = max_clust;
  }
  std::vector<dgpu_result*> res(ns, nullptr);
  const int rc = batch_run(B, res.data());
  for (size_t s = 0; s < ns; ++s) B.confs[s].max_clust = keep[s];
  acc.assign(size_t(16) * nq, 0u);
  for (dgpu_result* R : res) {
    if (!R) continue;
    if (!rc && R->transitions.size() == acc.size())
      for (size_t b = 0; b < acc.size(); ++b) acc[b] += R->transitions[b];
    dgpu_result_free(R);
  }
  return rc;
}
}  // namespace dgpu

extern "C" {

const char* dgpu_last_error(void) { return g_err.c_str(); }

int dgpu_device_count(int* count) {
  if (!count) return fail(DGPU_E_INVALID, "null count");
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *count = 0;
    return fail(DGPU_E_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  }
  *count = c;
  return 0;
}

int dgpu_ctx_create(int device, const dgpu_align_params* params, const double* err_mat, int ncol, int use_quals,
                    dgpu_ctx** out) {
  if (!params || !err_mat || !out || ncol <= 0) return fail(DGPU_E_INVALID, "null argument or ncol <= 0");
  if (params->kmer_size < 3 || params->kmer_size > 8)
    return fail(DGPU_E_INVALID, "kmer_size out of supported range (3..=8).");
  dgpu_ctx* c = new dgpu_ctx();
  int rc = c->pool.init(device);
  if (rc) {
    delete c;
    return rc;
  }
  c->pool.replay_graphs = true;  // a compare context serves many calls
  c->kp = to_kparams(*params, use_quals, 1, ncol);
  c->err.assign(err_mat, err_mat + 16 * size_t(ncol));
  *out = c;
  return 0;
}

void dgpu_ctx_destroy(dgpu_ctx* ctx) { delete ctx; }

int dgpu_upload_raws(dgpu_ctx* ctx, int nraw, const uint8_t* seqs, const uint32_t* offs, const uint32_t* lens,
                     const uint8_t* quals, const uint32_t* reads) {
  if (!ctx || nraw <= 0 || !seqs || !offs || !lens || !reads) return fail(DGPU_E_INVALID, "null argument or nraw <= 0");
  for (int t = 0; t < nraw; ++t) {
    if (lens[t] <= uint32_t(ctx->kp.kmer_size)) return fail(DGPU_E_INVALID, "sequence not longer than the k-mer size");
    if (lens[t] >= 9999) return fail(DGPU_E_INVALID, "sequence length >= 9999");
    for (uint32_t p = 0; p < lens[t]; ++p)
      if (seqs[offs[t] + p] < 1 || seqs[offs[t] + p] > 4) return fail(DGPU_E_INVALID, "non-ACGT code in sequence");
    if (quals)
      for (uint32_t p = 0; p < lens[t]; ++p)
        if (quals[offs[t] + p] >= ctx->kp.ncol) return fail(DGPU_E_INVALID, "quality beyond the error matrix");
  }
  ctx->reads.assign(reads, reads + nraw);
  TRY(ctx->pool.upload(uint32_t(nraw), seqs, offs, lens, quals, reads, ctx->kp, ctx->err.data()));
  ctx->uploaded = true;
  return 0;
}

int dgpu_set_locks(dgpu_ctx* ctx, const uint8_t* lock) {
  if (!ctx || !ctx->uploaded || !lock) return fail(DGPU_E_INVALID, "no raws uploaded or null lock");
  std::memcpy(ctx->pool.lock_host.h, lock, ctx->pool.nraw);
  TRY(ctx->pool.push_locks(0, ctx->pool.nraw, ctx->pool.st));
  CUDA_TRY(cudaStreamSynchronize(ctx->pool.st));
  return 0;
}

int dgpu_reset_e_minmax(dgpu_ctx* ctx) {
  if (!ctx || !ctx->uploaded) return fail(DGPU_E_INVALID, "no raws uploaded");
  return ctx->pool.reset_e_minmax();
}

int dgpu_get_e_minmax(dgpu_ctx* ctx, double* out) {
  if (!ctx || !ctx->uploaded || !out) return fail(DGPU_E_INVALID, "no raws uploaded or null output");
  CUDA_TRY(cudaMemcpy(out, ctx->pool.e_minmax.p, size_t(ctx->pool.nraw) * 8, cudaMemcpyDeviceToHost));
  return 0;
}

static int ctx_task(dgpu_ctx* ctx, int center, int cluster_i, double cutoff, int greedy) {
  if (!ctx || !ctx->uploaded) return fail(DGPU_E_INVALID, "no raws uploaded");
  if (center < 0 || uint32_t(center) >= ctx->pool.nraw) return fail(DGPU_E_INVALID, "center out of range");
  ctx->pool.kp.greedy = greedy ? 1 : 0;
  TRY(ctx->pool.slot0().ensure_tasks(1));
  TaskDev T{};
  T.base = 0;
  T.n = ctx->pool.nraw;
  T.center = uint32_t(center);
  T.center_reads = ctx->reads[size_t(center)];
  uint64_t tot = 0;
  for (uint32_t r : ctx->reads) tot += r;
  T.total_reads = double(uint32_t(tot));
  T.cutoff = cutoff;
  T.cluster = uint32_t(cluster_i);
  ctx->pool.slot0().task_stage.h[0] = T;
  return 0;
}

static void fill_counters(const uint32_t* c, uint32_t stored, dgpu_counters* cnt) {
  if (!cnt) return;
  cnt->screened = c[TC_SCREENED];
  cnt->aligned = c[TC_ALIGNED];
  cnt->shrouded = c[TC_SHROUD];
  cnt->stored = stored;
  cnt->gapless = c[TC_GAPLESS];
  cnt->vectorized = c[TC_VECTORIZED];
  cnt->homo = c[TC_HOMO];
  cnt->endsfree = c[TC_ENDSFREE];
}

int dgpu_ctx_set_lambda32(dgpu_ctx* ctx, int enable) {
  if (!ctx) return fail(DGPU_E_INVALID, "null context");
  ctx->kp.lambda32 = enable ? 1 : 0;
  ctx->pool.kp.lambda32 = ctx->kp.lambda32;
  return 0;
}

int dgpu_get_loglambda32(dgpu_ctx* ctx, float* out) {
  if (!ctx || !out) return fail(DGPU_E_INVALID, "null argument");
  if (!ctx->uploaded) return fail(DGPU_E_INVALID, "no raws uploaded");
  CUDA_TRY(cudaMemcpy(out, ctx->pool.loglam32.p, size_t(ctx->pool.nraw) * 4, cudaMemcpyDeviceToHost));
  return 0;
}

double dgpu_calc_pA(uint32_t reads, double e_reads, int prior) {
  return SampleState::calc_pA(reads, e_reads, prior != 0);
}

int dgpu_compare(dgpu_ctx* ctx, int center, double kdist_cutoff, int greedy, double* lambda_out,
                 uint32_t* hamming_out, uint8_t* skipped_out, dgpu_counters* cnt) {
  TRY(ctx_task(ctx, center, 0, kdist_cutoff, greedy));
  Pool& P = ctx->pool;
  TRY(P.slot0().run_compare(1, false, nullptr));
  const uint32_t n = P.nraw;
  std::vector<uint8_t> st(n);
  if (lambda_out) CUDA_TRY(cudaMemcpy(lambda_out, P.lambda.p, size_t(n) * 8, cudaMemcpyDeviceToHost));
  if (hamming_out) CUDA_TRY(cudaMemcpy(hamming_out, P.ham.p, size_t(n) * 4, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(st.data(), P.status.p, n, cudaMemcpyDeviceToHost));
  if (skipped_out)
    for (uint32_t t = 0; t < n; ++t) skipped_out[t] = (st[t] & 3u) == ST_SKIPPED;
  if (cnt) {
    uint32_t c[TC_NCOUNTERS] = {0};
    for (uint32_t t = 0; t < n; ++t) {
      const uint8_t o = st[t] & 3u, m = st[t] >> 2;
      c[TC_SCREENED] += o != ST_SKIPPED;
      c[TC_ALIGNED] += o == ST_ALIGNED;
      c[TC_SHROUD] += o == ST_SHROUDED;
      c[TC_GAPLESS] += m == AM_GAPLESS;
      c[TC_VECTORIZED] += m == AM_VECTORIZED;
      c[TC_HOMO] += m == AM_HOMO;
      c[TC_ENDSFREE] += m == AM_ENDSFREE;
    }
    fill_counters(c, 0, cnt);
  }
  return 0;
}

int dgpu_get_methods(dgpu_ctx* ctx, uint8_t* out) {
  if (!ctx || !out) return fail(DGPU_E_INVALID, "null argument");
  Pool& P = ctx->pool;
  const uint32_t n = P.nraw;
  CUDA_TRY(cudaMemcpy(out, P.status.p, n, cudaMemcpyDeviceToHost));
  for (uint32_t t = 0; t < n; ++t) out[t] = uint8_t(out[t] >> 2);
  return 0;
}

int dgpu_compare_store(dgpu_ctx* ctx, int center, int cluster_i, double kdist_cutoff, int greedy,
                       uint32_t* comp_index, double* comp_lambda, uint32_t* comp_hamming, int* nstored,
                       double* self_out, dgpu_counters* cnt) {
  TRY(ctx_task(ctx, center, cluster_i, kdist_cutoff, greedy));
  Slot& P = ctx->pool.slot0();
  TRY(P.run_compare(1, true, nullptr));
  uint32_t ctr[TC_NCOUNTERS];
  P.task_counters(0, ctr);
  uint32_t k = 0;
  P.for_each_stored(0, [&](uint32_t idx, double lam, uint32_t ham, float) {
    if (comp_index) comp_index[k] = idx;
    if (comp_lambda) comp_lambda[k] = lam;
    if (comp_hamming) comp_hamming[k] = ham;
    ++k;
  });
  if (nstored) *nstored = int(k);
  if (self_out) *self_out = P.task_self.h[0];
  fill_counters(ctr, k, cnt);
  return 0;
}

int dgpu_batch_prepare(int device, const dgpu_dada_params* params, int nsamples, const uint32_t* sample_start,
                       const char* seqs, const uint32_t* offs, const uint32_t* lens, const uint32_t* abund,
                       const uint8_t* prior, const uint32_t* qual_sums, const double* err_mat, int ncol,
                       dgpu_batch** out) {
  if (!out) return fail(DGPU_E_INVALID, "null output");
  dgpu_batch* b = new dgpu_batch();
  int rc = batch_prepare(b->b, device, params, nsamples, sample_start, seqs, offs, lens, abund, prior, qual_sums,
                         err_mat, ncol);
  if (rc) {
    delete b;
    return rc;
  }
  b->b.pool.replay_graphs = true;  // a resident batch runs many times
  *out = b;
  return 0;
}

int dgpu_batch_run(dgpu_batch* batch, dgpu_result** out) {
  if (!batch || !out) return fail(DGPU_E_INVALID, "null argument");
  return batch_run(batch->b, out);
}

void dgpu_batch_free(dgpu_batch* batch) { delete batch; }

int dgpu_dada(int device, const dgpu_dada_params* params, int nraw, const char* seqs, const uint32_t* offs,
              const uint32_t* lens, const uint32_t* abund, const uint8_t* prior, const uint32_t* qual_sums,
              const double* err_mat, int ncol, dgpu_result** out) {
  if (nraw <= 0) return fail(DGPU_E_INVALID, "Zero input sequences.");
  if (!params) return fail(DGPU_E_INVALID, "null params");
  const uint32_t ss[2] = {0, uint32_t(nraw)};
  dgpu_dada_params p1 = *params;
  p1.host_threads = 1;
  return dgpu_dada_batch(device, &p1, 1, ss, seqs, offs, lens, abund, prior, qual_sums, err_mat, ncol, out);
}

int dgpu_dada_sharded(int device, const dgpu_dada_params* params, int nraw, const char* seqs, const uint32_t* offs,
                      const uint32_t* lens, const uint32_t* abund, const uint8_t* prior, const uint32_t* qual_sums,
                      const double* err_mat, int ncol, int rank, int world, dgpu_allgather_fn gather, void* user,
                      dgpu_result** out) {
  // argument errors return before the first exchange: they are the caller's on every rank
  if (!out || !gather) return fail(DGPU_E_INVALID, "null output or gather");
  if (world < 1 || rank < 0 || rank >= world) return fail(DGPU_E_INVALID, "rank out of range of world");
  *out = nullptr;
  const ShardGather g = [&](const void* s, uint64_t bytes, void* r) { return gather(user, s, bytes, r); };
  Batch b;
  int prep = 0;
  if (nraw <= 0) {
    prep = fail(DGPU_E_INVALID, "Zero input sequences.");
  } else if (!params) {
    prep = fail(DGPU_E_INVALID, "null params");
  } else {
    const uint32_t ss[2] = {0, uint32_t(nraw)};
    dgpu_dada_params p1 = *params;
    p1.host_threads = 1;
    prep = batch_prepare(b, device, &p1, 1, ss, seqs, offs, lens, abund, prior, qual_sums, err_mat, ncol);
  }
  const int rc = shard_run(b, prep, rank, world, g, out);
  if (rc) {
    delete *out;
    *out = nullptr;
  }
  return rc;
}

int dgpu_dada_batch(int device, const dgpu_dada_params* params, int nsamples, const uint32_t* sample_start,
                    const char* seqs, const uint32_t* offs, const uint32_t* lens, const uint32_t* abund,
                    const uint8_t* prior, const uint32_t* qual_sums, const double* err_mat, int ncol,
                    dgpu_result** out) {
  if (!out) return fail(DGPU_E_INVALID, "null output");
  dgpu_batch b;
  TRY(batch_prepare(b.b, device, params, nsamples, sample_start, seqs, offs, lens, abund, prior, qual_sums, err_mat,
                    ncol));
  return batch_run(b.b, out);
}

int dgpu_learn_errors(int device, const dgpu_dada_params* params, const dgpu_errfun* errfun, int max_consist,
                      int nsamples, const uint32_t* sample_start, const char* seqs, const uint32_t* offs,
                      const uint32_t* lens, const uint32_t* abund, const uint32_t* qual_sums, dgpu_learn** out) {
  using namespace dgpu;
  if (!out || !params || !errfun || max_consist < 0 || nsamples <= 0 || !sample_start || !lens || !abund)
    return fail(DGPU_E_INVALID, "bad argument");
  if (!qual_sums) return fail(DGPU_E_INVALID, "learn-errors needs quality sums: without them no transition is counted");
  *out = nullptr;
  // nq: the largest round(sum / reads) over every position of every sample,
  // plus one (src/learn_errors.rs:494-506)
  uint32_t qmax = 0;
  for (uint32_t t = sample_start[0]; t < sample_start[nsamples]; ++t) {
    const double ab = double(abund[t]);
    for (uint32_t p = 0; p < lens[t]; ++p) {
      const double q = std::round(double(qual_sums[size_t(offs[t]) + p]) / ab);
      if (q > double(qmax)) qmax = uint32_t(std::min(q, 1e9));
    }
  }
  const int nq = int(qmax) + 1;
  std::vector<double> err(size_t(16) * nq, 1.0);  // the init pass: every entry 1 (src/learn_errors.rs:536-540)
  dgpu_dada_params prm = *params;
  prm.transitions = 1;
  prm.lambda_fp32 = 0;
  dgpu_batch b;
  TRY(batch_prepare(b.b, device, &prm, nsamples, sample_start, seqs, offs, lens, abund, nullptr, qual_sums, err.data(),
                    nq));
  Batch& B = b.b;
  B.learn_nq = nq;
  B.pool.replay_graphs = true;  // several passes over the same pool
  std::unique_ptr<dgpu_learn> L(new dgpu_learn());
  L->nq = nq;
  std::vector<uint32_t> acc;
  std::string msg;
  // init pass: one cluster per sample, fit, diagonals forced to 1
  TRY(learn_pass(B, err, 1, nq, acc));
  std::vector<double> fit(size_t(16) * nq);
  if (int rc = errfun_apply(*errfun, acc.data(), nq, fit.data(), &msg)) return fail(rc, "init-pass errfun failed: " + msg);
  for (int r : {0, 5, 10, 15})
    for (int q = 0; q < nq; ++q) fit[size_t(r) * nq + q] = 1.0;
  err = fit;
  L->trans.assign(size_t(16) * nq, 0u);
  L->err_in = err;
  L->err_out = err;
  std::vector<std::vector<double>> history;
  for (int it = 0; it < max_consist; ++it) {
    L->passes = it + 1;
    history.push_back(err);
    TRY(learn_pass(B, err, 0, nq, acc));
    if (int rc = errfun_apply(*errfun, acc.data(), nq, fit.data(), &msg)) return fail(rc, "errfun failed: " + msg);
    // converged when the fit equals (as f64 values) a matrix already used
    // as input (src/learn_errors.rs:962-967)
    bool conv = false;
    for (const auto& h : history) conv |= h == fit;
    L->err_in = err;
    L->trans = acc;
    L->err_out = fit;
    if (conv) {
      L->converged = 1;
      break;
    }
    err = fit;
  }
  *out = L.release();
  return 0;
}

int dgpu_learn_read(const dgpu_learn* l, int32_t* info, uint32_t* trans, double* err_in, double* err_out) {
  if (!l) return dgpu::fail(DGPU_E_INVALID, "null argument");
  if (info) {
    info[0] = l->nq;
    info[1] = l->passes;
    info[2] = l->converged;
  }
  if (trans) std::copy(l->trans.begin(), l->trans.end(), trans);
  if (err_in) std::copy(l->err_in.begin(), l->err_in.end(), err_in);
  if (err_out) std::copy(l->err_out.begin(), l->err_out.end(), err_out);
  return 0;
}

void dgpu_learn_free(dgpu_learn* l) { delete l; }

int dgpu_cache_release(int device, uint64_t* freed) {
  const size_t n = cache_release(device);
  if (freed) *freed = uint64_t(n);
  return 0;
}

int dgpu_stats_reset(void) {
  std::lock_guard<std::mutex> g(g_stats.mu);
  g_stats.s = dgpu_kernel_stats{};
  g_stats.round_ms.clear();
  return 0;
}

int dgpu_stats_latencies(double* out, int cap) {
  std::lock_guard<std::mutex> g(g_stats.mu);
  const int n = int(std::min<size_t>(g_stats.round_ms.size(), size_t(cap > 0 ? cap : 0)));
  if (out && n > 0) std::memcpy(out, g_stats.round_ms.data(), size_t(n) * 8);
  return int(g_stats.round_ms.size());
}

int dgpu_stats_timing(int every) {
  g_stats.timing_every.store(every > 0 ? uint64_t(every) : 0u);
  g_stats.call_seq.store(0);
  return 0;
}

int dgpu_stats_read(dgpu_kernel_stats* out) {
  if (!out) return fail(DGPU_E_INVALID, "null output");
  std::lock_guard<std::mutex> g(g_stats.mu);
  *out = g_stats.s;
  return 0;
}

int dgpu_result_sizes(const dgpu_result* r, int64_t* sizes) {
  if (!r || !sizes) return fail(DGPU_E_INVALID, "null argument");
  sizes[0] = int64_t(r->cl_reads.size());
  sizes[1] = int64_t(r->nraw);
  sizes[2] = int64_t(r->mem_raw.size());
  sizes[3] = int64_t(r->cl_seq.size());
  return 0;
}

int dgpu_result_fp32_stats(const dgpu_result* r, uint64_t* out2) {
  if (!r || !out2) return fail(DGPU_E_INVALID, "null argument");
  out2[0] = r->fp32[0];
  out2[1] = r->fp32[1];
  return 0;
}

int dgpu_tuning_get(int max_len, dgpu_tuning* out) {
  if (!out || max_len < 0) return fail(DGPU_E_INVALID, "bad argument");
  *out = tuning_for(uint32_t(max_len));
  return 0;
}

int dgpu_tuning_set(int length_class, const dgpu_tuning* t) {
  if (!t || length_class < 0 || length_class > 2) return fail(DGPU_E_INVALID, "bad argument");
  if (!tuning_valid(*t)) return fail(DGPU_E_INVALID, "tuning value out of range");
  std::lock_guard<std::mutex> g(g_tune_mu);
  tuning_first_use();  // the default file must not overwrite this later
  g_tune[length_class] = *t;
  return 0;
}

int dgpu_tuning_load(const char* path) {
  if (!path) return fail(DGPU_E_INVALID, "null path");
  std::lock_guard<std::mutex> g(g_tune_mu);
  tuning_first_use();
  std::string msg;
  const int rc = tuning_load_file(path, &msg);
  return rc ? fail(rc, msg) : 0;
}

int dgpu_tuning_save(const char* path) {
  if (!path) return fail(DGPU_E_INVALID, "null path");
  const dgpu_tuning t[3] = {tuning_class(0), tuning_class(1), tuning_class(2)};
  const std::string text = tuning_format(t);
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(DGPU_E_INVALID, std::string("cannot write ") + path);
  const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
  std::fclose(f);
  return ok ? 0 : fail(DGPU_E_INVALID, std::string("short write to ") + path);
}

int dgpu_tuning_reset(void) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune_loaded = true;  // the built-in table; no file is read afterwards
  for (int c = 0; c < 3; ++c) g_tune[c] = kTuneDefault;
  return 0;
}

int dgpu_result_margins(const dgpu_result* r, double* out3) {
  if (!r || !out3) return fail(DGPU_E_INVALID, "null argument");
  std::copy(r->margin, r->margin + 3, out3);
  return 0;
}

int dgpu_result_transitions(const dgpu_result* r, uint32_t* out) {
  if (!r) return fail(DGPU_E_INVALID, "null argument");
  if (out && !r->transitions.empty())
    std::memcpy(out, r->transitions.data(), r->transitions.size() * sizeof(uint32_t));
  return r->tncol;
}

int dgpu_result_fill(const dgpu_result* r, const dgpu_dada_out* o) {
  if (!r || !o) return fail(DGPU_E_INVALID, "null argument");
  auto cp = [](auto* dst, const auto& v) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
  };
  cp(o->cl_reads, r->cl_reads);
  cp(o->cl_birth_type, r->cl_birth_type);
  cp(o->cl_birth_from, r->cl_birth_from);
  cp(o->cl_birth_pval, r->cl_birth_pval);
  cp(o->cl_birth_fold, r->cl_birth_fold);
  cp(o->cl_birth_e, r->cl_birth_e);
  cp(o->cl_birth_hamming, r->cl_birth_hamming);
  cp(o->cl_seq_off, r->cl_seq_off);
  cp(o->cl_seq, r->cl_seq);
  cp(o->cl_mem_off, r->cl_mem_off);
  cp(o->mem_raw, r->mem_raw);
  cp(o->mem_hamming, r->mem_hamming);
  cp(o->mem_lambda, r->mem_lambda);
  cp(o->mem_pval, r->mem_pval);
  cp(o->map, r->map);
  cp(o->pvals, r->pvals);
  if (o->counters) std::memcpy(o->counters, r->counters, sizeof(r->counters));
  if (o->times) std::memcpy(o->times, r->times, sizeof(r->times));
  return 0;
}

void dgpu_result_free(dgpu_result* r) { delete r; }

int dgpu_align_debug(int device, int which, int npairs, const uint8_t* s1cat, const uint32_t* off1,
                     const uint32_t* len1, const uint8_t* s2cat, const uint32_t* off2, const uint32_t* len2,
                     const dgpu_align_params* params, int end_gap, uint8_t* al0, uint8_t* al1, const uint32_t* al_off,
                     uint32_t* al_len) {
  if (npairs <= 0 || !params || !s1cat || !s2cat || which < 0 || which > 2) return fail(DGPU_E_INVALID, "bad argument");
  CUDA_TRY(cudaSetDevice(device));
  uint32_t lmax = 0, lmin = 0xffffffffu;
  size_t b1 = 0, b2 = 0, bal = 0;
  for (int t = 0; t < npairs; ++t) {
    lmax = std::max({lmax, len1[t], len2[t]});
    lmin = std::min({lmin, len1[t], len2[t]});
    b1 = std::max<size_t>(b1, size_t(off1[t]) + len1[t]);
    b2 = std::max<size_t>(b2, size_t(off2[t]) + len2[t]);
    bal = std::max<size_t>(bal, size_t(al_off[t]) + len1[t] + len2[t]);
    if (which == 0 && (len1[t] > 3500 || len2[t] > 3500)) return fail(DGPU_E_INVALID, "vectorized aligner needs len <= 3500");
  }
  KParams kp = to_kparams(*params, 0, 0, 1);
  kp.gap = params->gap_p;
  NwGeom g{};
  g.lmax = int32_t(lmax);
  const int64_t bb = kp.band < 0 ? int64_t(lmax) : int64_t(kp.band);
  const int64_t diff = int64_t(lmax) - int64_t(lmin);
  g.vec_ncol = int32_t(4 + (std::min<int64_t>(bb, lmax) + 1) / 2 + std::min<int64_t>(bb + diff, lmax) / 2);
  g.vec_nrow = int32_t(2 * lmax + 1);
  int64_t W = kp.band < 0 ? int64_t(2 * lmax + 1) : std::min<int64_t>(2 * bb + diff + 1, 2 * int64_t(lmax) + 1);
  g.rm_pairs = int32_t(std::min<int64_t>((W + 1) / 2, 512));
  g.vec_scratch = align16(size_t(g.vec_nrow) * std::max<size_t>(size_t(g.vec_ncol), 32));
  g.rm_scratch = align16(size_t(2 * lmax + 1) * 2 * rm_kbound(g.rm_pairs) * 4);
  g.nwarps = npairs;
  const size_t per = which == 0 ? g.vec_scratch : g.rm_scratch;
  DBuf<uint8_t> d1, d2, scr, a0, a1;
  DBuf<uint32_t> o1, l1, o2, l2, ao, al, ew;
  TRY(d1.alloc(b1));
  TRY(d2.alloc(b2));
  TRY(scr.alloc(per * size_t(npairs)));
  TRY(a0.alloc(bal));
  TRY(a1.alloc(bal));
  TRY(o1.alloc(npairs));
  TRY(l1.alloc(npairs));
  TRY(o2.alloc(npairs));
  TRY(l2.alloc(npairs));
  TRY(ao.alloc(npairs));
  TRY(al.alloc(npairs));
  TRY(ew.alloc(1));
  CUDA_TRY(cudaMemcpy(d1.p, s1cat, b1, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(d2.p, s2cat, b2, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(o1.p, off1, 4 * size_t(npairs), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(l1.p, len1, 4 * size_t(npairs), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(o2.p, off2, 4 * size_t(npairs), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(l2.p, len2, 4 * size_t(npairs), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(ao.p, al_off, 4 * size_t(npairs), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemset(al.p, 0, 4 * size_t(npairs)));
  CUDA_TRY(cudaMemset(ew.p, 0, 4));
  launch_align_debug(which, d1.p, o1.p, l1.p, d2.p, o2.p, l2.p, uint32_t(npairs), kp, end_gap, g, scr.p, a0.p, a1.p,
                     ao.p, al.p, ew.p, nullptr);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaDeviceSynchronize());
  uint32_t e = 0;
  CUDA_TRY(cudaMemcpy(&e, ew.p, 4, cudaMemcpyDeviceToHost));
  std::vector<uint8_t> h0(bal), h1(bal);
  CUDA_TRY(cudaMemcpy(h0.data(), a0.p, bal, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(h1.data(), a1.p, bal, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(al_len, al.p, 4 * size_t(npairs), cudaMemcpyDeviceToHost));
  for (int t = 0; t < npairs; ++t) {  // traceback order -> left to right
    const uint32_t o = al_off[t], n = al_len[t];
    for (uint32_t q = 0; q < n; ++q) {
      al0[o + q] = h0[o + n - 1 - q];
      al1[o + q] = h1[o + n - 1 - q];
    }
  }
  if (e) return fail(e & DERR_UNSUPPORTED ? DGPU_E_UNSUPPORTED : DGPU_E_DEVICE, "device error flag " + std::to_string(e));
  return 0;
}

}  // extern "C"

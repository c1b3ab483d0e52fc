// CUDA kernels of the dada compare step (sm_100a).
//
//   k_profiles  -- K1: dense saturating u8 k-mer counts per unique (src/kmers.rs:79-101)
//   k_screen    -- K2/K3/K6: greedy skip, k-mer screen, ordered-k-mer distance, gapless
//                  alignment and the FP64 lambda product, one warp per (center, raw)
//                  (src/cluster.rs:279-330, src/nwalign.rs:1244-1327, src/pval.rs:253-320)
//   k_nw_vec    -- K4: replica of the rolling i16 anti-diagonal aligner + traceback
//                  (src/nwalign.rs:665-1140), one warp per pair, persistent
//   k_nw_rm     -- K5: the row-major i32 ends-free / homopolymer aligner
//                  (src/nwalign.rs:336-528) evaluated as an anti-diagonal wavefront,
//                  one warp per pair, persistent
//   k_store     -- K7: ordered store + e_minmax update + counters (src/cluster.rs:351-397)
//
// Built with --fmad=false: the FP64 product and the k-mer distances must round
// exactly like the reference's separately-rounded operations.
#include <atomic>
#include <algorithm>
#include <type_traits>
#include <cfloat>
#include <cstdio>
#include <mutex>

#include "dada2_b200.h"
#include "dgpu_common.h"

namespace dgpu {

#define FULL 0xffffffffu
static constexpr int kNegSentinel = -9999;  // BAND_SENTINEL, src/nwalign.rs:30

__device__ __forceinline__ int16_t sadd16(int16_t a, int16_t b) {
  int s = int(a) + int(b);
  s = s > 32767 ? 32767 : (s < -32768 ? -32768 : s);
  return int16_t(s);
}

__device__ __forceinline__ uint32_t find_task(const uint32_t* prefix, uint32_t ntask, uint32_t item) {
  uint32_t lo = 0, hi = ntask;  // largest t with prefix[t] <= item
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (prefix[mid] <= item) lo = mid;
    else hi = mid;
  }
  return lo;
}

// ---------------------------------------------------------------------------
// K1: k-mer profiles
// ---------------------------------------------------------------------------
__global__ void k_profiles(const uint8_t* __restrict__ seq, const uint32_t* __restrict__ off,
                           const uint32_t* __restrict__ len, uint32_t nraw, int k,
                           uint8_t* __restrict__ kmer8, uint8_t* __restrict__ sat) {
  extern __shared__ uint32_t cnt[];
  __shared__ int any_sat;
  const int nk = 1 << (2 * k);
  for (uint32_t g = blockIdx.x; g < nraw; g += gridDim.x) {
    if (threadIdx.x == 0) any_sat = 0;
    for (int t = threadIdx.x; t < nk; t += blockDim.x) cnt[t] = 0;
    __syncthreads();
    const uint8_t* s = seq + off[g];
    const int L = int(len[g]);
    for (int p = threadIdx.x; p + k <= L; p += blockDim.x) {
      int idx = 0;
      bool ok = true;
      for (int q = 0; q < k; ++q) {
        unsigned nt = s[p + q];
        if (nt < 1u || nt > 4u) {
          ok = false;
          break;
        }
        idx = idx * 4 + int(nt - 1u);
      }
      if (ok) atomicAdd(&cnt[idx], 1u);
    }
    __syncthreads();
    uint32_t* out = reinterpret_cast<uint32_t*>(kmer8 + size_t(g) * size_t(nk));
    int my_sat = 0;
    for (int t = threadIdx.x; t < nk / 4; t += blockDim.x) {
      uint32_t w = 0;
      for (int b = 0; b < 4; ++b) {
        w |= min(cnt[4 * t + b], 255u) << (8 * b);
        my_sat |= cnt[4 * t + b] >= 255u;
      }
      out[t] = w;
    }
    if (my_sat) any_sat = 1;
    __syncthreads();
    if (threadIdx.x == 0) sat[g] = uint8_t(any_sat);
    __syncthreads();
  }
}

void launch_profiles(const uint8_t* seq, const uint32_t* off, const uint32_t* len, uint32_t nraw, int k,
                     uint8_t* kmer8, uint8_t* sat, cudaStream_t st) {
  if (nraw == 0) return;
  size_t smem = size_t(4) << (2 * k);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_profiles, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  int grid = int(nraw < 148u * 16u ? nraw : 148u * 16u);
  k_profiles<<<grid, 256, smem, st>>>(seq, off, len, nraw, k, kmer8, sat);
}

// K1 for k = 8 (src/kmers.rs:113-120): one CTA per raw sorts its window codes
// in shared memory (bitonic), then run-length encodes them into ascending
// (index, count) pairs with counts saturating at 255 (the u16 count is exact up
// to 9,991 windows, so `count >= 255` also gives the saturation flag).
__global__ void __launch_bounds__(256) k_profiles_sparse(const uint8_t* __restrict__ seq,
                                                         const uint32_t* __restrict__ off,
                                                         const uint32_t* __restrict__ len, uint32_t nraw,
                                                         uint16_t* __restrict__ kidx, uint8_t* __restrict__ kcnt,
                                                         uint32_t* __restrict__ knum, uint8_t* __restrict__ sat) {
  extern __shared__ uint32_t keys[];  // padded to a power of two >= the longest window count
  __shared__ uint32_t warp_tot[8];
  __shared__ int any_sat;
  constexpr int K = 8;
  for (uint32_t g = blockIdx.x; g < nraw; g += gridDim.x) {
    const uint8_t* s = seq + off[g];
    const int L = int(len[g]);
    const int nwin = L >= K ? L - K + 1 : 0;
    int np2 = 1;
    while (np2 < nwin) np2 <<= 1;
    for (int p = threadIdx.x; p < np2; p += blockDim.x) {
      uint32_t x = 0xffffffffu;  // padding sorts last
      if (p < nwin) {
        x = 0;
        for (int q = 0; q < K; ++q) x = x * 4u + (unsigned(s[p + q]) - 1u);  // codes are 1..4 (validated)
      }
      keys[p] = x;
    }
    if (threadIdx.x == 0) any_sat = 0;
    __syncthreads();
    for (int size = 2; size <= np2; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int i = threadIdx.x; i < np2; i += blockDim.x) {
          const int j = i ^ stride;
          if (j > i) {
            const bool up = (i & size) == 0;
            const uint32_t a = keys[i], b = keys[j];
            if ((a > b) == up) {
              keys[i] = b;
              keys[j] = a;
            }
          }
        }
        __syncthreads();
      }
    }
    // run starts -> ascending distinct indices with their counts
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t written = 0;
    for (int base = 0; base < nwin; base += blockDim.x) {
      const int i = base + threadIdx.x;
      const bool start = i < nwin && (i == 0 || keys[i] != keys[i - 1]);
      const uint32_t bal = __ballot_sync(FULL, start);
      if (lane == 0) warp_tot[w] = __popc(bal);
      __syncthreads();
      uint32_t before = written;
      for (int q = 0; q < w; ++q) before += warp_tot[q];
      uint32_t tot = 0;
      for (int q = 0; q < int(blockDim.x >> 5); ++q) tot += warp_tot[q];
      if (start) {
        int e = i + 1;
        while (e < nwin && keys[e] == keys[i]) ++e;
        const int cnt = e - i;
        const uint32_t slot = before + __popc(bal & ((1u << lane) - 1u));
        kidx[off[g] + slot] = uint16_t(keys[i]);
        kcnt[off[g] + slot] = uint8_t(cnt < 255 ? cnt : 255);
        if (cnt >= 255) any_sat = 1;
      }
      written += tot;
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      knum[g] = written;
      sat[g] = uint8_t(any_sat);
    }
    __syncthreads();
  }
}

void launch_profiles_sparse(const uint8_t* seq, const uint32_t* off, const uint32_t* len, uint32_t nraw, uint32_t lmax,
                            uint16_t* kidx, uint8_t* kcnt, uint32_t* knum, uint8_t* sat, cudaStream_t st) {
  if (nraw == 0) return;
  size_t np2 = 1;
  while (np2 < lmax) np2 <<= 1;
  const size_t smem = np2 * 4;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_profiles_sparse, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  const int grid = int(nraw < 148u * 8u ? nraw : 148u * 8u);
  k_profiles_sparse<<<grid, 256, smem, st>>>(seq, off, len, nraw, kidx, kcnt, knum, sat);
}

__global__ void k_fill_f64(double* __restrict__ p, size_t n, double v) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) p[i] = v;
}

void launch_fill_f64(double* p, size_t n, double v, cudaStream_t st) {
  if (n == 0) return;
  const size_t blocks = std::min<size_t>((n + 255) / 256, size_t(148) * 8);
  k_fill_f64<<<unsigned(blocks), 256, 0, st>>>(p, n, v);
}

// ---------------------------------------------------------------------------
// Shared helpers for the lambda product
// ---------------------------------------------------------------------------
// tcode[p]: the error-matrix row of raw position p -- 4 * (center nt) + raw nt
// where the traceback aligned p to a center base, else kUnaligned | 5 * (raw nt)
// (an insertion in the raw, weighed as a match by compute_lambda and left out
// of the transition counts).
constexpr unsigned kUnaligned = 0x80u;

// fidx[p] = err row * ncol + quality column for raw position p; lane 0 then forms
// the left-to-right product (src/pval.rs:311-313). Returns the product on all lanes.
__device__ double lambda_chain(int lane, const uint16_t* fidx, int L, const double* err_s) {
  double lam = 1.0;
  if (lane == 0) {
    int p = 0;
    for (; p + 4 <= L; p += 4) {
      double f0 = err_s[fidx[p]], f1 = err_s[fidx[p + 1]], f2 = err_s[fidx[p + 2]], f3 = err_s[fidx[p + 3]];
      lam = __dmul_rn(lam, f0);
      lam = __dmul_rn(lam, f1);
      lam = __dmul_rn(lam, f2);
      lam = __dmul_rn(lam, f3);
    }
    for (; p < L; ++p) lam = __dmul_rn(lam, err_s[fidx[p]]);
  }
  return __shfl_sync(FULL, lam, 0);
}

// ln(lambda) as a compensated FP32 sum of logf(err) over the raw's positions
// (the precision variant of compute_lambda): each lane runs a Kahan sum over
// its positions, then the lanes' (sum, correction) pairs are combined with an
// error-free two-sum. Returns the result on all lanes.
__device__ float loglambda32(int lane, const uint16_t* fidx, int L, const double* err_s) {
  float s = 0.0f, c = 0.0f;
  for (int p = lane; p < L; p += 32) {
    const float y = logf(float(err_s[fidx[p]])) - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  float e = -c;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    const float so = __shfl_xor_sync(FULL, s, d), eo = __shfl_xor_sync(FULL, e, d);
    const float sum = s + so;
    const float bb = sum - s;
    const float err = (s - (sum - bb)) + (so - bb);
    s = sum;
    e = e + eo + err;
  }
  return s + e;
}

// tcode[p] (row of the error matrix for raw position p) + quality -> fidx.
__device__ bool build_fidx(int lane, const uint8_t* tcode, const uint8_t* qual_g, int L, int ncol, int use_quals,
                           uint16_t* fidx) {
  bool bad = false;
  for (int p = lane; p < L; p += 32) {
    unsigned t = tcode[p] & 0x7fu;  // insertions in the raw weigh as matches (src/pval.rs:269-291)
    bad |= t > 15u;
    unsigned q = (use_quals && qual_g) ? qual_g[p] : 0u;
    bad |= q >= unsigned(ncol);
    fidx[p] = uint16_t(t * unsigned(ncol) + q);
  }
  return __any_sync(FULL, bad);
}

// ---------------------------------------------------------------------------
// K2/K3/K6: screen, gapless alignment, lambda
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t mismatch_word(const uint8_t* a, const uint8_t* b, int base, int n, int lane) {
  int p = base + lane;
  bool mm = p < n && a[p] != b[p];
  return __ballot_sync(FULL, mm);
}

// Lean streaming screen: greedy skip, profile dot product, strict cutoff
// (src/cluster.rs:295-298, src/kmers.rs:254-269, src/nwalign.rs:1299).
// A graph replay's per-call values (CompareLaunch::hdr) into the kernel's
// own copy of the launch parameters.
__device__ __forceinline__ void load_call(CompareLaunch& L) {
  if (!L.hdr) return;
  const CallHeader H = *L.hdr;
  const uint8_t* base = reinterpret_cast<const uint8_t*>(L.hdr);
  L.ntask = H.ntask;
  L.total_items = H.total_items;
  L.screen_chunk = H.screen_chunk;
  L.nstore_blocks = H.nstore_blocks;
  L.pivot = H.pivot;
  L.cdot_ready = H.cdot_ready;
  L.total_cl = H.total_cl;
  L.tasks = reinterpret_cast<const TaskDev*>(base + H.o_tasks);
  L.task_prefix = reinterpret_cast<const uint32_t*>(base + H.o_pref);
  L.task_cl_prefix = reinterpret_cast<const uint32_t*>(base + H.o_clp);
  L.store_task = reinterpret_cast<const uint32_t*>(base + H.o_map);
  L.store_chunk = L.store_task + H.nstore_blocks;
}

// Pivot dots: for every task of the launch and every earlier cluster i of its
// sample, cdot[base + i] = the u8 k-mer dot of the task's center with cluster
// i's center (cl_center[base + i]); the screen's pivot bound reads them. One
// warp per (task, cluster) item, 16-byte vector loads of both profiles.
template <int K>
__global__ void __launch_bounds__(256) k_pivot_dots(CompareLaunch Lp) {
  CompareLaunch L = Lp;
  load_call(L);
  if (!L.cdot_ready) return;
  constexpr int NK16 = (1 << (2 * K)) / 16;
  const int lane = threadIdx.x & 31;
  const uint32_t warps_total = gridDim.x * (blockDim.x >> 5);
  for (uint32_t item = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); item < L.total_cl; item += warps_total) {
    const uint32_t t = find_task(L.task_cl_prefix, L.ntask, item);
    const TaskDev T = L.tasks[t];
    const uint32_t ci = item - L.task_cl_prefix[t];
    const uint32_t p = L.pool.cl_center[T.base + ci];
    const uint4* pc = reinterpret_cast<const uint4*>(L.pool.kmer8 + size_t(T.center) * size_t(NK16) * 16);
    const uint4* pp = reinterpret_cast<const uint4*>(L.pool.kmer8 + size_t(p) * size_t(NK16) * 16);
    uint32_t dot = 0;
    for (int v = lane; v < NK16; v += 32) {
      const uint4 a = __ldg(pc + v), b = __ldg(pp + v);
      dot = __dp4a(__vminu4(a.x, b.x), 0x01010101u, dot);
      dot = __dp4a(__vminu4(a.y, b.y), 0x01010101u, dot);
      dot = __dp4a(__vminu4(a.z, b.z), 0x01010101u, dot);
      dot = __dp4a(__vminu4(a.w, b.w), 0x01010101u, dot);
    }
    dot = __reduce_add_sync(FULL, dot);
    if (lane == 0) L.pool.cdot[T.base + ci] = dot;
  }
}

// A warp takes 32 consecutive items: lane l resolves item l's task and raw
// metadata, then the warp streams the raw profiles four at a time against the
// center profile held in registers. Survivors go to the align queue with their
// kdist parked in res_lambda.
template <int K>
__global__ void __launch_bounds__(kScreenWarps * 32, 4) k_screen(CompareLaunch Lp) {
  CompareLaunch L = Lp;
  load_call(L);
  // every screen block is running: the alignment kernel may start launching
  // (its blocks wait for this grid's results in cudaGridDependencySynchronize)
  cudaTriggerProgrammaticLaunchCompletion();
  constexpr int NK16 = (1 << (2 * K)) / 16;            // 16-byte vectors per profile
  constexpr int VPL = NK16 >= 32 ? NK16 / 32 : 1;      // vectors per lane
  constexpr bool CENTER_REGS = VPL <= 2;               // k <= 5: center stays in registers
  constexpr int NB = VPL == 1 ? 4 : (VPL == 2 ? 3 : 1); // raw profiles in flight per warp
  const KParams& kp = L.kp;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t warps_total = gridDim.x * kScreenWarps;
  const uint8_t* kmer8 = L.pool.kmer8;
  // The task table and its prefix go to shared memory when they fit, so the
  // per-item task search costs no global round trips.
  __shared__ uint32_t s_prefix[kScreenSmemTasks + 1];
  __shared__ uint32_t s_base[kScreenSmemTasks], s_center[kScreenSmemTasks], s_creads[kScreenSmemTasks];
  __shared__ double s_cutoff[kScreenSmemTasks];
  __shared__ uint32_t s_cluster[kScreenSmemTasks];
  const bool tasks_smem = L.ntask <= uint32_t(kScreenSmemTasks);
  if (tasks_smem) {
    for (uint32_t t = threadIdx.x; t <= L.ntask; t += blockDim.x) {
      s_prefix[t] = L.task_prefix[t];
      if (t < L.ntask) {
        const TaskDev T = L.tasks[t];
        s_base[t] = T.base;
        s_center[t] = T.center;
        s_creads[t] = T.center_reads;
        s_cutoff[t] = T.cutoff;
        s_cluster[t] = T.cluster;
      }
    }
    __syncthreads();
  }
  // the pivot bound (k <= 7 only): every task's center becomes a pivot
  // candidate for the sample's later calls
  const bool pivot = K < 8 && L.pivot != 0 && kp.use_kmers;
  if (pivot && blockIdx.x == 0)
    for (uint32_t t = threadIdx.x; t < L.ntask; t += blockDim.x) {
      const TaskDev T = L.tasks[t];
      if (T.cluster < T.n) L.pool.cl_center[T.base + T.cluster] = T.center;
    }
  const uint32_t CH = L.screen_chunk;  // lanes [0, CH) carry an item
  for (uint32_t chunk = (blockIdx.x * kScreenWarps + wib) * CH; chunk < L.total_items; chunk += warps_total * CH) {
    const uint32_t item = chunk + lane;
    const bool valid = uint32_t(lane) < CH && item < L.total_items;
    uint32_t t = 0, g = 0, c = 0, ccl = 0, tbase = 0;
    bool skip = false, bounded = false, pivot_raw = false, cl_fits = false;
    if (valid) {
      uint32_t creads;
      if (tasks_smem) {
        t = find_task(s_prefix, L.ntask, item);
        tbase = s_base[t];
        c = s_center[t];
        creads = s_creads[t];
        ccl = s_cluster[t];
      } else {
        t = find_task(L.task_prefix, L.ntask, item);
        tbase = L.tasks[t].base;
        c = L.tasks[t].center;
        creads = L.tasks[t].center_reads;
        ccl = L.tasks[t].cluster;
      }
      const uint32_t t0 = tasks_smem ? s_prefix[t] : L.task_prefix[t];
      const uint32_t tn = (tasks_smem ? s_prefix[t + 1] : L.task_prefix[t + 1]) - t0;
      g = tbase + (item - t0);
      cl_fits = ccl < tn;  // cluster indices of a whole sample stay below its raw count
      skip = kp.greedy && (L.pool.reads[g] > creads || L.pool.lock[g]);
      if (pivot && !skip) {
        // Exact exclusion without reading the raw's profile. For non-negative
        // count vectors min(c, r) <= min(c, p) + r - min(r, p) elementwise, so
        // dot(c, r) <= dot(c, p) + |r| - dot(r, p) for the raw's pivot center
        // p (|r| = len - K + 1 windows while no count saturates). kdist =
        // 1 - dot / (minlen - K + 1) falls as the dot rises, in floating point
        // too, so a bound kdist above the cutoff means the exact one is above
        // it as well: the raw is shrouded (src/nwalign.rs:1295-1301). Raws or
        // centers with a saturated count take the exact path and never this.
        const int lc = int(L.pool.len[c]), lg = int(L.pool.len[g]);
        pivot_raw = cl_fits && !L.pool.sat[g] && !L.pool.sat[c] && lc >= K && lg >= K;
        if (pivot_raw && L.cdot_ready) {
          const uint32_t pc = L.pool.piv_cl[g];
          if (pc < ccl) {
            const int minl = lc < lg ? lc : lg;
            const uint32_t ub = L.pool.cdot[tbase + pc] + uint32_t(lg - K + 1) - L.pool.piv_dot[g];
            const double kd_lb = 1.0 - double(ub) / double(minl - K + 1);
            bounded = kd_lb > (tasks_smem ? s_cutoff[t] : L.tasks[t].cutoff);
          }
        }
      }
    }
    const bool need = valid && !skip && kp.use_kmers && !bounded;
    {
      const uint32_t needm = __ballot_sync(FULL, need);  // profiles this chunk reads
      if (lane == 0 && needm) atomicAdd(&L.queue_counts[5], uint32_t(__popc(needm)));
    }
    uint32_t mydot = 0, myovf = 0;
    uint32_t todo = __ballot_sync(FULL, need);
    if constexpr (K >= 8) {
      // Sparse screen (src/kmers.rs:280-308): only k-mers present in both
      // sequences contribute min(count, count); one item at a time, each lane
      // takes raw entries and finds their index in the center's ascending list.
      while (todo) {
        const int j = __ffs(todo) - 1;
        todo &= todo - 1;
        const uint32_t gj = __shfl_sync(FULL, g, j), cj = __shfl_sync(FULL, c, j);
        const uint32_t na = L.pool.knum[gj], nc = L.pool.knum[cj];
        const uint16_t* ai = L.pool.kidx + L.pool.off[gj];
        const uint8_t* ac = L.pool.kcnt + L.pool.off[gj];
        const uint16_t* ci = L.pool.kidx + L.pool.off[cj];
        const uint8_t* cc = L.pool.kcnt + L.pool.off[cj];
        uint32_t dot = 0;
        for (uint32_t e = lane; e < na; e += 32) {
          const uint16_t x = ai[e];
          uint32_t lo = 0, hi = nc;
          while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (ci[mid] < x) lo = mid + 1;
            else hi = mid;
          }
          if (lo < nc && ci[lo] == x) dot += min(unsigned(ac[e]), unsigned(cc[lo]));
        }
        dot = __reduce_add_sync(FULL, dot);
        if (lane == j) mydot = dot;
      }
    } else {
      // center profile of the chunk's first needing item, kept in registers
      uint32_t cur_c = 0xffffffffu;
      uint4 cv[CENTER_REGS ? VPL : 1];
      (void)cur_c;
      while (todo) {
        int js[NB];
  #pragma unroll
        for (int q = 0; q < NB; ++q) {
          js[q] = -1;
          if (todo) {
            js[q] = __ffs(todo) - 1;
            todo &= todo - 1;
          }
        }
        uint32_t gq[NB], cq[NB];
  #pragma unroll
        for (int q = 0; q < NB; ++q) {
          const int src = js[q] < 0 ? 0 : js[q];
          gq[q] = __shfl_sync(FULL, g, src);
          cq[q] = __shfl_sync(FULL, c, src);
        }
        constexpr int RV = CENTER_REGS ? VPL : 1;
        uint4 rv[NB][RV];
        if (CENTER_REGS) {
  #pragma unroll
          for (int q = 0; q < NB; ++q) {
            if (js[q] >= 0) {
              const uint4* pg = reinterpret_cast<const uint4*>(kmer8 + size_t(gq[q]) * size_t(NK16) * 16);
  #pragma unroll
              for (int v = 0; v < RV; ++v) {
                const int idx = lane + 32 * v;
                rv[q][v] = idx < NK16 ? __ldcs(pg + idx) : make_uint4(0, 0, 0, 0);
              }
            }
          }
        }
  #pragma unroll
        for (int q = 0; q < NB; ++q) {
          if (js[q] < 0) continue;
          const uint4* pc = reinterpret_cast<const uint4*>(kmer8 + size_t(cq[q]) * size_t(NK16) * 16);
          const uint4* pg = reinterpret_cast<const uint4*>(kmer8 + size_t(gq[q]) * size_t(NK16) * 16);
          if (CENTER_REGS && cq[q] != cur_c) {
  #pragma unroll
            for (int v = 0; v < VPL; ++v) {
              const int idx = lane + 32 * v;
              cv[CENTER_REGS ? v : 0] = idx < NK16 ? __ldg(pc + idx) : make_uint4(0, 0, 0, 0);
            }
            cur_c = cq[q];
          }
          uint32_t dot = 0;
  #pragma unroll 4
          for (int v = 0; v < VPL; ++v) {
            const int idx = lane + 32 * v;
            const uint4 a = CENTER_REGS ? cv[CENTER_REGS ? v : 0] : (idx < NK16 ? __ldg(pc + idx) : make_uint4(0, 0, 0, 0));
            const uint4 b2 = CENTER_REGS ? rv[q][CENTER_REGS ? v : 0] : (idx < NK16 ? __ldcs(pg + idx) : make_uint4(0, 0, 0, 0));
            const uint32_t m0 = __vminu4(a.x, b2.x), m1 = __vminu4(a.y, b2.y), m2 = __vminu4(a.z, b2.z),
                           m3 = __vminu4(a.w, b2.w);
            dot = __dp4a(m0, 0x01010101u, dot);
            dot = __dp4a(m1, 0x01010101u, dot);
            dot = __dp4a(m2, 0x01010101u, dot);
            dot = __dp4a(m3, 0x01010101u, dot);
          }
          dot = __reduce_add_sync(FULL, dot);
          if (lane == js[q]) mydot = dot;
        }
      }
    }
    // kmer_dist8 returns -1 (and the reference falls back to the exact u16
    // distance, src/nwalign.rs:1270-1277) when some k-mer's min count is 255,
    // which needs a saturated count in both profiles. Whenever both have one,
    // the exact dot is taken instead: it equals the u8 dot when no min
    // saturates, so the result is the reference's in every case. One item at a
    // time by the whole warp: each window of the raw contributes 1 when its rank
    // among equal windows of the raw is below the center's count of that k-mer.
    const bool maybe_ovf = need && L.pool.sat[g] && L.pool.sat[c];
    (void)myovf;
    uint32_t ovf_mask = __ballot_sync(FULL, maybe_ovf);
    while (ovf_mask) {
      const int j = __ffs(ovf_mask) - 1;
      ovf_mask &= ovf_mask - 1;
      const uint32_t gj = __shfl_sync(FULL, g, j), cj = __shfl_sync(FULL, c, j);
      const int lc = int(L.pool.len[cj]), lg = int(L.pool.len[gj]);
      const uint8_t* sc = L.pool.seq + L.pool.off[cj];
      const uint8_t* sg = L.pool.seq + L.pool.off[gj];
      uint32_t exact = 0;
      for (int p = lane; p + K <= lg; p += 32) {
        int x = 0;
        for (int q = 0; q < K; ++q) x = x * 4 + int(sg[p + q]) - 1;
        uint32_t rank = 0, cnt = 0;
        for (int p2 = 0; p2 < p; ++p2) {
          int y = 0;
          for (int q = 0; q < K; ++q) y = y * 4 + int(sg[p2 + q]) - 1;
          rank += (y == x);
        }
        for (int p2 = 0; p2 + K <= lc; ++p2) {
          int y = 0;
          for (int q = 0; q < K; ++q) y = y * 4 + int(sc[p2 + q]) - 1;
          cnt += (y == x);
        }
        exact += rank < cnt ? 1u : 0u;
      }
      exact = __reduce_add_sync(FULL, exact);
      if (lane == j) mydot = exact;
    }
    // the dot becomes the raw's pivot when it beats the one it has
    if (pivot && need && pivot_raw) {
      const uint32_t pc = L.pool.piv_cl[g];
      if (pc == kNoPivot || mydot > L.pool.piv_dot[g]) {
        L.pool.piv_dot[g] = mydot;
        L.pool.piv_cl[g] = ccl;
      }
    }
    bool pass = false;
    if (valid) {
      if (kp.lambda32) L.pool.res_loglam32[g] = -INFINITY;
      if (bounded) {
        L.pool.res_lambda[g] = 0.0;
        L.pool.res_ham[g] = 0xffffffffu;
        L.pool.res_status[g] = ST_SHROUDED;
      } else if (skip) {
        L.pool.res_lambda[g] = 0.0;
        L.pool.res_ham[g] = 0xffffffffu;
        L.pool.res_status[g] = ST_SKIPPED;
      } else {
        double kdist = 0.0;
        bool shroud = false;
        if (kp.use_kmers) {
          const int lc = int(L.pool.len[c]), lg = int(L.pool.len[g]);
          const int minl = lc < lg ? lc : lg;
          kdist = 1.0 - double(mydot) / double(minl - K + 1);
          shroud = kdist > (tasks_smem ? s_cutoff[t] : L.tasks[t].cutoff);
        }
        if (shroud) {
          L.pool.res_lambda[g] = 0.0;
          L.pool.res_ham[g] = 0xffffffffu;
          L.pool.res_status[g] = ST_SHROUDED;
        } else {
          L.pool.res_lambda[g] = kdist;
          pass = true;
        }
      }
    }
    const uint32_t pm = __ballot_sync(FULL, pass);
    if (pm) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(&L.queue_counts[4], uint32_t(__popc(pm)));
      base = __shfl_sync(FULL, base, 0);
      if (pass) L.queue_pass[base + __popc(pm & ((1u << lane) - 1u))] = item;
    }
  }
}

// ---------------------------------------------------------------------------
// K4: vectorized (compressed anti-diagonal) aligner
// ---------------------------------------------------------------------------
struct VecSmem {
  uint8_t* s1;
  uint8_t* s2;
  int16_t* rows;  // 3 x ncol rolling slots
  int16_t* diag;
  uint8_t* prow;
  uint8_t* stage;
  uint8_t* tcode;
  uint16_t* fidx;  // followed by lmax bytes for the raw's staged qualities (vec_qual)
};

__device__ __forceinline__ int sat_sub1(int v) { return v == 0 ? 0 : v - 1; }

// Aligns s1_in (center) against s2_in (raw). On success fills tcode[] for the
// raw positions and returns the substitution count in *ham. With dbg0/dbg1 the
// alignment rows are written in traceback (reversed) order for the tests.
__device__ bool vec_align_warp(int lane, const uint8_t* g1, int l1, const uint8_t* g2, int l2, int16_t match,
                               int16_t mismatch, int16_t gap, int16_t egp, int band_in, const VecSmem& S,
                               uint8_t* pmat, int ncol_bound, int nrow_bound, uint32_t* ham_out,
                               uint32_t* err_word, uint8_t* dbg0, uint8_t* dbg1, uint32_t* dbg_len) {
  const bool swap = l1 > l2;
  const int len1 = swap ? l2 : l1, len2 = swap ? l1 : l2;
  {
    const uint8_t* a = swap ? g2 : g1;
    const uint8_t* b = swap ? g1 : g2;
    for (int p = lane; p < len1; p += 32) S.s1[p] = a[p];
    for (int p = lane; p < len2; p += 32) S.s2[p] = b[p];
  }
  const int band = band_in < 0 ? len2 : band_in;
  const int start_col = 1 + (min(band, len1) + 1) / 2;
  const int ncol = 2 + start_col + min(band + len2 - len1, len2) / 2;
  const int nrow = len1 + len2 + 1;
  if (ncol > ncol_bound || nrow > nrow_bound || ncol < 4) {
    if (lane == 0) atomicOr(err_word, DERR_GEOMETRY);
    return false;
  }
  int16_t min_score = min(min(min(mismatch, gap), match), int16_t(0));
  const int16_t fill = int16_t(uint16_t(uint16_t(0x8000u) - uint16_t(min_score)));
  const int lfl = 1 + min(band, len1);
  const int tfl = 1 + min(band + len2 - len1, len2);
  for (int c = lane; c < 3 * ncol; c += 32) S.rows[c] = 0;
  for (int c = lane; c < ncol; c += 32) S.diag[c] = 0;
  for (int c = lane; c < 2 * ncol; c += 32) pmat[c] = 0;
  __syncwarp();
  auto left_col = [&](int row) { int a = start_col - 1, b = (row - 1) / 2; return a > b ? a - b : 0; };
  auto top_col = [&](int row) { return start_col + row / 2; };
  if (lane == 0) {
    for (int row = 0; row < 2; ++row) {
      int16_t* slot = S.rows + row * ncol;
      slot[0] = fill;
      slot[1] = fill;
      slot[ncol - 2] = fill;
      slot[ncol - 1] = fill;
      if (row == 0) {
        slot[start_col] = 0;
      } else {
        if (row < lfl) {
          slot[left_col(row)] = egp;
          pmat[row * ncol + left_col(row)] = 3;
        }
        if (row < tfl) {
          slot[top_col(row)] = egp;
          pmat[row * ncol + top_col(row)] = 2;
        }
      }
    }
    pmat[start_col] = 0;
  }
  __syncwarp();
  int16_t row_free = egp;
  int sl0 = 0, sl1 = 1, sl2 = 2;
  int col_min = start_col, col_max = start_col, i_max = 0, j_min = 0;
  bool even = true, recalc_left = false, recalc_right = false;
  const int band_mod2 = band % 2;
  const int top_limit = min(band + len2 - len1, len2);
  const int full_band = band + len2 - len1;
  for (int row = 2; row <= len1 + len2; ++row) {
    if (!(col_max >= col_min && col_max < ncol)) {
      if (lane == 0) atomicOr(err_word, DERR_BAND_RANGE);
      return false;
    }
    const int n = col_max - col_min + 1;
    row_free = sadd16(row_free, egp);
    int16_t* cur = S.rows + sl2 * ncol;
    const int16_t* prev = S.rows + sl1 * ncol;
    const int16_t* prev2 = S.rows + sl0 * ncol;
    for (int c = lane; c < ncol; c += 32) S.prow[c] = 0;
    __syncwarp();
    if (lane == 0) {
      cur[0] = fill;
      cur[1] = fill;
      cur[ncol - 2] = fill;
      cur[ncol - 1] = fill;
      if (row < lfl) {
        cur[left_col(row)] = row_free;
        S.prow[left_col(row)] = 3;
      }
      if (row < tfl) {
        cur[top_col(row)] = row_free;
        S.prow[top_col(row)] = 2;
      }
    }
    __syncwarp();
    {
      int k_lo = i_max - len1 + 1;
      k_lo = k_lo < 0 ? 0 : (k_lo > n ? n : k_lo);
      int k_hi = min(i_max + 1, len2 - j_min);
      k_hi = k_hi < 0 ? 0 : (k_hi > n ? n : k_hi);
      k_hi = max(k_hi, k_lo);
      for (int k = lane; k < n; k += 32) {
        const int c = col_min + k;
        int16_t v;
        if (k < k_lo || k >= k_hi) v = fill;
        else v = (S.s1[i_max - k] == S.s2[j_min + k]) ? match : mismatch;
        S.diag[c] = sadd16(prev2[c], v);
      }
    }
    __syncwarp();
    const int eo = even ? 1 : 0;
    const int left_off = col_min - eo, up_off = col_min + 1 - eo;
    if (left_off < 0 || up_off + n > ncol) {
      if (lane == 0) atomicOr(err_word, DERR_BAND_RANGE);
      return false;
    }
    for (int k = lane; k < n; k += 32) {
      int16_t l = sadd16(prev[left_off + k], gap);
      int16_t u = sadd16(prev[up_off + k], gap);
      int16_t dg = S.diag[col_min + k];
      int16_t e;
      uint8_t pe;
      if (swap) {
        if (l >= u) { e = l; pe = 2; } else { e = u; pe = 3; }
      } else {
        if (u >= l) { e = u; pe = 3; } else { e = l; pe = 2; }
      }
      if (dg > e) { e = dg; pe = 1; }
      cur[col_min + k] = e;
      S.prow[col_min + k] = pe;
    }
    __syncwarp();
    if (row == min(band, len1)) {
      col_min = sat_sub1(col_min);
      i_max += 1;
      j_min -= 1;
    }
    if (row == min(band + len2 - len1, len2)) col_max += 1;
    if (egp > gap) {
      if (recalc_left && lane == 0) {
        int16_t d_free = sadd16(prev[left_off], egp);
        int16_t cv = cur[col_min];
        uint8_t pc = S.prow[col_min];
        if (d_free > cv) {
          cur[col_min] = d_free;
          S.prow[col_min] = 2;
        } else if (!(d_free != cv || (!swap && pc != 1) || (swap && pc == 2))) {
          S.prow[col_min] = 2;
        }
      }
      if (i_max == len1 - 1) recalc_left = true;
      if (recalc_right) {
        const int idx = up_off + col_max - col_min;
        if (idx < 0 || idx >= ncol || col_max >= ncol) {
          if (lane == 0) atomicOr(err_word, DERR_BAND_RANGE);
          return false;
        }
        if (lane == 0) {
          int16_t d_free = sadd16(prev[idx], egp);
          int16_t cv = cur[col_max];
          uint8_t pc = S.prow[col_max];
          if (d_free > cv) {
            cur[col_max] = d_free;
            S.prow[col_max] = 3;
          } else if (!(d_free != cv || (!swap && pc == 3) || (swap && pc != 1))) {
            S.prow[col_max] = 3;
          }
        }
      }
      if ((row + 1) / 2 + col_max - start_col == len2) recalc_right = true;
    }
    __syncwarp();
    for (int c = lane; c < ncol; c += 32) pmat[size_t(row) * ncol + c] = S.prow[c];
    if (row < band && row < len1) {
      if (even) col_min = sat_sub1(col_min);
      i_max += 1;
    } else if (i_max < len1 - 1) {
      if (band_mod2 == 0) {
        if (even) j_min += 1;
        else i_max += 1;
      } else if (even) {
        col_min = sat_sub1(col_min);
        i_max += 1;
      } else {
        col_min += 1;
        j_min += 1;
      }
    } else {
      if (!even) col_min += 1;
      j_min += 1;
    }
    if (row < top_limit) {
      if (!even) col_max += 1;
    } else if ((row + 1) / 2 + col_max - start_col < len2) {
      if (full_band % 2 == 0) {
        if (even) col_max = sat_sub1(col_max);
        else col_max += 1;
      }
    } else if (even) {
      col_max = sat_sub1(col_max);
    }
    const int t = sl0;
    sl0 = sl1;
    sl1 = sl2;
    sl2 = t;
    even = !even;
  }
  __syncwarp();
  // Traceback (src/nwalign.rs:1090-1139), staged through shared memory in row chunks.
  const uint8_t* raw = swap ? S.s1 : S.s2;
  const int lraw = swap ? len1 : len2;
  for (int p = lane; p < lraw; p += 32) S.tcode[p] = uint8_t(kUnaligned | ((unsigned(raw[p]) - 1u) * 5u));
  const int rps = kStageBytes / ncol;
  int slo = 0x7fffffff;
  int i = len1, j = len2;
  uint32_t ham = 0, alen = 0;
  bool ok = true;
  __syncwarp();
  while (i > 0 || j > 0) {
    const int cs = 2 * start_col + j - i;
    if (cs < 0) { ok = false; break; }
    const int col = cs / 2;
    const int r = i + j;
    if (r < slo) {
      const int nlo = max(0, r - rps + 1);
      __syncwarp();
      const int nb = (r - nlo + 1) * ncol;
      const uint8_t* src = pmat + size_t(nlo) * ncol;
      for (int x = lane; x < nb; x += 32) S.stage[x] = src[x];
      __syncwarp();
      slo = nlo;
    }
    const uint8_t v = S.stage[(r - slo) * ncol + col];
    if (v == 1 && i > 0 && j > 0) {
      const uint8_t a = S.s1[i - 1], b = S.s2[j - 1];
      const int rp = swap ? i - 1 : j - 1;
      const uint8_t cn = swap ? b : a, rn = swap ? a : b;
      if (lane == 0) S.tcode[rp] = uint8_t((unsigned(cn) - 1u) * 4u + (unsigned(rn) - 1u));
      ham += (a != b) ? 1u : 0u;
      if (dbg0 && lane == 0) {
        dbg0[alen] = swap ? b : a;
        dbg1[alen] = swap ? a : b;
      }
      --i;
      --j;
    } else if (v == 2 && j > 0) {
      if (dbg0 && lane == 0) {
        dbg0[alen] = swap ? S.s2[j - 1] : uint8_t('-');
        dbg1[alen] = swap ? uint8_t('-') : S.s2[j - 1];
      }
      --j;
    } else if (v == 3 && i > 0) {
      if (dbg0 && lane == 0) {
        dbg0[alen] = swap ? uint8_t('-') : S.s1[i - 1];
        dbg1[alen] = swap ? S.s1[i - 1] : uint8_t('-');
      }
      --i;
    } else {
      ok = false;
      break;
    }
    ++alen;
  }
  __syncwarp();
  if (!ok) {
    if (lane == 0) atomicOr(err_word, DERR_TRACEBACK);
    return false;
  }
  if (dbg_len && lane == 0) *dbg_len = alen;
  *ham_out = ham;
  return true;
}

__device__ VecSmem carve_vec(unsigned char* base, int lmax, int ncol_bound) {
  VecSmem S;
  size_t o = 0;
  auto take = [&](size_t bytes) { unsigned char* p = base + o; o += (bytes + 15) & ~size_t(15); return p; };
  S.s1 = take(lmax + 2 * kSeqPad) + kSeqPad;  // guard bytes before and after
  S.s2 = take(lmax + 2 * kSeqPad) + kSeqPad;
  S.rows = reinterpret_cast<int16_t*>(take(size_t(3) * ncol_bound * 2));
  S.diag = reinterpret_cast<int16_t*>(take(size_t(ncol_bound) * 2));
  S.prow = take(ncol_bound);
  S.stage = take(kStageBytes);
  S.tcode = take(lmax);
  S.fidx = reinterpret_cast<uint16_t*>(take(size_t(lmax) * 2));
  return S;
}
__device__ __forceinline__ uint8_t* vec_qual(const VecSmem& S, int lmax) {
  return reinterpret_cast<uint8_t*>(S.fidx) + align16(size_t(lmax) * 2);
}

// Copies a (n bytes), b (m bytes) and, when q is given, q (m bytes) from
// global to shared memory with every load of a 256-position block issued
// before the first store, so a pair's inputs arrive in one round trip.
__device__ __forceinline__ void stage3(int lane, const uint8_t* __restrict__ a, int n, uint8_t* da,
                                       const uint8_t* __restrict__ b, int m, uint8_t* db,
                                       const uint8_t* __restrict__ q, uint8_t* dq) {
  const int top = n > m ? n : m;
  for (int base = 0; base < top; base += 256) {
    uint8_t va[8], vb[8], vq[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int p = base + lane + 32 * i;
      va[i] = p < n ? __ldg(a + p) : uint8_t(0);
      vb[i] = p < m ? __ldg(b + p) : uint8_t(0);
      vq[i] = (q && p < m) ? __ldg(q + p) : uint8_t(0);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int p = base + lane + 32 * i;
      if (p < n) da[p] = va[i];
      if (p < m) {
        db[p] = vb[i];
        if (q) dq[p] = vq[i];
      }
    }
  }
}


// Traceback through the pointer bit-planes of the register aligners
// (src/nwalign.rs:1090-1139). With planes_smem the planes of every row are
// already in S.stage; otherwise they are read from the per-warp scratch.
template <int M>
__device__ bool reg_traceback(int lane, bool swap, int len1, int len2, int start_col, int ncol, const VecSmem& S,
                              const uint32_t* pscr, bool planes_smem, uint32_t* ham_out, uint32_t* err_word,
                              uint8_t* dbg0, uint8_t* dbg1, uint32_t* dbg_len) {
  bool ok = true;
  // Traceback through the bit-planes. A window of up to 64 rows is staged in
  // shared memory; lane t tests whether the t-th next step is diagonal (cell
  // (i-t, j-t): row r-2t, same compressed column), so a run of f diagonal steps
  // is taken at once, each lane doing one. A gap step is taken singly.
  const uint8_t* raw = swap ? S.s1 : S.s2;
  const int lraw = swap ? len1 : len2;
  for (int p = lane; p < lraw; p += 32) S.tcode[p] = uint8_t(kUnaligned | ((unsigned(raw[p]) - 1u) * 5u));
  uint32_t* stage = reinterpret_cast<uint32_t*>(S.stage);
  int slo = planes_smem ? 0 : 0x7fffffff;  // planes already in shared memory: no staging
  int i = len1, j = len2;
  uint32_t ham = 0, alen = 0;
  __syncwarp();
  while (i > 0 || j > 0) {
    const int cs = 2 * start_col + j - i;
    if (cs < 0 || cs / 2 >= ncol) { ok = false; break; }
    const int col = cs / 2;
    const int r = i + j;
    if (!planes_smem && (r < slo || (r - slo < 16 && slo > 0))) {
      const int nlo = max(0, r - 63);
      __syncwarp();
      const int nw = (r - nlo + 1) * 2 * M;
      const uint32_t* src = pscr + size_t(nlo) * (2 * M);
      for (int x = lane; x < nw; x += 32) stage[x] = src[x];
      __syncwarp();
      slo = nlo;
    }
    const int rr = r - 2 * lane;
    const bool inwin = rr >= slo;
    int v = 0;
    if (inwin) {
      const uint32_t* wrow = stage + (rr - slo) * (2 * M) + 2 * (col >> 5);
      const int bit = col & 31;
      v = int((wrow[0] >> bit) & 1u) | (int((wrow[1] >> bit) & 1u) << 1);
    }
    const bool diag = inwin && v == 1 && i - lane > 0 && j - lane > 0;
    const uint32_t nd = __ballot_sync(FULL, !diag);
    const int f = nd ? __ffs(nd) - 1 : 32;
    if (f > 0) {
      bool mm = false;
      if (lane < f) {
        const uint8_t a = S.s1[i - 1 - lane], b = S.s2[j - 1 - lane];
        const int rp = (swap ? i : j) - 1 - lane;
        const uint8_t cn = swap ? b : a, rn = swap ? a : b;
        S.tcode[rp] = uint8_t((unsigned(cn) - 1u) * 4u + (unsigned(rn) - 1u));
        mm = a != b;
        if (dbg0) {
          dbg0[alen + lane] = swap ? b : a;
          dbg1[alen + lane] = swap ? a : b;
        }
      }
      ham += __popc(__ballot_sync(FULL, mm));
      i -= f;
      j -= f;
      alen += uint32_t(f);
      continue;
    }
    const int v0 = __shfl_sync(FULL, v, 0);
    if (v0 == 2 && j > 0) {
      if (dbg0 && lane == 0) {
        dbg0[alen] = swap ? S.s2[j - 1] : uint8_t('-');
        dbg1[alen] = swap ? uint8_t('-') : S.s2[j - 1];
      }
      --j;
    } else if (v0 == 3 && i > 0) {
      if (dbg0 && lane == 0) {
        dbg0[alen] = swap ? uint8_t('-') : S.s1[i - 1];
        dbg1[alen] = swap ? S.s1[i - 1] : uint8_t('-');
      }
      --i;
    } else {
      ok = false;
      break;
    }
    ++alen;
  }
  __syncwarp();
  if (!ok) {
    if (lane == 0) atomicOr(err_word, DERR_TRACEBACK);
    return false;
  }
  if (dbg_len && lane == 0) *dbg_len = alen;
  *ham_out = ham;
  return true;
}

// Register form of the same aligner for compressed widths up to 32*M columns:
// lane l owns columns l + 32m; the three rolling rows live in registers
// (r3 = the slot being overwritten, still holding row-3 values, as in the
// reference's rotating buffer), left/up neighbours come from warp shuffles and
// each row's 2-bit pointers are two ballot bit-planes per 32 columns, buffered
// 32 rows per flush to the per-warp scratch.
template <int M>
__device__ bool vec_align_reg(int lane, const uint8_t* g1, int l1, const uint8_t* g2, int l2, int16_t match16,
                              int16_t mismatch16, int16_t gap16, int16_t egp16, int band_in, const VecSmem& S,
                              uint32_t* pscr, int nrow_bound, uint32_t* ham_out, uint32_t* err_word, uint8_t* dbg0,
                              uint8_t* dbg1, uint32_t* dbg_len) {
  const bool swap = l1 > l2;
  const int len1 = swap ? l2 : l1, len2 = swap ? l1 : l2;
  {
    const uint8_t* a = swap ? g2 : g1;
    const uint8_t* b = swap ? g1 : g2;
    for (int p = lane; p < len1; p += 32) S.s1[p] = a[p];
    for (int p = lane; p < len2; p += 32) S.s2[p] = b[p];
  }
  const int band = band_in < 0 ? len2 : band_in;
  const int start_col = 1 + (min(band, len1) + 1) / 2;
  const int ncol = 2 + start_col + min(band + len2 - len1, len2) / 2;
  const int nrow = len1 + len2 + 1;
  if (ncol > 32 * M || nrow > nrow_bound || ncol < 4) {
    if (lane == 0) atomicOr(err_word, DERR_GEOMETRY);
    return false;
  }
  // i16 scores held in int lanes; every add saturates to the i16 range exactly
  // as i16::saturating_add does.
  const int match = match16, mismatch = mismatch16, gap = gap16, egp = egp16;
  const int min_score = min(min(min(mismatch, gap), match), 0);
  const int fill = int(int16_t(uint16_t(uint16_t(0x8000u) - uint16_t(min_score))));
  auto sat = [](int v) { return max(-32768, min(32767, v)); };
  const int lfl = 1 + min(band, len1);
  const int tfl = 1 + min(band + len2 - len1, len2);
  const int edge_rows = max(lfl, tfl);
  auto left_col = [&](int row) { int a = start_col - 1, b = (row - 1) / 2; return a > b ? a - b : 0; };
  auto top_col = [&](int row) { return start_col + row / 2; };
  int r3[M], r2[M], r1[M];
  bool sentinel[M];
  uint32_t pbuf[2 * M];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int c = lane + 32 * m;
    sentinel[m] = c == 0 || c == 1 || c == ncol - 2 || c == ncol - 1;
    int v0 = sentinel[m] ? fill : 0;
    if (c == start_col) v0 = 0;
    int v1 = sentinel[m] ? fill : 0;
    uint32_t c1 = 0;
    if (1 < lfl && c == left_col(1)) { v1 = egp; c1 = 3; }
    if (1 < tfl && c == top_col(1)) { v1 = egp; c1 = 2; }
    r3[m] = 0;
    r2[m] = v0;
    r1[m] = v1;
    const uint32_t w0 = __ballot_sync(FULL, c1 & 1), w1 = __ballot_sync(FULL, (c1 >> 1) & 1);
    pbuf[2 * m] = lane == 1 ? w0 : 0u;
    pbuf[2 * m + 1] = lane == 1 ? w1 : 0u;
  }
  __syncwarp();
  int row_free = egp;
  int col_min = start_col, col_max = start_col, i_max = 0, j_min = 0;
  bool recalc_left = false, recalc_right = false;
  const int band_mod2 = band % 2;
  const int top_limit = min(band + len2 - len1, len2);
  const int full_band = band + len2 - len1;
  const int last = len1 + len2;
  const int bt_row1 = min(band, len1);
  const int bt_row2 = min(band + len2 - len1, len2);
  const bool fb_even = full_band % 2 == 0;
  const bool do_recalc = egp > gap;
  bool bad = false;
  // Rows go in even/odd pairs so that the anti-diagonal parity is known at
  // compile time: an even row reads its left neighbour from column c-1 and its
  // up neighbour from column c of the previous row, an odd row from c and c+1.
  // A corrupted band state cannot address memory out of bounds (sequence reads
  // are range-tested, lane indexes are masked), so it is checked once per pair.
  for (int row0 = 2; row0 <= last; row0 += 2) {
#pragma unroll
    for (int ph = 0; ph < 2; ++ph) {
      const int row = row0 + ph;
      if (ph == 1 && row > last) break;
      const bool E = ph == 0;
      const int n = col_max - col_min + 1;
      const int eo = E ? 1 : 0;
      const int left_off = col_min - eo, up_off = col_min + 1 - eo;
      bad |= (col_max < col_min) | (col_max >= ncol) | (left_off < 0) | (up_off + n > ncol);
      row_free = sat(row_free + egp);
      int lcol = -1, tcol = -1;
      if (row < edge_rows) {  // ends-free edge cells exist only near the start
        lcol = row < lfl ? left_col(row) : -1;
        tcol = row < tfl ? top_col(row) : -1;
      }
      int cur[M];
      uint32_t cc[M];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        int nb;  // the previous row's value in the column this parity reads besides c
        if (E) {
          const int a = __shfl_up_sync(FULL, r1[m], 1);
          const int a31 = m > 0 ? __shfl_sync(FULL, r1[m > 0 ? m - 1 : 0], 31) : 0;
          nb = lane == 0 ? a31 : a;  // column c-1
        } else {
          const int b = __shfl_down_sync(FULL, r1[m], 1);
          const int b0 = (m + 1 < M) ? __shfl_sync(FULL, r1[m + 1 < M ? m + 1 : m], 0) : 0;
          nb = lane == 31 ? b0 : b;  // column c+1
        }
        const int c = lane + 32 * m;
        int v = sentinel[m] ? fill : r3[m];
        uint32_t code = 0;
        if (c == lcol) { v = row_free; code = 3; }
        if (c == tcol) { v = row_free; code = 2; }
        const int k = c - col_min;
        if ((unsigned)k < (unsigned)n) {
          const int si = i_max - k, sj = j_min + k;
          int sc = fill;
          if ((unsigned)si < (unsigned)len1 && (unsigned)sj < (unsigned)len2)
            sc = (S.s1[si] == S.s2[sj]) ? match : mismatch;
          const int dg = sat(r2[m] + sc);
          const int l = sat((E ? nb : r1[m]) + gap);
          const int u = sat((E ? r1[m] : nb) + gap);
          int e;
          uint32_t pe;
          if (swap) {
            const bool lw = l >= u;
            e = lw ? l : u;
            pe = lw ? 2u : 3u;
          } else {
            const bool uw = u >= l;
            e = uw ? u : l;
            pe = uw ? 3u : 2u;
          }
          const bool dw = dg > e;
          v = dw ? dg : e;
          code = dw ? 1u : pe;
        }
        cur[m] = v;
        cc[m] = code;
      }
      {  // band transition at the wedge boundaries (src/nwalign.rs:980-987)
        const bool t1 = row == bt_row1;
        col_min = t1 ? sat_sub1(col_min) : col_min;
        i_max += t1 ? 1 : 0;
        j_min -= t1 ? 1 : 0;
        col_max += (row == bt_row2) ? 1 : 0;
      }
      if (do_recalc) {
        if (recalc_left) {
          int pv = r1[0];
#pragma unroll
          for (int m = 1; m < M; ++m)
            if ((left_off >> 5) == m) pv = r1[m];
          pv = __shfl_sync(FULL, pv, left_off & 31);
          const int d_free = sat(pv + egp);
#pragma unroll
          for (int m = 0; m < M; ++m) {
            if (lane + 32 * m == col_min) {
              const int cv = cur[m];
              const uint32_t pc = cc[m];
              if (d_free > cv) {
                cur[m] = d_free;
                cc[m] = 2;
              } else if (!(d_free != cv || (!swap && pc != 1) || (swap && pc == 2))) {
                cc[m] = 2;
              }
            }
          }
        }
        if (i_max == len1 - 1) recalc_left = true;
        if (recalc_right) {
          const int idx = up_off + col_max - col_min;
          bad |= idx < 0 || idx >= ncol || col_max >= ncol;
          int pv = r1[0];
#pragma unroll
          for (int m = 1; m < M; ++m)
            if ((idx >> 5) == m) pv = r1[m];
          pv = __shfl_sync(FULL, pv, idx & 31);
          const int d_free = sat(pv + egp);
#pragma unroll
          for (int m = 0; m < M; ++m) {
            if (lane + 32 * m == col_max) {
              const int cv = cur[m];
              const uint32_t pc = cc[m];
              if (d_free > cv) {
                cur[m] = d_free;
                cc[m] = 3;
              } else if (!(d_free != cv || (!swap && pc == 3) || (swap && pc != 1))) {
                cc[m] = 3;
              }
            }
          }
        }
        if ((row + 1) / 2 + col_max - start_col == len2) recalc_right = true;
      }
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const uint32_t w0 = __ballot_sync(FULL, cc[m] & 1u), w1 = __ballot_sync(FULL, cc[m] & 2u);
        if (lane == (row & 31)) {
          pbuf[2 * m] = w0;
          pbuf[2 * m + 1] = w1;
        }
      }
      if ((row & 31) == 31 || row == last) {
        const int base = row & ~31;
        if (base + lane <= row) {
          uint32_t* dst = pscr + size_t(base + lane) * (2 * M);
#pragma unroll
          for (int w = 0; w < 2 * M; ++w) dst[w] = pbuf[w];
        }
      }
      {  // advance the band for the next anti-diagonal (src/nwalign.rs:1028-1079)
        const bool regA = row < band && row < len1;
        const bool regB = !regA && i_max < len1 - 1;
        const int cm = col_min, im = i_max, jm = j_min;
        const int cmA = E ? sat_sub1(cm) : cm, imA = im + 1, jmA = jm;
        int cmB, imB, jmB;
        if (band_mod2 == 0) {
          cmB = cm;
          imB = E ? im : im + 1;
          jmB = E ? jm + 1 : jm;
        } else {
          cmB = E ? sat_sub1(cm) : cm + 1;
          imB = E ? im + 1 : im;
          jmB = E ? jm : jm + 1;
        }
        const int cmC = E ? cm : cm + 1, imC = im, jmC = jm + 1;
        col_min = regA ? cmA : (regB ? cmB : cmC);
        i_max = regA ? imA : (regB ? imB : imC);
        j_min = regA ? jmA : (regB ? jmB : jmC);
        const int cx = col_max;
        const bool rt = row < top_limit;
        const bool mid = !rt && ((row + 1) / 2 + cx - start_col < len2);
        const int cxA = E ? cx : cx + 1;
        const int cxB = fb_even ? (E ? sat_sub1(cx) : cx + 1) : cx;
        const int cxC = E ? sat_sub1(cx) : cx;
        col_max = rt ? cxA : (mid ? cxB : cxC);
      }
#pragma unroll
      for (int m = 0; m < M; ++m) {
        r3[m] = r2[m];
        r2[m] = r1[m];
        r1[m] = cur[m];
      }
    }
    if (bad) break;
  }
  bool ok = !bad;
  if (!ok) {
    if (lane == 0) atomicOr(err_word, DERR_BAND_RANGE);
    return false;
  }
  if (last < 2) {  // rows 0/1 only: flush the buffered words
    if (lane <= last) {
      uint32_t* dst = pscr + size_t(lane) * (2 * M);
#pragma unroll
      for (int w = 0; w < 2 * M; ++w) dst[w] = pbuf[w];
    }
  }
  __syncwarp();
  return reg_traceback<M>(lane, swap, len1, len2, start_col, ncol, S, pscr, false, ham_out, err_word, dbg0, dbg1,
                          dbg_len);
}

// Fast register form: the cells, pointers and band bookkeeping of
// vec_align_reg, computed with fewer instructions and a shorter dependency
// chain per anti-diagonal. Bit-identical results rest on three facts:
//  * With gap <= 0, end gap <= 0 and P = max(match, mismatch, 0), a value on
//    anti-diagonal r is at most P*floor(r/2) (each row adds at most P over the
//    row two back, and nothing else increases a value), so when
//    P*((len1+len2)/2 + 1) <= 32767 no sum can pass 32767 and i16::saturating_add
//    reduces to max(a + b, -32768), one DPX add-max.
//  * The swap tie rule is a template parameter.
//  * The band state of anti-diagonal r+1 and its sequence bytes are formed
//    before the cells of r, so bookkeeping and shared-memory loads overlap the
//    shuffle -> add -> max chain that carries the recurrence.
// The caller has copied the (swapped) sequences to S.s1/S.s2. The pointer
// bit-planes go straight to S.stage when every row fits there (PS),
// else to the per-warp global scratch in 32-row flushes.
template <int M, bool SWAP, bool PS>
__device__ bool vec_align_fast(int lane, int len1, int len2, int match, int mismatch, int gap, int egp, int band,
                               const VecSmem& S, uint32_t* pscr, uint32_t* ham_out,
                               uint32_t* err_word, uint8_t* dbg0, uint8_t* dbg1, uint32_t* dbg_len) {
  constexpr int LO = -32768;
  const int start_col = 1 + (min(band, len1) + 1) / 2;
  const int ncol = 2 + start_col + min(band + len2 - len1, len2) / 2;
  const int min_score = min(min(min(mismatch, gap), match), 0);
  const int fill = int(int16_t(uint16_t(uint16_t(0x8000u) - uint16_t(min_score))));
  const int lfl = 1 + min(band, len1);
  const int tfl = 1 + min(band + len2 - len1, len2);
  const int edge_rows = max(lfl, tfl);
  auto left_col = [&](int row) { int a = start_col - 1, b = (row - 1) / 2; return a > b ? a - b : 0; };
  auto top_col = [&](int row) { return start_col + row / 2; };
  uint32_t* planes = reinterpret_cast<uint32_t*>(S.stage);
  int r3[M], r2[M], r1[M];
  bool sentinel[M];
  uint32_t pbuf[2 * M];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int c = lane + 32 * m;
    sentinel[m] = c == 0 || c == 1 || c == ncol - 2 || c == ncol - 1;
    int v0 = sentinel[m] ? fill : 0;
    if (c == start_col) v0 = 0;
    int v1 = sentinel[m] ? fill : 0;
    uint32_t c1 = 0;
    if (1 < lfl && c == left_col(1)) { v1 = egp; c1 = 3; }
    if (1 < tfl && c == top_col(1)) { v1 = egp; c1 = 2; }
    r3[m] = 0;
    r2[m] = v0;
    r1[m] = v1;
    const uint32_t w0 = __ballot_sync(FULL, c1 & 1), w1 = __ballot_sync(FULL, (c1 >> 1) & 1);
    if (PS) {
      if (lane == 0) {
        planes[2 * m] = 0u;
        planes[2 * m + 1] = 0u;
        planes[2 * M + 2 * m] = w0;
        planes[2 * M + 2 * m + 1] = w1;
      }
    } else {
      pbuf[2 * m] = lane == 1 ? w0 : 0u;
      pbuf[2 * m + 1] = lane == 1 ? w1 : 0u;
    }
  }
  int row_free = egp;
  int col_min = start_col, col_max = start_col, i_max = 0, j_min = 0;
  bool recalc_left = false, recalc_right = false;
  const int band_mod2 = band % 2;
  const int top_limit = min(band + len2 - len1, len2);
  const int full_band = band + len2 - len1;
  const int last = len1 + len2;
  const int bt_row1 = min(band, len1);
  const int bt_row2 = min(band + len2 - len1, len2);
  const bool fb_even = full_band % 2 == 0;
  const bool do_recalc = egp > gap;
  bool bad = false;
  // Diagonal scores. Lane c reads s1[A - c] and s2[B + c] with A = i_max +
  // col_min and B = j_min - col_min; the guard bytes around each sequence
  // (0x10 before/after s1, 0x20 around s2) make every out-of-range position
  // score `fill`, and clamping the uniform A, B keeps every read inside the
  // guards whatever the band state.
  const uint8_t* p1[M];
  const uint8_t* p2[M];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    p1[m] = S.s1 - (lane + 32 * m);
    p2[m] = S.s2 + (lane + 32 * m);
  }
  auto scores_at = [&](int A, int B, int* out) {
    A = min(max(A, 32 * M - 1 - kSeqPad), len1 + kSeqPad - 1);
    B = min(max(B, -kSeqPad), len2 + kSeqPad - 32 * M);
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const uint32_t a = p1[m][A], b = p2[m][B];
      out[m] = a == b ? match : (((a | b) & 0x30u) ? fill : mismatch);
    }
  };
  int sc[M];
  scores_at(i_max + col_min, j_min - col_min, sc);
  // Middle rows: past the ends-free edge cells and both wedge transitions,
  // inside regime B of the band advance with no recalc pending. There the
  // advance is fixed by the row's parity -- an even row adds 1 to B, an odd row
  // adds 1 to A, col_min moves by -1/+1 when the band is odd and col_max by
  // -1/+1 when band + len2 - len1 is even -- so (col_min, col_max) repeat every
  // two rows and the range checks of the first middle pair cover the rest.
  const int mid_lo = max(edge_rows - 1, max(bt_row1, bt_row2));
  const int dcm = band_mod2 ? -1 : 0;  // col_min change on an even row (undone on the odd row)
  const int dcx = fb_even ? -1 : 0;    // col_max change on an even row (undone on the odd row)
  bool mid_checked = false;
  for (int row0 = 2; row0 <= last; row0 += 2) {
    const bool mid_pair = row0 > mid_lo && row0 + 1 <= last && !recalc_left && !recalc_right &&
                          i_max + band_mod2 < len1 - 1 && (row0 + 1) / 2 + col_max - start_col < len2 &&
                          (row0 + 2) / 2 + col_max + dcx - start_col < len2;
    if (mid_pair) {
      if (!mid_checked) {  // the checks of the generic rows, for this pair's two rows
        const int cm1 = col_min + dcm, cx1 = col_max + dcx;
        bad |= (col_max < col_min) | (col_max >= ncol) | (col_min - 1 < 0) | (col_max + 1 > ncol);
        bad |= (cx1 < cm1) | (cx1 >= ncol) | (cm1 < 0) | (cx1 + 2 > ncol);
        mid_checked = true;
        if (bad) break;
      }
      int A = i_max + col_min, B = j_min - col_min;
      // (col_min, col_max) on the even and odd rows of every middle pair
      const int cmE = col_min, cxE = col_max, cmO = col_min + dcm, cxO = col_max + dcx;
      bool inE[M], inO[M];
      int sc1[M];  // the odd row's diagonal scores
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int c = lane + 32 * m;
        inE[m] = unsigned(c - cmE) < unsigned(cxE - cmE + 1);
        inO[m] = unsigned(c - cmO) < unsigned(cxO - cmO + 1);
        const uint32_t x = p1[m][A], y = p2[m][B + 1];
        sc1[m] = x == y ? match : (((x | y) & 0x30u) ? fill : mismatch);
      }
      int r0 = row0;
      // The pairs stay in the middle regime while r0 + 1 <= last,
      // A - cmE + band_mod2 < len1 - 1, (r0 + 1) / 2 + cxE - start_col < len2
      // and (r0 + 2) / 2 + cxO - start_col < len2. With r0 (even) rising by 2
      // and A by 1 per pair each test is linear in the pair count, so the
      // count is fixed here and the loop carries no data-dependent exit.
      int npairs;
      {
        auto fdiv2 = [](int x) { return x >= 0 ? x / 2 : -((1 - x) / 2); };  // floor(x / 2)
        const int h = r0 / 2;
        int k = fdiv2(last - 1 - r0);
        k = min(k, len1 - 2 - A + cmE - band_mod2);
        k = min(k, len2 - cxE + start_col - 1 - h);
        k = min(k, len2 - cxO + start_col - 2 - h);
        npairs = 1 + max(k, 0);
      }
      for (int pr = 0; pr < npairs; ++pr) {
        // Scores two rows ahead: over a pair A and B each rise by one, so the
        // loads for rows r0+2 / r0+3 go out while rows r0 / r0+1 are computed.
        int sc2[M], sc3[M];
#pragma unroll
        for (int m = 0; m < M; ++m) {
          const uint32_t x = p1[m][A + 1], y = p2[m][B + 1];
          sc2[m] = x == y ? match : (((x | y) & 0x30u) ? fill : mismatch);
          const uint32_t x3 = p1[m][A + 1], y3 = p2[m][B + 2];
          sc3[m] = x3 == y3 ? match : (((x3 | y3) & 0x30u) ? fill : mismatch);
        }
#pragma unroll
        for (int ph = 0; ph < 2; ++ph) {
          const bool E = ph == 0;
          const int row = r0 + ph;
          int cur[M];
          bool b0[M], b1[M];
#pragma unroll
          for (int m = 0; m < M; ++m) {
            int nb;
            if (E) {
              const int a = __shfl_up_sync(FULL, r1[m], 1);
              if (M > 1) {
                const int a31 = m > 0 ? __shfl_sync(FULL, r1[m > 0 ? m - 1 : 0], 31) : 0;
                nb = lane == 0 ? a31 : a;
              } else {
                nb = a;
              }
            } else {
              const int b = __shfl_down_sync(FULL, r1[m], 1);
              if (M > 1) {
                const int b0 = (m + 1 < M) ? __shfl_sync(FULL, r1[m + 1 < M ? m + 1 : m], 0) : 0;
                nb = lane == 31 ? b0 : b;
              } else {
                nb = b;
              }
            }
            // The value needs only max(dg, left, up): the shuffled term joins
            // last with one add-max (dg >= -32768 already, so the clamp is
            // implied). The pointer (tie rules) is formed beside it.
            const int dg = max(r2[m] + (E ? sc[m] : sc1[m]), LO);
            const int own = max(r1[m] + gap, LO);  // up on even rows, left on odd rows
            const int shf = max(nb + gap, LO);     // left on even rows, up on odd rows
            const int v = max(nb + gap, max(dg, own));
            const int l = E ? shf : own, u = E ? own : shf;
            const bool in = E ? inE[m] : inO[m];
            cur[m] = in ? v : (sentinel[m] ? fill : r3[m]);
            const bool dw = dg > max(l, u);
            // code 1 (diag), 3 (up) or 2 (left) as two bits: bit 0 = diag or up, bit 1 = not diag
            const bool upw = SWAP ? !(l >= u) : (u >= l);
            b0[m] = in && (dw || upw);
            b1[m] = in && !dw;
          }
#pragma unroll
          for (int m = 0; m < M; ++m) {
            const uint32_t w0 = __ballot_sync(FULL, b0[m]), w1 = __ballot_sync(FULL, b1[m]);
            if (PS) {
              if (lane == 0) *reinterpret_cast<uint2*>(planes + size_t(row) * (2 * M) + 2 * m) = make_uint2(w0, w1);
            } else if (lane == (row & 31)) {
              pbuf[2 * m] = w0;
              pbuf[2 * m + 1] = w1;
            }
          }
          if (!PS && (row & 31) == 31) {
            const int base = row & ~31;
            uint32_t* dst = pscr + size_t(base + lane) * (2 * M);
#pragma unroll
            for (int w = 0; w < 2 * M; ++w) dst[w] = pbuf[w];
          }
#pragma unroll
          for (int m = 0; m < M; ++m) {
            r3[m] = r2[m];
            r2[m] = r1[m];
            r1[m] = cur[m];
          }
        }
        A += 1;
        B += 1;
        r0 += 2;
#pragma unroll
        for (int m = 0; m < M; ++m) {
          sc[m] = sc2[m];
          sc1[m] = sc3[m];
        }
      }
      col_min = cmE;
      col_max = cxE;
      i_max = A - cmE;
      j_min = B + cmE;
      row0 = r0 - 2;  // the outer loop resumes at row r0
      continue;
    }
    mid_checked = false;
#pragma unroll
    for (int ph = 0; ph < 2; ++ph) {
      const int row = row0 + ph;
      if (ph == 1 && row > last) break;
      const bool E = ph == 0;
      // ---- uniform bookkeeping for this anti-diagonal and the next ----
      const int n = col_max - col_min + 1;
      const int eo = E ? 1 : 0;
      const int left_off = col_min - eo, up_off = col_min + 1 - eo;
      bad |= (col_max < col_min) | (col_max >= ncol) | (left_off < 0) | (up_off + n > ncol);
      row_free = max(row_free + egp, LO);
      int lcol = -1, tcol = -1;
      if (row < edge_rows) {  // ends-free edge cells exist only near the start
        lcol = row < lfl ? left_col(row) : -1;
        tcol = row < tfl ? top_col(row) : -1;
      }
      // band transition at the wedge boundaries (src/nwalign.rs:980-987)
      const bool t1 = row == bt_row1;
      const int cmT = t1 ? sat_sub1(col_min) : col_min;
      const int imT = i_max + (t1 ? 1 : 0);
      const int jmT = j_min - (t1 ? 1 : 0);
      const int cxT = col_max + ((row == bt_row2) ? 1 : 0);
      // advance the band for the next anti-diagonal (src/nwalign.rs:1028-1079)
      int ncm, nim, njm, ncx;
      {
        const bool regA = row < band && row < len1;
        const bool regB = !regA && imT < len1 - 1;
        const int cmA = E ? sat_sub1(cmT) : cmT, imA = imT + 1, jmA = jmT;
        int cmB, imB, jmB;
        if (band_mod2 == 0) {
          cmB = cmT;
          imB = E ? imT : imT + 1;
          jmB = E ? jmT + 1 : jmT;
        } else {
          cmB = E ? sat_sub1(cmT) : cmT + 1;
          imB = E ? imT + 1 : imT;
          jmB = E ? jmT : jmT + 1;
        }
        const int cmC = E ? cmT : cmT + 1, imC = imT, jmC = jmT + 1;
        ncm = regA ? cmA : (regB ? cmB : cmC);
        nim = regA ? imA : (regB ? imB : imC);
        njm = regA ? jmA : (regB ? jmB : jmC);
        const bool rt = row < top_limit;
        const bool mid = !rt && ((row + 1) / 2 + cxT - start_col < len2);
        const int cxA = E ? cxT : cxT + 1;
        const int cxB = fb_even ? (E ? sat_sub1(cxT) : cxT + 1) : cxT;
        const int cxC = E ? sat_sub1(cxT) : cxT;
        ncx = rt ? cxA : (mid ? cxB : cxC);
      }
      // next anti-diagonal's diagonal scores (loads issued now, used next row)
      int scn[M];
      scores_at(nim + ncm, njm - ncm, scn);
      // ---- the cells of this anti-diagonal ----
      int cur[M];
      uint32_t cc[M];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        int nb;  // the previous row's value in the column this parity reads besides c
        if (E) {
          const int a = __shfl_up_sync(FULL, r1[m], 1);
          if (M > 1) {
            const int a31 = m > 0 ? __shfl_sync(FULL, r1[m > 0 ? m - 1 : 0], 31) : 0;
            nb = lane == 0 ? a31 : a;  // column c-1
          } else {
            nb = a;  // lane 0 is column 0, a sentinel: never in band
          }
        } else {
          const int b = __shfl_down_sync(FULL, r1[m], 1);
          if (M > 1) {
            const int b0 = (m + 1 < M) ? __shfl_sync(FULL, r1[m + 1 < M ? m + 1 : m], 0) : 0;
            nb = lane == 31 ? b0 : b;  // column c+1
          } else {
            nb = b;  // column 31 is past the last in-band column when ncol <= 32
          }
        }
        const int c = lane + 32 * m;
        int v = sentinel[m] ? fill : r3[m];
        uint32_t code = 0;
        if (c == lcol) { v = row_free; code = 3; }
        if (c == tcol) { v = row_free; code = 2; }
        const int dg = max(r2[m] + sc[m], LO);
        const int l = max((E ? nb : r1[m]) + gap, LO);
        const int u = max((E ? r1[m] : nb) + gap, LO);
        int e;
        uint32_t pe;
        if (SWAP) {
          const bool lw = l >= u;
          e = lw ? l : u;
          pe = lw ? 2u : 3u;
        } else {
          const bool uw = u >= l;
          e = uw ? u : l;
          pe = uw ? 3u : 2u;
        }
        const bool dw = dg > e;
        if ((unsigned)(c - col_min) < (unsigned)n) {
          v = dw ? dg : e;
          code = dw ? 1u : pe;
        }
        cur[m] = v;
        cc[m] = code;
      }
      if (do_recalc) {
        if (recalc_left) {
          int pv = r1[0];
#pragma unroll
          for (int m = 1; m < M; ++m)
            if ((left_off >> 5) == m) pv = r1[m];
          pv = __shfl_sync(FULL, pv, left_off & 31);
          const int d_free = max(pv + egp, LO);
#pragma unroll
          for (int m = 0; m < M; ++m) {
            if (lane + 32 * m == cmT) {
              const int cv = cur[m];
              const uint32_t pc = cc[m];
              if (d_free > cv) {
                cur[m] = d_free;
                cc[m] = 2;
              } else if (!(d_free != cv || (!SWAP && pc != 1) || (SWAP && pc == 2))) {
                cc[m] = 2;
              }
            }
          }
        }
        if (imT == len1 - 1) recalc_left = true;
        if (recalc_right) {
          const int idx = up_off + cxT - cmT;
          bad |= idx < 0 || idx >= ncol || cxT >= ncol;
          int pv = r1[0];
#pragma unroll
          for (int m = 1; m < M; ++m)
            if ((idx >> 5) == m) pv = r1[m];
          pv = __shfl_sync(FULL, pv, idx & 31);
          const int d_free = max(pv + egp, LO);
#pragma unroll
          for (int m = 0; m < M; ++m) {
            if (lane + 32 * m == cxT) {
              const int cv = cur[m];
              const uint32_t pc = cc[m];
              if (d_free > cv) {
                cur[m] = d_free;
                cc[m] = 3;
              } else if (!(d_free != cv || (!SWAP && pc == 3) || (SWAP && pc != 1))) {
                cc[m] = 3;
              }
            }
          }
        }
        if ((row + 1) / 2 + cxT - start_col == len2) recalc_right = true;
      }
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const uint32_t w0 = __ballot_sync(FULL, cc[m] & 1u), w1 = __ballot_sync(FULL, cc[m] & 2u);
        if (PS) {
          if (lane == 0) *reinterpret_cast<uint2*>(planes + size_t(row) * (2 * M) + 2 * m) = make_uint2(w0, w1);
        } else if (lane == (row & 31)) {
          pbuf[2 * m] = w0;
          pbuf[2 * m + 1] = w1;
        }
      }
      if (!PS && ((row & 31) == 31 || row == last)) {
        const int base = row & ~31;
        if (base + lane <= row) {
          uint32_t* dst = pscr + size_t(base + lane) * (2 * M);
#pragma unroll
          for (int w = 0; w < 2 * M; ++w) dst[w] = pbuf[w];
        }
      }
      col_min = ncm;
      i_max = nim;
      j_min = njm;
      col_max = ncx;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        r3[m] = r2[m];
        r2[m] = r1[m];
        r1[m] = cur[m];
        sc[m] = scn[m];
      }
    }
    if (bad) break;
  }
  if (bad) {
    if (lane == 0) atomicOr(err_word, DERR_BAND_RANGE);
    return false;
  }
  if (!PS && last < 2) {  // rows 0/1 only: flush the buffered words
    if (lane <= last) {
      uint32_t* dst = pscr + size_t(lane) * (2 * M);
#pragma unroll
      for (int w = 0; w < 2 * M; ++w) dst[w] = pbuf[w];
    }
  }
  __syncwarp();
  return reg_traceback<M>(lane, SWAP, len1, len2, start_col, ncol, S, pscr, PS, ham_out, err_word, dbg0,
                          dbg1, dbg_len);
}

// Picks the register form when the pair's compressed width fits 128 columns.
// With `staged` the caller has already put the shorter sequence (the first on
// ties) in S.s1 and the other in S.s2, and g1/g2 point at those copies.
// ONLY_M1: the caller has shown that every pair takes the fast form with one
// lane group (kFormsVec1); the other forms are not compiled in, and a pair
// outside it is refused.
template <bool ONLY_M1 = false>
__device__ bool vec_align_any(int lane, const uint8_t* g1, int l1, const uint8_t* g2, int l2, int16_t match,
                              int16_t mismatch, int16_t gap, int16_t egp, int band_in, const VecSmem& S,
                              uint8_t* scratch, int ncol_bound, int nrow_bound, uint32_t* ham_out, uint32_t* err_word,
                              uint8_t* dbg0, uint8_t* dbg1, uint32_t* dbg_len, bool staged = false) {
  const int len1 = min(l1, l2), len2 = max(l1, l2);
  const int band = band_in < 0 ? len2 : band_in;
  const int start_col = 1 + (min(band, len1) + 1) / 2;
  const int ncol = 2 + start_col + min(band + len2 - len1, len2) / 2;
  uint32_t* w = reinterpret_cast<uint32_t*>(scratch);
  const int nrow = len1 + len2 + 1;
  const int pmax = max(max(int(match), int(mismatch)), 0);
  const bool fast = ncol >= 4 && ncol <= 128 && len1 >= 1 && nrow <= nrow_bound && gap <= 0 && egp <= 0 &&
                    pmax * ((len1 + len2) / 2 + 1) <= 32767;
  if (ONLY_M1 && !(fast && ncol <= 32)) {
    if (lane == 0) atomicOr(err_word, DERR_UNSUPPORTED);
    return false;
  }
  if (fast) {
    const bool swap = l1 > l2;
    {
      const uint8_t* a = swap ? g2 : g1;
      const uint8_t* b = swap ? g1 : g2;
      if (!staged) {
        for (int p = lane; p < len1; p += 32) S.s1[p] = a[p];
        for (int p = lane; p < len2; p += 32) S.s2[p] = b[p];
      }
      for (int p = lane; p < kSeqPad; p += 32) {  // guard bytes: out-of-range positions score `fill`
        S.s1[-1 - p] = 0x10;
        S.s1[len1 + p] = 0x10;
        S.s2[-1 - p] = 0x20;
        S.s2[len2 + p] = 0x20;
      }
    }
    __syncwarp();
    const int mw = ncol <= 32 ? 1 : (ncol <= 64 ? 2 : 4);
    const bool psm = size_t(nrow) * size_t(2 * mw) * 4u <= size_t(kStageBytes);
#define VEC_FAST(MM, SW)                                                                                     \
  return psm ? vec_align_fast<MM, SW, true>(lane, len1, len2, match, mismatch, gap, egp, band, S, w, ham_out,     \
                                            err_word, dbg0, dbg1, dbg_len)                                      \
             : vec_align_fast<MM, SW, false>(lane, len1, len2, match, mismatch, gap, egp, band, S, w, ham_out,    \
                                             err_word, dbg0, dbg1, dbg_len)
    if (mw == 1) {
      if (swap) VEC_FAST(1, true);
      VEC_FAST(1, false);
    }
    if constexpr (!ONLY_M1) {
      if (mw == 2) {
        if (swap) VEC_FAST(2, true);
        VEC_FAST(2, false);
      }
      if (swap) VEC_FAST(4, true);
      VEC_FAST(4, false);
    }
#undef VEC_FAST
  }
  if constexpr (ONLY_M1) return false;  // not reached: refused above
  if (ncol <= 32)
    return vec_align_reg<1>(lane, g1, l1, g2, l2, match, mismatch, gap, egp, band_in, S, w, nrow_bound, ham_out,
                            err_word, dbg0, dbg1, dbg_len);
  if (ncol <= 64)
    return vec_align_reg<2>(lane, g1, l1, g2, l2, match, mismatch, gap, egp, band_in, S, w, nrow_bound, ham_out,
                            err_word, dbg0, dbg1, dbg_len);
  if (ncol <= 128)
    return vec_align_reg<4>(lane, g1, l1, g2, l2, match, mismatch, gap, egp, band_in, S, w, nrow_bound, ham_out,
                            err_word, dbg0, dbg1, dbg_len);
  return vec_align_warp(lane, g1, l1, g2, l2, match, mismatch, gap, egp, band_in, S, scratch, ncol_bound, nrow_bound,
                        ham_out, err_word, dbg0, dbg1, dbg_len);
}

// ---------------------------------------------------------------------------
// K5: row-major ends-free / homopolymer aligner as an anti-diagonal wavefront
// ---------------------------------------------------------------------------
struct RmSmem {
  uint8_t* h1;      // base code (bits 0-3) | homopolymer bit 16, per position
  uint8_t* h2;
  uint32_t* stage;  // kRmStageRows diagonals x 2K words
  uint8_t* tcode;
  uint16_t* fidx;   // inside stage when it fits there (built after the traceback)
};

// m[p] = the base code s[p] (1..4) with bit 4 set when p lies in a run of
// >= 3 equal bases (src/nwalign.rs:211-227) and `homo` is on, so the aligner
// reads a position's base and its gap class with one load.
__device__ void code_mask_warp(int lane, const uint8_t* s, int n, uint8_t* m, bool homo) {
  for (int p = lane; p < n; p += 32) {
    bool in = false;
    if (homo) {
      if (p >= 2 && s[p - 2] == s[p] && s[p - 1] == s[p]) in = true;
      if (p >= 1 && p + 1 < n && s[p - 1] == s[p] && s[p + 1] == s[p]) in = true;
      if (p + 2 < n && s[p + 1] == s[p] && s[p + 2] == s[p]) in = true;
    }
    m[p] = uint8_t(s[p] | (in ? 16u : 0u));
  }
}

// Row-major ends-free aligner (src/nwalign.rs:336-528) evaluated as an
// anti-diagonal wavefront: cell (i, j) sits on anti-diagonal t = i + j at
// offset o = j - i; lane q of group m owns offsets o_lo + 2(q + 32 m) + par,
// par = (t - o_lo) & 1, so every anti-diagonal's band cells are spread over
// the lanes and each needs only its own lane's and one neighbour's previous
// values (one shuffle). Gaps inside homopolymer runs cost homo_gap; the last
// row and column are free; ties prefer up, then left, then diagonal.
// Traceback of the row-major aligner (src/nwalign.rs:234-273) over the
// pointer planes the DP left in pscr (rows t = 0 .. len1 + len2 of 2K words).
template <int K>
__device__ __forceinline__ bool rm_traceback(int lane, int len1, int len2, int o_lo, int o_hi, const RmSmem& S,
                                             const uint32_t* pscr, uint32_t* ham_out, uint32_t* err_word,
                                             uint8_t* dbg0, uint8_t* dbg1, uint32_t* dbg_len) {
  // Row 0 moves left, column 0 moves up.
  // A window of kRmStageRows anti-diagonals of pointer planes is staged in
  // shared memory; lane k tests whether the k-th next step is diagonal (cell
  // (i-k, j-k): anti-diagonal t-2k, same offset), so a run of f diagonal
  // steps is taken at once, one per lane. Other steps are taken singly.
  for (int p = lane; p < len2; p += 32) S.tcode[p] = uint8_t(kUnaligned | (((S.h2[p] & 15u) - 1u) * 5u));
  int i = len1, j = len2, slo = 0x7fffffff;
  uint32_t ham = 0, alen = 0;
  bool ok = true;
  __syncwarp();
  while (i > 0 || j > 0) {
    int v;
    if (i == 0) v = 2;
    else if (j == 0) v = 3;
    else {
      const int o = j - i, t = i + j;
      if (o < o_lo || o > o_hi) { ok = false; break; }
      if (t < slo || (t - slo < kRmStageRows / 2 && slo > 0)) {  // keep half a window below t
        const int nlo = max(0, t - (kRmStageRows - 1));
        __syncwarp();
        const int nw = (t - nlo + 1) * 2 * K;
        const uint32_t* src = pscr + size_t(nlo) * (2 * K);
        for (int x = lane; x < nw; x += 32) S.stage[x] = src[x];
        __syncwarp();
        slo = nlo;
      }
      const int q = (o - o_lo) >> 1, L = q & 31, m = q >> 5;
      const int tk = t - 2 * lane;
      bool diag = false;
      if (tk >= slo && i - lane >= 1 && j - lane >= 1) {
        const uint32_t* wk = S.stage + (tk - slo) * (2 * K) + 2 * m;
        diag = (((wk[0] >> L) & 1u) | (((wk[1] >> L) & 1u) << 1)) == 1u;
      }
      const uint32_t nd = __ballot_sync(FULL, !diag);
      const int f = nd ? __ffs(nd) - 1 : 32;
      if (f > 0) {
        bool mm = false;
        if (lane < f) {
          const uint8_t a = S.h1[i - 1 - lane] & 15u, b = S.h2[j - 1 - lane] & 15u;
          S.tcode[j - 1 - lane] = uint8_t((unsigned(a) - 1u) * 4u + (unsigned(b) - 1u));
          mm = a != b;
          if (dbg0) {
            dbg0[alen + lane] = a;
            dbg1[alen + lane] = b;
          }
        }
        ham += __popc(__ballot_sync(FULL, mm));
        i -= f;
        j -= f;
        alen += uint32_t(f);
        continue;
      }
      const uint32_t* w = S.stage + (t - slo) * (2 * K) + 2 * m;
      v = int((w[0] >> L) & 1u) | (int((w[1] >> L) & 1u) << 1);
    }
    if (v == 2) {
      if (dbg0 && lane == 0) { dbg0[alen] = '-'; dbg1[alen] = S.h2[j - 1] & 15u; }
      --j;
    } else if (v == 3) {
      if (dbg0 && lane == 0) { dbg0[alen] = S.h1[i - 1] & 15u; dbg1[alen] = '-'; }
      --i;
    } else {
      ok = false;
      break;
    }
    ++alen;
  }
  __syncwarp();
  if (!ok) {
    if (lane == 0) atomicOr(err_word, DERR_TRACEBACK);
    return false;
  }
  if (dbg_len && lane == 0) *dbg_len = alen;
  *ham_out = ham;
  return true;
}

template <int K>
__device__ bool rm_align_warp(int lane, const uint8_t* g1, int len1, const uint8_t* g2, int len2, int match,
                              int mismatch, int gap, int homo_gap, int band, bool homo, const RmSmem& S,
                              uint32_t* pscr, uint32_t* ham_out, uint32_t* err_word, uint8_t* dbg0, uint8_t* dbg1,
                              uint32_t* dbg_len) {
  code_mask_warp(lane, g1, len1, S.h1, homo);
  code_mask_warp(lane, g2, len2, S.h2, homo);
  int lband, rband, o_lo, o_hi;
  if (band >= 0) {
    if (len2 > len1) { lband = band; rband = band + (len2 - len1); }
    else if (len1 > len2) { lband = band + (len1 - len2); rband = band; }
    else { lband = band; rband = band; }
    o_lo = max(-lband, -len1);
    o_hi = min(rband, len2);
  } else {
    lband = len1;
    rband = len2;
    o_lo = -len1;
    o_hi = len2;
  }
  const int W = o_hi - o_lo + 1;
  const int P = (W + 1) / 2;
  if (P > 32 * K) {
    if (lane == 0) atomicOr(err_word, DERR_UNSUPPORTED);
    return false;
  }
  __syncwarp();
  const int hgap = homo ? homo_gap : gap;
  // What a cell needs besides its neighbours' values depends only on its
  // position: the up and left gap costs (free on the last row / column,
  // homo_gap inside a homopolymer run), the diagonal score and whether it is
  // a band cell, row 0 / column 0 or outside. Those of anti-diagonal t + 1
  // are loaded and formed while anti-diagonal t's values are computed, so
  // the shared-memory loads stay off the dependency chain.
  //
  // On anti-diagonal t of relative parity p = (t - o_lo) & 1, lane q = lane +
  // 32 m holds cell (i, j) = (E - q, E + q + o_lo + p) with E = (t - o_lo - p)
  // / 2. From one anti-diagonal to the next i steps up when the parity turns
  // even and j when it turns odd, so a lane keeps its two sequence bytes in
  // registers and loads one new byte per group per anti-diagonal.
  struct Cost {
    int gu, gl, sd;
    bool cell, edge;  // band cell; row 0 / column 0 inside the band
  };
  uint32_t inb = 0;  // bit 2m + p: q < P and o_lo + 2q + p <= o_hi
#pragma unroll
  for (int m = 0; m < K; ++m) {
    const int q = lane + 32 * m;
#pragma unroll
    for (int p = 0; p < 2; ++p)
      if (q < P && o_lo + 2 * q + p <= o_hi) inb |= 1u << (2 * m + p);
  }
  // clamped reads: a lane outside the matrix reads a valid byte it ignores
  const unsigned cl1 = unsigned(len1 > 0 ? len1 - 1 : 0), cl2 = unsigned(len2 > 0 ? len2 - 1 : 0);
  uint32_t xb[K], yb[K];
  // LD: 1 loads the h1 byte (i moved), 2 the h2 byte (j moved), 3 both
  auto cost_of = [&](int E, int m, auto par_tag, auto ld_tag) {
    constexpr int PN = decltype(par_tag)::value;
    constexpr int LD = decltype(ld_tag)::value;
    const int q = lane + 32 * m;
    const int i = E - q, j = E + q + o_lo + PN;
    if (LD & 1) xb[m] = S.h1[min(unsigned(i - 1), cl1)];
    if (LD & 2) yb[m] = S.h2[min(unsigned(j - 1), cl2)];
    const uint32_t x = xb[m], y = yb[m];
    const bool inband = (inb >> (2 * m + PN)) & 1u;
    Cost c;
    c.cell = inband && unsigned(i - 1) < unsigned(len1) && unsigned(j - 1) < unsigned(len2);
    c.edge = inband && !c.cell && unsigned(i) <= unsigned(len1) && unsigned(j) <= unsigned(len2);
    c.gu = (j == len2) ? 0 : ((x & 16u) ? hgap : gap);
    c.gl = (i == len1) ? 0 : ((y & 16u) ? hgap : gap);
    c.sd = ((x ^ y) & 15u) == 0u ? match : mismatch;
    return c;
  };
  using Even = std::integral_constant<int, 0>;
  using Odd = std::integral_constant<int, 1>;
  using LoadX = std::integral_constant<int, 1>;
  using LoadY = std::integral_constant<int, 2>;
  using LoadXY = std::integral_constant<int, 3>;
  int ve[K], vo[K];
  Cost cur[K];
  {
    const int p0 = o_lo & 1;  // parity of t = 0
    const int E0 = (0 - o_lo - p0) >> 1;
#pragma unroll
    for (int m = 0; m < K; ++m) {
      ve[m] = kNegSentinel;
      vo[m] = kNegSentinel;
      cur[m] = p0 ? cost_of(E0, m, Odd{}, LoadXY{}) : cost_of(E0, m, Even{}, LoadXY{});
    }
  }
  uint32_t pw[2 * K];
#pragma unroll
  for (int m = 0; m < 2 * K; ++m) pw[m] = 0;
  const int tmax = len1 + len2;
  // One anti-diagonal; PAR = (t - o_lo) & 1 is a template argument, so the
  // loop below runs two anti-diagonals per iteration with no branch on it.
  auto diag = [&](int t, auto par_tag) {
    constexpr int PAR = decltype(par_tag)::value;
    Cost nxt[K];
    const int En = (t - o_lo + PAR) >> 1;  // E of anti-diagonal t + 1 (parity 1 - PAR)
#pragma unroll
    for (int m = 0; m < K; ++m) {  // past tmax: unused
      if (PAR) nxt[m] = cost_of(En, m, Even{}, LoadX{});
      else nxt[m] = cost_of(En, m, Odd{}, LoadY{});
    }
#pragma unroll
    for (int m = 0; m < K; ++m) {
      const int q = lane + 32 * m;
      const int own = PAR ? vo[m] : ve[m];
      int left_nb, up_nb;
      if (PAR == 0) {
        const int a = __shfl_up_sync(FULL, vo[m], 1);
        const int a31 = (m > 0) ? __shfl_sync(FULL, vo[m > 0 ? m - 1 : 0], 31) : kNegSentinel;
        left_nb = (lane == 0) ? a31 : a;
        if (q == 0) left_nb = kNegSentinel;
        up_nb = vo[m];
      } else {
        const int b = __shfl_down_sync(FULL, ve[m], 1);
        const int b0 = (m + 1 < K) ? __shfl_sync(FULL, ve[m + 1 < K ? m + 1 : m], 0) : kNegSentinel;
        up_nb = (lane == 31) ? b0 : b;
        if (q + 1 >= P) up_nb = kNegSentinel;
        left_nb = ve[m];
      }
      const int up = up_nb + cur[m].gu;
      const int left = left_nb + cur[m].gl;
      const int dg = own + cur[m].sd;
      const bool upw = up >= dg && up >= left;
      const bool lw = !upw && left >= dg;
      int val = upw ? up : (lw ? left : dg);
      uint32_t code = upw ? 3u : (lw ? 2u : 1u);
      if (!cur[m].cell) {
        val = cur[m].edge ? 0 : kNegSentinel;
        code = 0u;
      }
      if (PAR) vo[m] = val;
      else ve[m] = val;
      const uint32_t b0w = __ballot_sync(FULL, code & 1u);
      const uint32_t b1w = __ballot_sync(FULL, code & 2u);
      if (lane == (t & 31)) {
        pw[2 * m] = b0w;
        pw[2 * m + 1] = b1w;
      }
    }
    if ((t & 31) == 31 || t == tmax) {
      const int base = t & ~31;
      if (base + lane <= t) {
        uint32_t* dst = pscr + size_t(base + lane) * (2 * K);
#pragma unroll
        for (int m = 0; m < 2 * K; ++m) dst[m] = pw[m];
      }
    }
#pragma unroll
    for (int m = 0; m < K; ++m) cur[m] = nxt[m];
  };
  if ((o_lo & 1) == 0) {  // t = 0 has parity 0
    for (int t = 0; t <= tmax; t += 2) {
      diag(t, Even{});
      if (t + 1 <= tmax) diag(t + 1, Odd{});
    }
  } else {
    for (int t = 0; t <= tmax; t += 2) {
      diag(t, Odd{});
      if (t + 1 <= tmax) diag(t + 1, Even{});
    }
  }
  __syncwarp();
  return rm_traceback<K>(lane, len1, len2, o_lo, o_hi, S, pscr, ham_out, err_word, dbg0, dbg1, dbg_len);
}

// Cooperative form of rm_align_warp for calls that carry few pairs: the
// kNwWarps warps of a CTA share one pair. Warp w owns lane groups
// [w G, (w + 1) G) of the K (G = K / NW, NW = min(K, kNwWarps) warps; the
// others only keep the barriers), so each warp computes G groups per
// anti-diagonal instead of K. The values at a warp boundary -- lane 31 of a
// warp's last group and lane 0 of its first -- pass through shared memory
// (xch[(side * 2 + (t & 1)) * kNwWarps + warp]) with one __syncthreads per
// anti-diagonal. Every warp of the CTA calls this with the same pair, and
// every branch depends on the pair alone, so the barriers line up. S and
// pscr are warp 0's; warp 0 takes the traceback and returns the result, the
// other warps return false.
template <int K>
__device__ bool rm_align_coop(int lane, int wib, const uint8_t* g1, int len1, const uint8_t* g2, int len2, int match,
                              int mismatch, int gap, int homo_gap, int band, bool homo, const RmSmem& S,
                              uint32_t* pscr, uint32_t* ham_out, uint32_t* err_word, int* xch) {
  constexpr int NW = K < kNwWarps ? K : kNwWarps;
  constexpr int G = K / NW;
  if (wib == 0) {
    code_mask_warp(lane, g1, len1, S.h1, homo);
    code_mask_warp(lane, g2, len2, S.h2, homo);
  }
  int o_lo, o_hi;
  if (band >= 0) {
    const int lband = band + (len1 > len2 ? len1 - len2 : 0);
    const int rband = band + (len2 > len1 ? len2 - len1 : 0);
    o_lo = max(-lband, -len1);
    o_hi = min(rband, len2);
  } else {
    o_lo = -len1;
    o_hi = len2;
  }
  const int P = (o_hi - o_lo + 2) / 2;
  if (P > 32 * K) {
    if (wib == 0 && lane == 0) atomicOr(err_word, DERR_UNSUPPORTED);
    return false;
  }
  // before the first anti-diagonal every neighbour holds the sentinel
  if (threadIdx.x < 4 * kNwWarps) xch[threadIdx.x] = kNegSentinel;
  __syncthreads();  // the code bytes and the exchange slots are ready
  const bool act = wib < NW;
  const int m0 = wib * G;
  const int hgap = homo ? homo_gap : gap;
  struct Cost {
    int gu, gl, sd;
    bool cell, edge;
  };
  uint32_t inb = 0;  // bit 2g + p: q < P and o_lo + 2q + p <= o_hi, q = lane + 32 (m0 + g)
#pragma unroll
  for (int g = 0; g < G; ++g) {
    const int q = lane + 32 * (m0 + g);
#pragma unroll
    for (int p = 0; p < 2; ++p)
      if (q < P && o_lo + 2 * q + p <= o_hi) inb |= 1u << (2 * g + p);
  }
  const unsigned cl1 = unsigned(len1 > 0 ? len1 - 1 : 0), cl2 = unsigned(len2 > 0 ? len2 - 1 : 0);
  uint32_t xb[G], yb[G];
  auto cost_of = [&](int E, int g, auto par_tag, auto ld_tag) {
    constexpr int PN = decltype(par_tag)::value;
    constexpr int LD = decltype(ld_tag)::value;
    const int q = lane + 32 * (m0 + g);
    const int i = E - q, j = E + q + o_lo + PN;
    if (LD & 1) xb[g] = S.h1[min(unsigned(i - 1), cl1)];
    if (LD & 2) yb[g] = S.h2[min(unsigned(j - 1), cl2)];
    const uint32_t x = xb[g], y = yb[g];
    const bool inband = (inb >> (2 * g + PN)) & 1u;
    Cost c;
    c.cell = inband && unsigned(i - 1) < unsigned(len1) && unsigned(j - 1) < unsigned(len2);
    c.edge = inband && !c.cell && unsigned(i) <= unsigned(len1) && unsigned(j) <= unsigned(len2);
    c.gu = (j == len2) ? 0 : ((x & 16u) ? hgap : gap);
    c.gl = (i == len1) ? 0 : ((y & 16u) ? hgap : gap);
    c.sd = ((x ^ y) & 15u) == 0u ? match : mismatch;
    return c;
  };
  using Even = std::integral_constant<int, 0>;
  using Odd = std::integral_constant<int, 1>;
  using LoadX = std::integral_constant<int, 1>;
  using LoadY = std::integral_constant<int, 2>;
  using LoadXY = std::integral_constant<int, 3>;
  auto X = [&](int side, int par, int w) -> int& { return xch[(side * 2 + par) * kNwWarps + w]; };
  int ve[G], vo[G];
  Cost cur[G];
  {
    const int p0 = o_lo & 1;  // parity of t = 0
    const int E0 = (0 - o_lo - p0) >> 1;
#pragma unroll
    for (int g = 0; g < G; ++g) {
      ve[g] = kNegSentinel;
      vo[g] = kNegSentinel;
      cur[g] = p0 ? cost_of(E0, g, Odd{}, LoadXY{}) : cost_of(E0, g, Even{}, LoadXY{});
    }
  }
  uint32_t pw[2 * G];
#pragma unroll
  for (int g = 0; g < 2 * G; ++g) pw[g] = 0;
  const int tmax = len1 + len2;
  auto diag = [&](int t, auto par_tag) {
    constexpr int PAR = decltype(par_tag)::value;
    if (act) {
      Cost nxt[G];
      const int En = (t - o_lo + PAR) >> 1;  // E of anti-diagonal t + 1 (parity 1 - PAR)
#pragma unroll
      for (int g = 0; g < G; ++g) {  // past tmax: unused
        if (PAR) nxt[g] = cost_of(En, g, Even{}, LoadX{});
        else nxt[g] = cost_of(En, g, Odd{}, LoadY{});
      }
      const int pt = (t - 1) & 1;  // the exchange slot of anti-diagonal t - 1
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const int q = lane + 32 * (m0 + g);
        const int own = PAR ? vo[g] : ve[g];
        int left_nb, up_nb;
        if (PAR == 0) {
          const int a = __shfl_up_sync(FULL, vo[g], 1);
          int a31;
          if (g > 0) a31 = __shfl_sync(FULL, vo[g > 0 ? g - 1 : 0], 31);
          else a31 = wib > 0 ? X(0, pt, wib > 0 ? wib - 1 : 0) : kNegSentinel;
          left_nb = (lane == 0) ? a31 : a;
          if (q == 0) left_nb = kNegSentinel;
          up_nb = vo[g];
        } else {
          const int b = __shfl_down_sync(FULL, ve[g], 1);
          int b0;
          if (g + 1 < G) b0 = __shfl_sync(FULL, ve[g + 1 < G ? g + 1 : g], 0);
          else b0 = wib + 1 < NW ? X(1, pt, wib + 1 < NW ? wib + 1 : wib) : kNegSentinel;
          up_nb = (lane == 31) ? b0 : b;
          if (q + 1 >= P) up_nb = kNegSentinel;
          left_nb = ve[g];
        }
        const int up = up_nb + cur[g].gu;
        const int left = left_nb + cur[g].gl;
        const int dg = own + cur[g].sd;
        const bool upw = up >= dg && up >= left;
        const bool lw = !upw && left >= dg;
        int val = upw ? up : (lw ? left : dg);
        uint32_t code = upw ? 3u : (lw ? 2u : 1u);
        if (!cur[g].cell) {
          val = cur[g].edge ? 0 : kNegSentinel;
          code = 0u;
        }
        if (PAR) vo[g] = val;
        else ve[g] = val;
        const uint32_t b0w = __ballot_sync(FULL, code & 1u);
        const uint32_t b1w = __ballot_sync(FULL, code & 2u);
        if (lane == (t & 31)) {
          pw[2 * g] = b0w;
          pw[2 * g + 1] = b1w;
        }
      }
      // this anti-diagonal's boundary values for the neighbouring warps
      if (lane == 31) X(0, t & 1, wib) = PAR ? vo[G - 1] : ve[G - 1];
      if (lane == 0) X(1, t & 1, wib) = PAR ? vo[0] : ve[0];
      if ((t & 31) == 31 || t == tmax) {
        const int base = t & ~31;
        if (base + lane <= t) {
          uint32_t* dst = pscr + size_t(base + lane) * (2 * K) + 2 * m0;
#pragma unroll
          for (int g = 0; g < 2 * G; ++g) dst[g] = pw[g];
        }
      }
#pragma unroll
      for (int g = 0; g < G; ++g) cur[g] = nxt[g];
    }
    __syncthreads();
  };
  if ((o_lo & 1) == 0) {  // t = 0 has parity 0
    for (int t = 0; t <= tmax; t += 2) {
      diag(t, Even{});
      if (t + 1 <= tmax) diag(t + 1, Odd{});
    }
  } else {
    for (int t = 0; t <= tmax; t += 2) {
      diag(t, Odd{});
      if (t + 1 <= tmax) diag(t + 1, Even{});
    }
  }
  // the last __syncthreads made every warp's pointer planes visible
  if (wib != 0) return false;
  return rm_traceback<K>(lane, len1, len2, o_lo, o_hi, S, pscr, ham_out, err_word, nullptr, nullptr, nullptr);
}

// rm_dispatch for the cooperative form: every warp of the CTA calls it with
// the same pair; a pair that needs one lane group runs on warp 0 alone.
__device__ bool rm_dispatch_coop(int lane, int wib, const uint8_t* g1, int len1, const uint8_t* g2, int len2,
                                 const KParams& kp, bool homo, int kbound, const RmSmem& S, uint32_t* pscr,
                                 uint32_t* ham, uint32_t* err_word, int* xch) {
  int o_lo, o_hi;
  if (kp.band >= 0) {
    const int lband = kp.band + (len1 > len2 ? len1 - len2 : 0);
    const int rband = kp.band + (len2 > len1 ? len2 - len1 : 0);
    o_lo = max(-lband, -len1);
    o_hi = min(rband, len2);
  } else {
    o_lo = -len1;
    o_hi = len2;
  }
  const int P = (o_hi - o_lo + 2) / 2;
  const int need = (P + 31) / 32;
  if (need > kbound) {
    if (wib == 0 && lane == 0) atomicOr(err_word, DERR_UNSUPPORTED);
    return false;
  }
  if (need <= 1) {
    if (wib != 0) return false;
    return rm_align_warp<1>(lane, g1, len1, g2, len2, kp.match, kp.mismatch, kp.gap, kp.homo_gap, kp.band, homo, S,
                            pscr, ham, err_word, nullptr, nullptr, nullptr);
  }
#define RM_COOP_CASE(KK)                                                                                            \
  if (need <= KK)                                                                                                   \
    return rm_align_coop<KK>(lane, wib, g1, len1, g2, len2, kp.match, kp.mismatch, kp.gap, kp.homo_gap, kp.band,    \
                             homo, S, pscr, ham, err_word, xch);
  RM_COOP_CASE(2)
  RM_COOP_CASE(4)
  RM_COOP_CASE(8)
  RM_COOP_CASE(16)
#undef RM_COOP_CASE
  return false;
}

__device__ RmSmem carve_rm(unsigned char* base, int lmax, int kbound) {
  RmSmem S;
  size_t o = 0;
  auto take = [&](size_t bytes) { unsigned char* p = base + o; o += (bytes + 15) & ~size_t(15); return p; };
  S.h1 = take(lmax);
  S.h2 = take(lmax);
  S.stage = reinterpret_cast<uint32_t*>(take(rm_stage_bytes(kbound)));
  S.tcode = take(lmax);
  S.fidx = rm_fidx_in_stage(lmax, kbound) ? reinterpret_cast<uint16_t*>(S.stage)
                                          : reinterpret_cast<uint16_t*>(take(size_t(lmax) * 2));
  return S;
}


__device__ bool rm_dispatch(int lane, const uint8_t* g1, int len1, const uint8_t* g2, int len2, const KParams& kp,
                            bool homo, int kbound, const RmSmem& S, uint32_t* pscr, uint32_t* ham, uint32_t* err_word,
                            uint8_t* d0, uint8_t* d1, uint32_t* dl) {
  int lband, rband, o_lo, o_hi;
  if (kp.band >= 0) {
    lband = kp.band + (len1 > len2 ? len1 - len2 : 0);
    rband = kp.band + (len2 > len1 ? len2 - len1 : 0);
    o_lo = max(-lband, -len1);
    o_hi = min(rband, len2);
  } else {
    o_lo = -len1;
    o_hi = len2;
  }
  const int P = (o_hi - o_lo + 2) / 2;
  const int need = (P + 31) / 32;
  if (need > kbound) {
    if (lane == 0) atomicOr(err_word, DERR_UNSUPPORTED);
    return false;
  }
#define RM_CASE(KK)                                                                                                  \
  if (need <= KK)                                                                                                    \
    return rm_align_warp<KK>(lane, g1, len1, g2, len2, kp.match, kp.mismatch, kp.gap, kp.homo_gap, kp.band, homo, S, \
                             pscr, ham, err_word, d0, d1, dl);
  RM_CASE(1)
  RM_CASE(2)
  RM_CASE(4)
  RM_CASE(8)
  RM_CASE(16)
#undef RM_CASE
  if (lane == 0) atomicOr(err_word, DERR_UNSUPPORTED);
  return false;
}

// One pair (center c, raw g) through method selection (src/nwalign.rs:1315-1414)
// and the chosen aligner. Both sequences (shorter first, as the vectorized
// aligner wants them) and, with `want_qual`, the raw's qualities are staged in
// the warp's shared memory in one round trip; the steps read them there. On
// return tcode[p] holds each raw position's error-matrix row (see kUnaligned)
// and qual the raw's qualities (staged copy, or the pool's, or null).
struct PairResult {
  bool ok;
  uint8_t method;
  uint32_t ham;
  int lg;
  const uint8_t* tcode;
  uint16_t* fidx;
  const uint8_t* qual;
};

// COOP: every warp of the CTA calls this with the same pair and warp 0's
// buffers (VS, RS, scratch); the row-major DP is shared (rm_dispatch_coop),
// everything else is warp 0's, and only warp 0's result is meaningful. It is
// used only in launches whose geometry rules out the register form, so every
// NW pair of such a launch is row-major.
// FORMS (kForms*): the forms this launch can reach; the others are not
// compiled in, and a pair that would need one is refused.
template <bool COOP, int FORMS = kFormsAll>
__device__ __forceinline__ PairResult align_pair(int lane, const KParams& kp, const PoolDev& pool, const NwGeom& geom,
                                                 uint32_t g, uint32_t c, double kdist, bool want_qual,
                                                 const VecSmem& VS, const RmSmem& RS, int kb, uint8_t* scratch,
                                                 uint32_t* err_word, int wib = 0, int* xch = nullptr) {
  const int k = kp.kmer_size;
  const int lc = int(pool.len[c]), lg = int(pool.len[g]);
  const uint8_t* sc = pool.seq + pool.off[c];
  const uint8_t* sg = pool.seq + pool.off[g];
  const uint8_t* qg = pool.qual ? pool.qual + pool.off[g] : nullptr;
  const bool use_homo = kp.homo_gap != kp.gap && kp.homo_gap <= 0;
  const bool rm_pair = use_homo || !kp.vectorized || lc > 3500 || lg > 3500;
  const bool rm = FORMS == kFormsRm ? true : (FORMS == kFormsVec1 ? false : rm_pair);
  if (rm != rm_pair) {
    if (lane == 0) atomicOr(err_word, DERR_UNSUPPORTED);
    return PairResult{false, AM_NONE, 0u, lg, VS.tcode, VS.fidx, qg};
  }
  if (!COOP && !rm) {
    const bool swap = lc > lg;
    uint8_t* dc = swap ? VS.s2 : VS.s1;
    uint8_t* dg = swap ? VS.s1 : VS.s2;
    uint8_t* dq = vec_qual(VS, geom.lmax);
    const bool stage_q = want_qual && qg != nullptr;
    stage3(lane, sc, lc, dc, sg, lg, dg, stage_q ? qg : nullptr, dq);
    __syncwarp();
    sc = dc;
    sg = dg;
    if (stage_q) qg = dq;
  }
  double kodist = -1.0;
  const int minl = lc < lg ? lc : lg;
  const bool want_kod = kp.use_kmers && kp.gapless && lc == lg;
  // the raw's transition codes and lambda indices live in the layout of the
  // form this pair takes (the per-warp region holds only the forms the
  // launch can reach)
  PairResult R{true, AM_NONE, 0u, lg, rm ? RS.tcode : VS.tcode, rm ? RS.fidx : VS.fidx, qg};
  uint32_t ham = 0;
  if (want_kod || kp.band == 0) {
    const int klen = lc - (k - 1);
    const uint32_t kmask = (k >= 32) ? 0xffffffffu : ((1u << k) - 1u);
    uint32_t eq = 0;
    uint32_t cur = mismatch_word(sc, sg, 0, minl, lane);
    for (int b = 0; b < minl; b += 32) {
      const uint32_t nxt = mismatch_word(sc, sg, b + 32, minl, lane);
      ham += __popc(cur);
      if (want_kod) {
        const unsigned long long both = (static_cast<unsigned long long>(nxt) << 32) | cur;
        const int j = b + lane;
        const bool ok = j < klen && ((uint32_t(both >> lane) & kmask) == 0u);
        eq += __popc(__ballot_sync(FULL, ok));
      }
      cur = nxt;
    }
    if (want_kod && klen > 0) kodist = 1.0 - double(eq) / double(klen);
  }
  const bool gapless = kp.band == 0 || (kp.gapless && fabs(kodist - kdist) < DBL_EPSILON);
  if (gapless) {
    // raw position p aligns to center position p while p < len(center)
    uint8_t* tcode = rm ? RS.tcode : VS.tcode;
    for (int p = (!COOP || wib == 0) ? lane : lg; p < lg; p += 32) {
      const unsigned r = sg[p];
      const unsigned code = (p < lc) ? (unsigned(sc[p]) - 1u) * 4u + (r - 1u) : (kUnaligned | ((r - 1u) * 5u));
      const bool valid = r >= 1u && r <= 4u && (p >= lc || (sc[p] >= 1 && sc[p] <= 4));
      tcode[p] = uint8_t(valid ? code : 255u);
    }
    R.method = AM_GAPLESS;
  } else if (!COOP && !rm) {
    R.ok = vec_align_any<FORMS == kFormsVec1>(lane, sc, lc, sg, lg, int16_t(kp.match), int16_t(kp.mismatch),
                                              int16_t(kp.gap), 0, kp.band,
                         VS, scratch, geom.vec_ncol, geom.vec_nrow, &ham, err_word, nullptr, nullptr, nullptr, true);
    R.method = AM_VECTORIZED;
  } else {
    if constexpr (FORMS != kFormsVec1) {
      if (COOP)
        R.ok = rm_dispatch_coop(lane, wib, sc, lc, sg, lg, kp, use_homo, kb, RS, reinterpret_cast<uint32_t*>(scratch),
                                &ham, err_word, xch);
      else
        R.ok = rm_dispatch(lane, sc, lc, sg, lg, kp, use_homo, kb, RS, reinterpret_cast<uint32_t*>(scratch), &ham,
                           err_word, nullptr, nullptr, nullptr);
    }
    R.tcode = RS.tcode;
    R.fidx = RS.fidx;
    R.method = use_homo ? AM_HOMO : AM_ENDSFREE;
  }
  R.ham = ham;
  __syncwarp();
  return R;
}

// ---------------------------------------------------------------------------
// Pairs that passed the screen (one warp per pair, grid-stride over the queue):
// ordered-k-mer distance (src/kmers.rs:314-328; equal windows <=> equal k-mer
// codes for ACGT input), method choice (src/nwalign.rs:1324-1403), then the
// gapless alignment or the vectorized / row-major aligner, then lambda.
// ---------------------------------------------------------------------------
template <int FORMS>
__global__ void __launch_bounds__(kNwWarps * 32, kAlignCtasPerSm) k_align(CompareLaunch Lp) {
  CompareLaunch L = Lp;
  load_call(L);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cudaTriggerProgrammaticLaunchCompletion();  // the store kernel may start launching
  const KParams& kp = L.kp;
  // the error matrix does not depend on the screen: staged while it finishes
  double* err_s = reinterpret_cast<double*>(smem_raw);
  const int nerr = 16 * kp.ncol;
  for (int t = threadIdx.x; t < nerr; t += blockDim.x) err_s[t] = L.pool.err[t];
  cudaGridDependencySynchronize();  // the screen's pass queue and results are complete
  const uint32_t count = *(volatile uint32_t*)&L.queue_counts[4];
  const int kb = rm_kbound(L.geom.rm_pairs);
  // Few pairs of a launch whose NW pairs are all row-major and span two to
  // four lane groups: the CTA's warps share each pair (rm_align_coop), which
  // cuts a long pair's latency, the bound of such calls. Wider bands (eight
  // or sixteen groups, G > 1 per warp) keep one warp per pair.
  const bool coop = FORMS != kFormsVec1 && L.geom.vec_scratch == 0 && kb >= 2 && kb <= kNwWarps &&
                    count <= 2u * gridDim.x;
  if (blockIdx.x * (coop ? 1u : uint32_t(kNwWarps)) >= count) return;  // nothing queued for this block
  const size_t err_bytes = err_smem_bytes(kp.ncol);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int gw = blockIdx.x * kNwWarps + wib;
  unsigned char* wbase = smem_raw + err_bytes + size_t(wib) * align_smem_per_warp(L.geom);
  const VecSmem VS = carve_vec(wbase, L.geom.lmax, L.geom.vec_ncol);
  const RmSmem RS = carve_rm(wbase, L.geom.lmax, kb);
  const size_t scr_stride = L.geom.vec_scratch > L.geom.rm_scratch ? L.geom.vec_scratch : L.geom.rm_scratch;
  uint8_t* scratch = L.nw_scratch + size_t(gw) * scr_stride;
  __syncthreads();
  // lambda and the raw's result entries, by the warp that holds the alignment
  auto finish = [&](const PairResult& R, uint32_t g) {
    double lam = 0.0;
    float ll32 = -INFINITY;
    if (R.ok) {
      const bool bad = build_fidx(lane, R.tcode, R.qual, R.lg, kp.ncol, kp.use_quals, R.fidx);
      __syncwarp();
      if (bad) {
        if (lane == 0) atomicOr(L.err_word, DERR_LAMBDA);
      } else {
        lam = lambda_chain(lane, R.fidx, R.lg, err_s);
        if (kp.lambda32) ll32 = loglambda32(lane, R.fidx, R.lg, err_s);
      }
    }
    if (lane == 0) {
      if (kp.lambda32) L.pool.res_loglam32[g] = ll32;
      L.pool.res_lambda[g] = lam;
      L.pool.res_ham[g] = R.ok ? R.ham : 0xffffffffu;
      L.pool.res_status[g] = uint8_t(ST_ALIGNED | (R.method << 2));
    }
    __syncwarp();
  };
  if constexpr (FORMS != kFormsVec1) if (coop) {
    // Thread 0 claims a slot for the CTA and reads the raw's screen distance
    // (which warp 0 overwrites with lambda when the pair is done) into shared
    // memory, so every warp takes the same branches through the pair and the
    // barriers inside the shared DP line up. Warp 0's buffers hold the pair.
    __shared__ uint32_t s_slot;
    __shared__ double s_kdist;
    __shared__ int s_xch[4 * kNwWarps];
    unsigned char* w0 = smem_raw + err_bytes;
    const VecSmem VS0 = carve_vec(w0, L.geom.lmax, L.geom.vec_ncol);
    const RmSmem RS0 = carve_rm(w0, L.geom.lmax, kb);
    uint8_t* scratch0 = L.nw_scratch + size_t(blockIdx.x) * kNwWarps * scr_stride;
    auto raw_of = [&](uint32_t slot, uint32_t* center) {
      const uint32_t item = L.queue_pass[slot];
      const uint32_t t = find_task(L.task_prefix, L.ntask, item);
      const TaskDev T = L.tasks[t];
      *center = T.center;
      return T.base + (item - L.task_prefix[t]);
    };
    for (;;) {
      if (threadIdx.x == 0) {
        const uint32_t sl = atomicAdd(&L.queue_counts[6], 1u);
        s_slot = sl;
        if (sl < count) {
          uint32_t c0;
          s_kdist = L.pool.res_lambda[raw_of(sl, &c0)];
        }
      }
      __syncthreads();
      const uint32_t slot = s_slot;
      const double kdist = slot < count ? s_kdist : 0.0;
      __syncthreads();  // every thread has read the slot before thread 0 claims again
      if (slot >= count) break;
      uint32_t center;
      const uint32_t g = raw_of(slot, &center);
      const PairResult R = align_pair<true, FORMS>(lane, kp, L.pool, L.geom, g, center, kdist, kp.use_quals != 0, VS0, RS0,
                                            kb, scratch0, L.err_word, wib, s_xch);
      if (wib == 0) finish(R, g);
    }
    return;
  }
  // Warps claim queue slots one at a time from a shared cursor (cleared with
  // the other counters after each call), so pairs of unequal cost -- gapless
  // against NW, short against long -- and CTAs that become resident late
  // (when shared memory admits fewer CTAs per SM than the grid assumes) even
  // out. Results go to each raw's own entries, so the order is free.
  for (;;) {
    uint32_t slot = 0;
    if (lane == 0) slot = atomicAdd(&L.queue_counts[6], 1u);
    slot = __shfl_sync(FULL, slot, 0);
    if (slot >= count) break;
    const uint32_t item = L.queue_pass[slot];
    const uint32_t t = find_task(L.task_prefix, L.ntask, item);
    const TaskDev T = L.tasks[t];
    const uint32_t g = T.base + (item - L.task_prefix[t]);
    const PairResult R = align_pair<false, FORMS>(lane, kp, L.pool, L.geom, g, T.center, L.pool.res_lambda[g],
                                           kp.use_quals != 0, VS, RS, kb, scratch, L.err_word);
    finish(R, g);
  }
}

// ---------------------------------------------------------------------------
// Final-subs pass and transition counts (src/dada.rs:609-673, src/error.rs:194-249)
// ---------------------------------------------------------------------------
// Every correct raw realigned against its cluster's center with the k-mer
// screen off; each raw position the traceback aligned to a center base adds
// the raw's reads at (4 * center nt + raw nt, the raw's quality there) of its
// sample's 16 x tncol matrix. Warps take contiguous runs of items (ordered by
// sample), count in a shared-memory histogram and flush it to the sample's
// matrix when the sample changes and at the end.
__global__ void __launch_bounds__(kNwWarps * 32, kAlignCtasPerSm) k_final_subs(FinalSubsLaunch F) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const KParams& kp = F.kp;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t gw = blockIdx.x * kNwWarps + wib;
  const uint32_t nwarps = gridDim.x * kNwWarps;
  const int kb = rm_kbound(F.geom.rm_pairs);
  const size_t per_warp = align_smem_per_warp(F.geom) + align16(size_t(16) * F.tncol * 4);
  unsigned char* wbase = smem_raw + size_t(wib) * per_warp;
  const VecSmem VS = carve_vec(wbase, F.geom.lmax, F.geom.vec_ncol);
  const RmSmem RS = carve_rm(wbase, F.geom.lmax, kb);
  uint32_t* hist = reinterpret_cast<uint32_t*>(wbase + align_smem_per_warp(F.geom));
  const int nbins = 16 * F.tncol;
  const size_t scr_stride = F.geom.vec_scratch > F.geom.rm_scratch ? F.geom.vec_scratch : F.geom.rm_scratch;
  uint8_t* scratch = F.nw_scratch + size_t(gw) * scr_stride;
  for (int b = lane; b < nbins; b += 32) hist[b] = 0;
  __syncwarp();
  const uint32_t per = (F.nitems + nwarps - 1) / nwarps;
  const uint32_t i0 = gw * per, i1 = min(F.nitems, i0 + per);
  uint32_t cur_s = 0xffffffffu;
  auto flush = [&]() {
    __syncwarp();
    if (cur_s != 0xffffffffu) {
      for (int b = lane; b < nbins; b += 32) {
        const uint32_t v = hist[b];
        if (v) {
          if (F.out64) atomicAdd(F.out64 + size_t(cur_s) * nbins + b, static_cast<unsigned long long>(v));
          else atomicAdd(F.out + size_t(cur_s) * nbins + b, v);
        }
        hist[b] = 0;
      }
    }
    __syncwarp();
  };
  uint64_t bound = 0;  // what the shared bins may hold since the last flush
  for (uint32_t i = i0; i < i1; ++i) {
    const uint32_t g = F.raw[i], c = F.center[i], smp = F.sample[i];
    // a raw adds at most reads x length to one bin: flush before a 32-bit
    // shared bin could wrap (a raw that could wrap one alone counts in global
    // memory directly)
    const uint64_t add = uint64_t(F.pool.reads[g]) * F.pool.len[g];
    if (smp != cur_s || bound + add > 0xffffffffull) {
      flush();
      cur_s = smp;
      bound = 0;
    }
    bound += add;
    const PairResult R = align_pair<false>(lane, kp, F.pool, F.geom, g, c, 0.0, F.has_quals != 0, VS, RS, kb, scratch,
                                    F.err_word);
    if (!R.ok) continue;  // the error word reports it
    const uint32_t reads = F.pool.reads[g];
    const bool direct = add > 0xffffffffull;  // alone it could wrap a 32-bit bin: count in global memory
    for (int p = lane; p < R.lg; p += 32) {
      const unsigned t = R.tcode[p];
      if (t > 15u) continue;  // an insertion in the raw (or an invalid code)
      const unsigned q = (F.has_quals && R.qual) ? R.qual[p] : 0u;
      if (q >= unsigned(F.tncol)) continue;
      if (!direct) atomicAdd(&hist[t * F.tncol + q], reads);
      else if (F.out64) atomicAdd(F.out64 + size_t(smp) * nbins + t * F.tncol + q, static_cast<unsigned long long>(reads));
      else atomicAdd(F.out + size_t(smp) * nbins + t * F.tncol + q, reads);
    }
    __syncwarp();
  }
  flush();
}

void launch_final_subs(const FinalSubsLaunch& F, cudaStream_t st) {
  if (F.nitems == 0) return;
  const size_t smem = size_t(kNwWarps) * (align_smem_per_warp(F.geom) + align16(size_t(16) * F.tncol * 4));
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_final_subs, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  k_final_subs<<<F.geom.nwarps / kNwWarps, kNwWarps * 32, smem, st>>>(F);
}

// ---------------------------------------------------------------------------
// K7: ordered store (one CTA per task)
// ---------------------------------------------------------------------------
// Each CTA owns kStoreSpan consecutive raws of one task; its stored comps go
// to that span's own segment of the task's output (so concatenating segments
// in order gives ascending raw order) with a per-CTA count and counters.
__global__ void __launch_bounds__(kStoreThreads) k_store(CompareLaunch Lp) {
  CompareLaunch L = Lp;
  load_call(L);
  if (blockIdx.x >= L.nstore_blocks) return;  // a replayed graph's spare CTAs
  constexpr int IPT = kStoreSpan / kStoreThreads;
  __shared__ uint32_t warp_off[32];
  __shared__ uint32_t ctr[TC_NCOUNTERS];
  __shared__ uint32_t s_idx[kStoreSpan], s_ham[kStoreSpan];
  __shared__ double s_lam[kStoreSpan];
  __shared__ float s_ll[kStoreSpan];
  cudaGridDependencySynchronize();  // the alignment kernel's results are complete
  const uint32_t blk = blockIdx.x;
  const uint32_t t = L.store_task[blk];
  const uint32_t span0 = L.store_chunk[blk] * uint32_t(kStoreSpan);
  const TaskDev T = L.tasks[t];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x < TC_NCOUNTERS) ctr[threadIdx.x] = 0;
  __syncthreads();
  uint32_t c_scr = 0, c_al = 0, c_sh = 0, c_gl = 0, c_ve = 0, c_ho = 0, c_ef = 0;
  const uint32_t r0 = span0 + threadIdx.x * IPT;
  uint32_t flags = 0;
  double lam[IPT];
  uint32_t ham[IPT];
#pragma unroll
  for (int q = 0; q < IPT; ++q) {
    lam[q] = 0.0;
    ham[q] = 0;
    const uint32_t r = r0 + q;
    if (r < T.n) {
      const uint32_t g = T.base + r;
      const uint8_t st = L.pool.res_status[g];
      const uint8_t outcome = st & 3u, meth = st >> 2;
      c_scr += outcome != ST_SKIPPED;
      c_al += outcome == ST_ALIGNED;
      c_sh += outcome == ST_SHROUDED;
      c_gl += meth == AM_GAPLESS;
      c_ve += meth == AM_VECTORIZED;
      c_ho += meth == AM_HOMO;
      c_ef += meth == AM_ENDSFREE;
      lam[q] = L.pool.res_lambda[g];
      ham[q] = L.pool.res_ham[g];
      const double e = L.pool.e_minmax[g];
      if (__dmul_rn(lam[q], T.total_reads) > e) {
        flags |= 1u << q;
        const double ne = __dmul_rn(lam[q], double(T.center_reads));
        if (ne > e) L.pool.e_minmax[g] = ne;
      }
      if (g == T.center) L.task_self[t] = lam[q];
    }
  }
  const uint32_t cnt = __popc(flags);
  uint32_t incl = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL, incl, d);
    if (lane >= d) incl += y;
  }
  if (lane == 31) warp_off[w] = incl;
  __syncthreads();
  if (w == 0) {
    const uint32_t v = lane < nw ? warp_off[lane] : 0u;
    uint32_t wi = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, wi, d);
      if (lane >= d) wi += y;
    }
    if (lane < nw) warp_off[lane] = wi - v;
    if (lane == 31) ctr[TC_STORED] = wi;
  }
  __syncthreads();
  // The CTA's stored comps are staged in shared memory in ascending raw order
  // and then written out contiguously, so each warp's stores to the mapped
  // host arrays cover consecutive addresses (few, full PCIe writes instead of
  // one small write per comp).
  uint32_t pos = warp_off[w] + (incl - cnt);
#pragma unroll
  for (int q = 0; q < IPT; ++q) {
    if (flags & (1u << q)) {
      s_idx[pos] = r0 + q;
      s_lam[pos] = lam[q];
      s_ham[pos] = (ham[q] == 0xffffffffu) ? 0u : ham[q];
      if (L.comp_ll32) s_ll[pos] = L.pool.res_loglam32[T.base + r0 + q];
      ++pos;
    }
  }
  __syncthreads();
  {
    const uint32_t nst = ctr[TC_STORED];
    const uint32_t o0 = T.out_off + span0;
    for (uint32_t k = threadIdx.x; k < nst; k += blockDim.x) {
      L.comp_index[o0 + k] = s_idx[k];
      L.comp_lambda[o0 + k] = s_lam[k];
      L.comp_ham[o0 + k] = s_ham[k];
      if (L.comp_ll32) L.comp_ll32[o0 + k] = s_ll[k];
    }
  }
  c_scr = __reduce_add_sync(FULL, c_scr);
  c_al = __reduce_add_sync(FULL, c_al);
  c_sh = __reduce_add_sync(FULL, c_sh);
  c_gl = __reduce_add_sync(FULL, c_gl);
  c_ve = __reduce_add_sync(FULL, c_ve);
  c_ho = __reduce_add_sync(FULL, c_ho);
  c_ef = __reduce_add_sync(FULL, c_ef);
  if (lane == 0) {
    atomicAdd(&ctr[TC_SCREENED], c_scr);
    atomicAdd(&ctr[TC_ALIGNED], c_al);
    atomicAdd(&ctr[TC_SHROUD], c_sh);
    atomicAdd(&ctr[TC_GAPLESS], c_gl);
    atomicAdd(&ctr[TC_VECTORIZED], c_ve);
    atomicAdd(&ctr[TC_HOMO], c_ho);
    atomicAdd(&ctr[TC_ENDSFREE], c_ef);
  }
  __syncthreads();
  if (threadIdx.x < TC_NCOUNTERS) L.blk_counters[size_t(blk) * TC_NCOUNTERS + threadIdx.x] = ctr[threadIdx.x];
  if (blk == 0) {
    // the screen and align kernels have finished: hand their error flags to
    // the host through mapped memory and rearm the queue for the next call
    if (threadIdx.x == 0) {
      reinterpret_cast<volatile uint32_t*>(L.err_host)[0] = *L.err_word;
      reinterpret_cast<volatile uint32_t*>(L.err_host)[1] = L.queue_counts[5];  // profiles the screen read
    }
    __syncthreads();
    if (threadIdx.x < 8) L.queue_counts[threadIdx.x] = 0;
  }
}

static int g_sm_count = 0;
static int sm_count() {
  if (g_sm_count == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm_count <= 0) g_sm_count = 148;
  }
  return g_sm_count;
}

// The screen's chunk for a call of `total` items.
// One wave: k_screen's 64 registers x 256 threads leave room for 4 blocks
// per SM. A warp screens its chunk a few items at a time, one dependent
// round of profile loads each. A call that fits the wave at one chunk per
// warp takes the smallest chunk that does (its items spread thin over many
// warps); a larger one takes the largest chunk that still shares the
// chunks evenly over the wave's warps (at least 90 % of them busy in the
// last round), so no partial second wave or ragged tail is left; chunks
// stay at 16 or more there, since a chunk's per-item bookkeeping runs on
// one lane per item.
// The wave's blocks per SM (at most 4) and the largest chunk (16 or 32)
// come from the tuning table.
uint32_t compare_screen_chunk(uint32_t total, uint32_t screen_blocks_per_sm, uint32_t screen_chunk_max) {
  const int sms = sm_count();
  const uint32_t bps = (screen_blocks_per_sm >= 1 && screen_blocks_per_sm <= 4) ? screen_blocks_per_sm : 4u;
  const uint32_t chmax = screen_chunk_max == 16 ? 16u : 32u;
  const uint32_t cap = uint32_t(sms) * bps;
  const uint64_t warps = uint64_t(cap) * kScreenWarps;
  auto nblocks = [&](uint32_t ch) {
    return uint32_t((uint64_t(total) + kScreenWarps * ch - 1) / (uint64_t(kScreenWarps) * ch));
  };
  uint32_t chunk = 4;
  if (nblocks(chmax) <= cap) {
    while (nblocks(chunk) > cap) chunk *= 2;
  } else {
    for (uint32_t ch = chmax; ch >= 16; ch /= 2) {
      const uint64_t chunks = (uint64_t(total) + ch - 1) / ch;
      const uint64_t rounds = (chunks + warps - 1) / warps;
      chunk = ch;
      if (double(chunks) >= 0.9 * double(rounds * warps)) break;
    }
  }
  return chunk;
}

// The k_align instance for the forms a launch can reach, with its attributes
// set once per device (dynamic shared memory above 48 KB, the largest
// carveout so that kAlignCtasPerSm CTAs fit beside each other).
static void (*align_kernel(const CompareLaunch& L, size_t smem))(CompareLaunch) {
  void (*kalign)(CompareLaunch) = L.geom.forms == kFormsVec1 ? k_align<kFormsVec1>
                                  : L.geom.forms == kFormsRm ? k_align<kFormsRm>
                                                             : k_align<kFormsAll>;
  const int fi = L.geom.forms == kFormsVec1 ? 1 : (L.geom.forms == kFormsRm ? 2 : 0);
  static std::atomic<int> limit[3][64];
  static std::atomic<uint64_t> carved[3];
  int dev = 0;
  cudaGetDevice(&dev);
  std::atomic<int>& lim = limit[fi][dev & 63];
  if (smem > 48 * 1024 && int(smem) > lim.load(std::memory_order_relaxed)) {
    cudaFuncSetAttribute(kalign, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    lim.store(int(smem), std::memory_order_relaxed);
  }
  const uint64_t bit = uint64_t(1) << (dev & 63);
  if (!(carved[fi].load(std::memory_order_relaxed) & bit)) {
    cudaFuncSetAttribute(kalign, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    carved[fi].fetch_or(bit);
  }
  return kalign;
}

// The launch sequence of one compare: k_pivot_dots (pivot_blocks > 0), the
// screen, k_align and the store (store_grid > 0), chained by programmatic
// dependent launch when the tuning asks for it.
static void launch_chain(const CompareLaunch& L, cudaStream_t st, cudaEvent_t* ev, uint32_t screen_blocks,
                         uint32_t pivot_blocks, uint32_t store_grid, void (*kalign)(CompareLaunch), size_t asmem) {
  if (ev) cudaEventRecord(ev[0], st);
  if (pivot_blocks > 0) {
    switch (L.kp.kmer_size) {
      case 3: k_pivot_dots<3><<<pivot_blocks, 256, 0, st>>>(L); break;
      case 4: k_pivot_dots<4><<<pivot_blocks, 256, 0, st>>>(L); break;
      case 5: k_pivot_dots<5><<<pivot_blocks, 256, 0, st>>>(L); break;
      case 6: k_pivot_dots<6><<<pivot_blocks, 256, 0, st>>>(L); break;
      default: k_pivot_dots<7><<<pivot_blocks, 256, 0, st>>>(L); break;
    }
  }
  switch (L.kp.kmer_size) {
    case 3: k_screen<3><<<screen_blocks, kScreenWarps * 32, 0, st>>>(L); break;
    case 4: k_screen<4><<<screen_blocks, kScreenWarps * 32, 0, st>>>(L); break;
    case 5: k_screen<5><<<screen_blocks, kScreenWarps * 32, 0, st>>>(L); break;
    case 6: k_screen<6><<<screen_blocks, kScreenWarps * 32, 0, st>>>(L); break;
    case 7: k_screen<7><<<screen_blocks, kScreenWarps * 32, 0, st>>>(L); break;
    default: k_screen<8><<<screen_blocks, kScreenWarps * 32, 0, st>>>(L); break;
  }
  if (ev) cudaEventRecord(ev[1], st);
  // Programmatic dependent launch: the alignment and store kernels are
  // scheduled while their predecessor drains and wait for its results in
  // cudaGridDependencySynchronize, so the launch gaps overlap with work.
  cudaLaunchAttribute pdl[1];
  pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  pdl[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.stream = st;
  cfg.attrs = pdl;
  cfg.numAttrs = L.pdl ? 1 : 0;
  cfg.gridDim = dim3(L.geom.nwarps / kNwWarps);
  cfg.blockDim = dim3(kNwWarps * 32);
  cfg.dynamicSmemBytes = asmem;
  cudaLaunchKernelEx(&cfg, kalign, L);
  if (ev) cudaEventRecord(ev[2], st);
  if (store_grid > 0) {
    cfg.gridDim = dim3(store_grid);
    cfg.blockDim = dim3(kStoreThreads);
    cfg.dynamicSmemBytes = 0;
    cudaLaunchKernelEx(&cfg, k_store, L);
  }
  if (ev) cudaEventRecord(ev[3], st);
}

void launch_compare(const CompareLaunch& L0, cudaStream_t st, cudaEvent_t* ev) {
  if (L0.total_items == 0) return;
  const int sms = sm_count();
  const uint32_t bps = (L0.screen_blocks_per_sm >= 1 && L0.screen_blocks_per_sm <= 4) ? L0.screen_blocks_per_sm : 4u;
  const uint32_t cap = uint32_t(sms) * bps;
  CompareLaunch L = L0;
  L.hdr = nullptr;
  L.screen_chunk = compare_screen_chunk(L.total_items, L0.screen_blocks_per_sm, L0.screen_chunk_max);
  uint32_t blocks = uint32_t((uint64_t(L.total_items) + kScreenWarps * L.screen_chunk - 1) /
                             (uint64_t(kScreenWarps) * L.screen_chunk));
  if (blocks > cap) blocks = cap;
  const uint32_t pb = (L.cdot_ready && L.total_cl > 0 && L.kp.kmer_size <= 7)
                          ? std::min<uint32_t>((L.total_cl + 7) / 8, uint32_t(sms) * 8u)
                          : 0u;
  const size_t asm_ = err_smem_bytes(L.kp.ncol) + size_t(kNwWarps) * align_smem_per_warp(L.geom);
  launch_chain(L, st, ev, blocks, pb, L.do_store ? L.nstore_blocks : 0u, align_kernel(L, asm_), asm_);
}

int capture_compare_graph(const CompareLaunch& L, cudaStream_t st, uint32_t screen_grid, bool pivot_dots,
                          uint32_t store_grid, cudaGraph_t* out) {
  const int sms = sm_count();
  const size_t asm_ = err_smem_bytes(L.kp.ncol) + size_t(kNwWarps) * align_smem_per_warp(L.geom);
  void (*kalign)(CompareLaunch) = align_kernel(L, asm_);  // attributes before the capture
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return int(e);
  launch_chain(L, st, nullptr, screen_grid, pivot_dots && L.kp.kmer_size <= 7 ? uint32_t(sms) * 8u : 0u,
               store_grid, kalign, asm_);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(st, &g);
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return int(e);
  }
  *out = g;
  return 0;
}

// ---------------------------------------------------------------------------
// Alignment-only debug kernel (parity tests): one warp per pair.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kNwWarps * 32) k_align_debug(int which, const uint8_t* s1cat, const uint32_t* off1,
                                                              const uint32_t* len1, const uint8_t* s2cat,
                                                              const uint32_t* off2, const uint32_t* len2,
                                                              uint32_t npairs, KParams kp, int end_gap, NwGeom geom,
                                                              uint8_t* scratch, uint8_t* al0, uint8_t* al1,
                                                              const uint32_t* aloff, uint32_t* alen, uint32_t* err_word) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t pair = blockIdx.x * kNwWarps + wib;
  if (pair >= npairs) return;
  const size_t scr = which == 0 ? geom.vec_scratch : geom.rm_scratch;
  uint8_t* my_scr = scratch + size_t(pair) * scr;
  uint32_t ham = 0;
  const uint8_t* a = s1cat + off1[pair];
  const uint8_t* b = s2cat + off2[pair];
  if (which == 0) {
    VecSmem S = carve_vec(smem_raw + size_t(wib) * nw_smem_per_warp_vec(geom), geom.lmax, geom.vec_ncol);
    vec_align_any(lane, a, int(len1[pair]), b, int(len2[pair]), int16_t(kp.match), int16_t(kp.mismatch),
                  int16_t(kp.gap), int16_t(end_gap), kp.band, S, my_scr, geom.vec_ncol, geom.vec_nrow, &ham, err_word,
                  al0 + aloff[pair], al1 + aloff[pair], alen + pair);
  } else {
    const int kb = rm_kbound(geom.rm_pairs);
    RmSmem S = carve_rm(smem_raw + size_t(wib) * nw_smem_per_warp_rm(geom), geom.lmax, kb);
    rm_dispatch(lane, a, int(len1[pair]), b, int(len2[pair]), kp, which == 1, kb, S, reinterpret_cast<uint32_t*>(my_scr),
                &ham, err_word, al0 + aloff[pair], al1 + aloff[pair], alen + pair);
  }
}

void launch_align_debug(int which, const uint8_t* s1cat, const uint32_t* off1, const uint32_t* len1,
                        const uint8_t* s2cat, const uint32_t* off2, const uint32_t* len2, uint32_t npairs, KParams kp,
                        int end_gap, const NwGeom& geom, uint8_t* scratch, uint8_t* al0, uint8_t* al1,
                        const uint32_t* aloff, uint32_t* alen, uint32_t* err_word, cudaStream_t st) {
  if (npairs == 0) return;
  const size_t per = which == 0 ? nw_smem_per_warp_vec(geom) : nw_smem_per_warp_rm(geom);
  const size_t smem = per * kNwWarps;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_align_debug, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  const uint32_t blocks = (npairs + kNwWarps - 1) / kNwWarps;
  k_align_debug<<<blocks, kNwWarps * 32, smem, st>>>(which, s1cat, off1, len1, s2cat, off2, len2, npairs, kp, end_gap,
                                                     geom, scratch, al0, al1, aloff, alen, err_word);
}

// ---------------------------------------------------------------------------
// Allocation-free alignment entry point (dgpu_align_pairs_noalloc).
//
// For callers that must not allocate device memory -- a host whose device
// memory is already reserved by its own pool allocator (where cudaMalloc
// fails or fragments that pool), or a latency-bound pipeline that cannot
// afford cudaFree's implicit device-wide synchronisation -- the
// pointer-matrix scratch the aligners need lives in this file-scope array
// instead of a cudaMalloc'd buffer. Every GPU that loads the library holds it
// until the process exits. Calls share it: two calls whose kernels overlap on
// one device race on it.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;  // 16 MiB per device
constexpr size_t kNoAllocHeader = 256;                     // error word, cleared per call
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

// One warp per pair, persistent: warp w reuses scratch slot w for every pair
// it takes, so any number of pairs fits as long as one slot does.
__global__ void __launch_bounds__(kNwWarps * 32) k_align_noalloc(int which, const uint8_t* s1cat, const uint32_t* off1,
                                                                const uint32_t* len1, const uint8_t* s2cat,
                                                                const uint32_t* off2, const uint32_t* len2,
                                                                uint32_t npairs, KParams kp, int end_gap, NwGeom geom,
                                                                uint8_t* scratch, size_t slot_bytes, uint8_t* al0,
                                                                uint8_t* al1, const uint32_t* aloff, uint32_t* alen,
                                                                uint32_t* err_word) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t gw = blockIdx.x * kNwWarps + wib;
  const uint32_t nw = gridDim.x * kNwWarps;
  uint8_t* my_scr = scratch + size_t(gw) * slot_bytes;
  const int kb = rm_kbound(geom.rm_pairs);
  for (uint32_t pair = gw; pair < npairs; pair += nw) {
    uint32_t ham = 0;
    // the shared-memory carve and the scratch slot are sized for geom.lmax:
    // a longer pair is refused before anything is staged
    if (len1[pair] > uint32_t(geom.lmax) || len2[pair] > uint32_t(geom.lmax)) {
      if (lane == 0) atomicOr(err_word, DERR_GEOMETRY);
      continue;
    }
    const uint8_t* a = s1cat + off1[pair];
    const uint8_t* b = s2cat + off2[pair];
    uint8_t* o0 = al0 + aloff[pair];
    uint8_t* o1 = al1 + aloff[pair];
    bool ok;
    if (which == 0) {
      VecSmem S = carve_vec(smem_raw + size_t(wib) * nw_smem_per_warp_vec(geom), geom.lmax, geom.vec_ncol);
      ok = vec_align_any(lane, a, int(len1[pair]), b, int(len2[pair]), int16_t(kp.match), int16_t(kp.mismatch),
                         int16_t(kp.gap), int16_t(end_gap), kp.band, S, my_scr, geom.vec_ncol, geom.vec_nrow, &ham,
                         err_word, o0, o1, alen + pair);
    } else {
      RmSmem S = carve_rm(smem_raw + size_t(wib) * nw_smem_per_warp_rm(geom), geom.lmax, kb);
      ok = rm_dispatch(lane, a, int(len1[pair]), b, int(len2[pair]), kp, which == 1, kb, S,
                       reinterpret_cast<uint32_t*>(my_scr), &ham, err_word, o0, o1, alen + pair);
    }
    __syncwarp();
    if (!ok) continue;
    // the traceback wrote the rows end first; put them left to right
    const uint32_t n = alen[pair];
    for (uint32_t q = lane; q < n / 2; q += 32) {
      const uint8_t x0 = o0[q], x1 = o1[q];
      o0[q] = o0[n - 1 - q];
      o1[q] = o1[n - 1 - q];
      o0[n - 1 - q] = x0;
      o1[n - 1 - q] = x1;
    }
    __syncwarp();
  }
}

// Device address of g_noalloc_scratch, resolved once per device with that
// device current (cudaGetSymbolAddress); host code must never hand the
// symbol itself to a kernel. The cached address belongs to the device's
// primary context: after cudaDeviceReset the module may load elsewhere, so
// this entry point must not be used again in that process.
static std::mutex g_noalloc_mu;
static uint8_t* g_noalloc_ptr[64] = {nullptr};

static cudaError_t noalloc_scratch(int device, uint8_t** out) {
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[device] = static_cast<uint8_t*>(p);
  }
  *out = g_noalloc_ptr[device];
  return cudaSuccess;
}

}  // namespace dgpu

extern "C" int dgpu_align_pairs_noalloc(int which, int npairs, int max_len, const uint8_t* s1cat,
                                        const uint32_t* off1, const uint32_t* len1, const uint8_t* s2cat,
                                        const uint32_t* off2, const uint32_t* len2, const dgpu_align_params* params,
                                        int end_gap, uint8_t* al0, uint8_t* al1, const uint32_t* al_off,
                                        uint32_t* al_len, void* stream) {
  using namespace dgpu;
  auto bad = [](int code, const char* msg) {
    set_last_error(msg);  // reported by dgpu_last_error()
    return code;
  };
  if (which < 0 || which > 2 || npairs <= 0 || !params || !s1cat || !off1 || !len1 || !s2cat || !off2 || !len2 ||
      !al0 || !al1 || !al_off || !al_len)
    return bad(DGPU_E_INVALID, "bad argument");
  if (max_len <= 0 || max_len > 9998) return bad(DGPU_E_INVALID, "max_len must be in 1..9998");
  if (which == 0 && max_len > 3500) return bad(DGPU_E_INVALID, "the vectorized aligner takes lengths <= 3500");
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return bad(DGPU_E_CUDA, cudaGetErrorString(e));
  uint8_t* base = nullptr;
  e = noalloc_scratch(device, &base);
  if (e != cudaSuccess) return bad(DGPU_E_CUDA, cudaGetErrorString(e));
  KParams kp{};
  kp.match = params->match_score;
  kp.mismatch = params->mismatch;
  kp.gap = params->gap_p;
  kp.homo_gap = params->homo_gap_p;
  kp.band = params->band;
  kp.ncol = 1;
  // geometry bounds for any pair of lengths in [1, max_len]
  NwGeom g{};
  g.lmax = max_len;
  const int64_t bb = kp.band < 0 ? int64_t(max_len) : int64_t(kp.band);
  g.vec_ncol = int32_t(4 + (std::min<int64_t>(bb, max_len) + 1) / 2 + std::min<int64_t>(bb + max_len - 1, max_len) / 2);
  g.vec_nrow = 2 * max_len + 1;
  const int64_t W = kp.band < 0 ? int64_t(2 * max_len + 1) : std::min<int64_t>(2 * bb + max_len, 2 * int64_t(max_len) + 1);
  g.rm_pairs = int32_t(std::min<int64_t>((W + 1) / 2, 512));
  g.vec_scratch = align16(size_t(g.vec_nrow) * std::max<size_t>(size_t(g.vec_ncol), 32));
  g.rm_scratch = align16(size_t(2 * max_len + 1) * 2 * rm_kbound(g.rm_pairs) * 4);
  const size_t slot = which == 0 ? g.vec_scratch : g.rm_scratch;
  const size_t avail = kNoAllocScratchBytes - kNoAllocHeader;
  const size_t max_warps = avail / slot;
  if (slot > avail || max_warps < size_t(kNwWarps))
    return bad(DGPU_E_INVALID, "max_len too long: four alignments' scratch exceeds the 16 MiB static area");
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  size_t warps = std::min<size_t>(max_warps, size_t(std::max(sms, 1)) * 4 * kNwWarps);
  warps = std::min<size_t>(warps, (size_t(npairs) + kNwWarps - 1) / kNwWarps * kNwWarps);
  warps = std::max<size_t>(kNwWarps, warps / kNwWarps * kNwWarps);  // multiple of 4, <= max_warps
  g.nwarps = int32_t(warps);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint32_t* err_word = reinterpret_cast<uint32_t*>(base);
  const size_t smem = (which == 0 ? nw_smem_per_warp_vec(g) : nw_smem_per_warp_rm(g)) * kNwWarps;
  int smem_optin = 0;
  e = cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if (e != cudaSuccess) return bad(DGPU_E_CUDA, cudaGetErrorString(e));
  if (smem > size_t(smem_optin))
    return bad(DGPU_E_INVALID, "max_len too long: four alignments' shared-memory staging exceeds the device's "
                               "per-block limit");
  if (smem > 48 * 1024) {
    e = cudaFuncSetAttribute(k_align_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return bad(DGPU_E_CUDA, cudaGetErrorString(e));
  }
  e = cudaMemsetAsync(err_word, 0, 4, st);
  if (e != cudaSuccess) return bad(DGPU_E_CUDA, cudaGetErrorString(e));
  (void)cudaGetLastError();  // so the check after the launch sees only this launch's error
  k_align_noalloc<<<uint32_t(warps / kNwWarps), kNwWarps * 32, smem, st>>>(which, s1cat, off1, len1, s2cat, off2, len2,
                                                                uint32_t(npairs), kp, end_gap, g, base + kNoAllocHeader,
                                                                slot, al0, al1, al_off, al_len, err_word);
  e = cudaGetLastError();
  if (e != cudaSuccess) return bad(DGPU_E_CUDA, cudaGetErrorString(e));
  uint32_t flag = 0;
  e = cudaMemcpyAsync(&flag, err_word, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return bad(DGPU_E_CUDA, cudaGetErrorString(e));
  if (flag & DERR_GEOMETRY)
    return bad(DGPU_E_DEVICE, "a pair exceeded the bounds sized for max_len and was refused (its outputs are left unwritten)");
  if (flag) return bad(flag & DERR_UNSUPPORTED ? DGPU_E_UNSUPPORTED : DGPU_E_DEVICE, "device error flag set");
  return 0;
}

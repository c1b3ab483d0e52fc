// Test driver (CPU only): the product's clustering loop (SampleState: absorb,
// shuffle, p-update, bud, final pass) driven by the oracle's compare in place
// of the GPU kernels, on one sample read from a file. Prints the result tables
// for tests/test_host_loop.py to hold against the oracle's full run_dada. The
// kernel launchers are stubs: nothing here touches a device.
//
// With a second argument W > 1 the loop runs as W ranks (threads) of a
// sharded run: each rank keeps the oracle's comps of its own share of the
// uniques (shard_bounds) and the ranks meet in the product's shard_exchange
// through an in-process all-gather; every rank's tables must be the same.
// A third argument "r:k" makes rank r report a failed compare at its k-th
// call: every rank must then leave the loop at that same exchange.
#include "dgpu_host.cpp"

#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

namespace dgpu {
void launch_profiles(const uint8_t*, const uint32_t*, const uint32_t*, uint32_t, int, uint8_t*, uint8_t*,
                     cudaStream_t) {}
void launch_profiles_sparse(const uint8_t*, const uint32_t*, const uint32_t*, uint32_t, uint32_t, uint16_t*,
                            uint8_t*, uint32_t*, uint8_t*, cudaStream_t) {}
void launch_compare(const CompareLaunch&, cudaStream_t, cudaEvent_t*) {}
uint32_t compare_screen_chunk(uint32_t, uint32_t, uint32_t) { return 4; }
// no graphs on the CPU: the host takes its direct-launch path
int capture_compare_graph(const CompareLaunch&, cudaStream_t, uint32_t, bool, uint32_t, cudaGraph_t*) { return 1; }
void launch_fill_f64(double*, size_t, double, cudaStream_t) {}
void launch_final_subs(const FinalSubsLaunch&, cudaStream_t) {}
void launch_align_debug(int, const uint8_t*, const uint32_t*, const uint32_t*, const uint8_t*, const uint32_t*,
                        const uint32_t*, uint32_t, KParams, int, const NwGeom&, uint8_t*, uint8_t*, uint8_t*,
                        const uint32_t*, uint32_t*, uint32_t*, cudaStream_t) {}
}  // namespace dgpu

extern "C" {
typedef struct {
  int32_t match_score, mismatch, gap_p, homo_gap_p;
  int32_t use_kmers;
  double kdist_cutoff;
  int32_t kmer_size, band, vectorized, gapless;
} orc_align_params;
void* orc_c_b_new(int, const uint8_t*, const uint32_t*, const uint32_t*, const uint8_t*, const uint32_t*,
                  const uint8_t*, int, int, double, double, int);
int orc_c_b_add_center(void*, int);
void orc_c_b_set_lock(void*, int, int);
int orc_c_b_compare(void*, int, const double*, int, const orc_align_params*, int, int, uint32_t*, double*,
                    uint32_t*, double*, double*, uint64_t*);
}

using namespace dgpu;

static void hex_row(std::string& o, const char* name, const double* v, size_t n) {
  o += name;
  char b[24];
  for (size_t k = 0; k < n; ++k) {
    uint64_t x;
    std::memcpy(&x, &v[k], 8);
    std::snprintf(b, sizeof b, " %016llx", static_cast<unsigned long long>(x));
    o += b;
  }
  o += "\n";
}

template <class T>
static void int_row(std::string& o, const char* name, const std::vector<T>& v) {
  o += name;
  for (const T& x : v) o += " " + std::to_string(static_cast<long long>(x));
  o += "\n";
}

// All-gather among the threads of one process: deposit, wait for all, copy
// out, wait again so that no block is overwritten before every rank read it.
struct ThreadGather {
  int world;
  std::mutex mu;
  std::condition_variable cv;
  std::vector<std::vector<uint8_t>> blocks;
  int arrived = 0;
  uint64_t gen = 0;
  explicit ThreadGather(int w) : world(w), blocks(size_t(w)) {}
  void barrier(std::unique_lock<std::mutex>& lk) {
    const uint64_t g = gen;
    if (++arrived == world) {
      arrived = 0;
      ++gen;
      cv.notify_all();
    } else {
      cv.wait(lk, [&] { return gen != g; });
    }
  }
  int run(int rank, const void* send, uint64_t bytes, void* recv) {
    std::unique_lock<std::mutex> lk(mu);
    const uint8_t* s = static_cast<const uint8_t*>(send);
    blocks[size_t(rank)].assign(s, s + bytes);
    barrier(lk);
    int bad = 0;
    for (int r = 0; r < world; ++r) {
      if (blocks[size_t(r)].size() != bytes) bad = 1;
      else std::memcpy(static_cast<uint8_t*>(recv) + size_t(r) * bytes, blocks[size_t(r)].data(), bytes);
    }
    barrier(lk);
    return bad;
  }
};

struct Input {
  int n = 0, ncol2 = 0;
  EncodedView in;
  std::vector<uint8_t> seqb, qualb, prior;
  std::vector<double> errx;
  DadaConf conf{};
};

static std::mutex oracle_mu;  // the oracle sessions are driven one call at a time

static int run_rank(const Input& I, int rank, int world, ThreadGather& G, std::string& out, int fail_rank,
                    int fail_call) {
  const int n = I.n;
  const EncodedView& in = I.in;
  const orc_align_params ap{5, -4, -8, -8, 1, 0.42, 5, 16, 1, 1};
  void* sess;
  {
    std::lock_guard<std::mutex> g(oracle_mu);
    sess = orc_c_b_new(n, in.seq, in.off.data(), in.len.data(), in.qual, in.reads.data(), I.prior.data(), 5, 1,
                       I.conf.omega_a, I.conf.omega_p, 1);
  }
  std::vector<uint8_t> lock(n, 0), pushed(n, 0);
  SampleState S;
  S.init(n, 0, in.reads.data(), I.prior.data(), lock.data(), &I.conf);
  const std::vector<uint32_t> bounds = shard_bounds(in.len.data(), uint32_t(n), world);
  const uint32_t lo = bounds[size_t(rank)], hi = bounds[size_t(rank) + 1];
  const ShardGather gather = [&](const void* s, uint64_t b, void* r) { return G.run(rank, s, b, r); };
  std::vector<uint32_t> ci_(n), ch(n);
  std::vector<double> cl(n), em(n);
  std::vector<ShardComp> local;
  int64_t ci = 0;
  for (int call = 0; ci >= 0; ++call) {
    ShardHead h{};
    int ns = 0;
    {
      std::lock_guard<std::mutex> g(oracle_mu);
      if (ci > 0 && orc_c_b_add_center(sess, int(S.clusters[size_t(ci)].center)) != ci) return 4;
      for (int r = 0; r < n; ++r)
        if (lock[r] && !pushed[r]) {
          orc_c_b_set_lock(sess, r, 1);
          pushed[r] = 1;
        }
      orc_align_params p = ap;
      p.kdist_cutoff = ci == 0 ? 1.0 : 0.42;
      uint64_t cnt[9];
      ns = orc_c_b_compare(sess, int(ci), I.errx.data(), I.ncol2, &p, I.conf.greedy ? 1 : 0, 2, ci_.data(),
                           cl.data(), ch.data(), em.data(), &h.self, cnt);
    }
    // this rank's share of the stored comps, as its device's store gives them
    local.clear();
    for (int k = 0; k < ns; ++k)
      if (ci_[k] >= lo && ci_[k] < hi)
        local.push_back(ShardComp{ci_[k], ch[k], cl[k],
                                  I.conf.fp32 ? (cl[k] > 0.0 ? float(std::log(cl[k]))
                                                             : -std::numeric_limits<float>::infinity())
                                              : std::numeric_limits<float>::quiet_NaN(),
                                  0u});
    const uint32_t center = uint32_t(S.clusters[size_t(ci)].center);
    h.has_self = center >= lo && center < hi ? 1u : 0u;
    if (!h.has_self) h.self = 0.0;
    h.ns = uint32_t(local.size());
    h.ctr[TC_STORED] = h.ns;
    if (rank == fail_rank && call == fail_call) {
      h = ShardHead{};
      h.err = DGPU_E_DEVICE;
      local.clear();
    }
    if (shard_exchange(S, size_t(ci), h, local, world, gather)) {
      out = "failed at call " + std::to_string(call) + ": " + dgpu_last_error();
      return 6;
    }
    ci = S.advance(size_t(ci));
  }
  dgpu_result* R = finish(S, SampleSeqs{in.seq, in.off.data(), in.len.data()});
  out = "nclust " + std::to_string(R->cl_reads.size()) + "\n";
  int_row(out, "map", R->map);
  hex_row(out, "pvals", R->pvals.data(), R->pvals.size());
  int_row(out, "cl_reads", R->cl_reads);
  int_row(out, "cl_birth_type", R->cl_birth_type);
  int_row(out, "cl_birth_from", R->cl_birth_from);
  int_row(out, "cl_mem_off", R->cl_mem_off);
  int_row(out, "mem_raw", R->mem_raw);
  int_row(out, "mem_hamming", R->mem_hamming);
  hex_row(out, "mem_lambda", R->mem_lambda.data(), R->mem_lambda.size());
  hex_row(out, "mem_pval", R->mem_pval.data(), R->mem_pval.size());
  hex_row(out, "cl_birth_pval", R->cl_birth_pval.data(), R->cl_birth_pval.size());
  hex_row(out, "cl_birth_fold", R->cl_birth_fold.data(), R->cl_birth_fold.size());
  hex_row(out, "cl_birth_e", R->cl_birth_e.data(), R->cl_birth_e.size());
  out += "fp32 " + std::to_string(R->fp32[0]) + " " + std::to_string(R->fp32[1]) + "\n";
  delete R;
  return 0;
}

// input: n, total bytes, ncol (int32); lens u32[n]; bases char[total];
// abund u32[n]; Phred sums u32[total]; err f64[16 * ncol]; then, optional,
// omega_a, omega_p, omega_c, min_fold (f64); detect_singletons, greedy,
// min_hamming, min_abund, max_clust (max_clust 0 = all), fp32 (int32);
// prior u8[n]. With fp32 the comps carry float(ln lambda) as their FP32
// log-sum, the stand-in for the kernel's compensated sum.
int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const int world = argc > 2 ? std::atoi(argv[2]) : 1;
  if (world < 1) return 2;
  int fail_rank = -1, fail_call = -1;
  if (argc > 3 && std::sscanf(argv[3], "%d:%d", &fail_rank, &fail_call) != 2) return 2;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  int n, tot, ncol;
  if (std::fread(&n, 4, 1, f) != 1 || std::fread(&tot, 4, 1, f) != 1 || std::fread(&ncol, 4, 1, f) != 1) return 2;
  std::vector<uint32_t> lens(n), ab(n), qs(tot);
  std::vector<char> seq(tot);
  std::vector<double> err(16 * size_t(ncol));
  if (std::fread(lens.data(), 4, n, f) != size_t(n) || std::fread(seq.data(), 1, tot, f) != size_t(tot) ||
      std::fread(ab.data(), 4, n, f) != size_t(n) || std::fread(qs.data(), 4, tot, f) != size_t(tot) ||
      std::fread(err.data(), 8, err.size(), f) != err.size())
    return 2;
  Input I;
  I.n = n;
  I.conf = DadaConf{1e-40, 1e-4, 1e-40, 1.0, 0.42, false, true, 1, 1, size_t(n)};
  I.prior.assign(size_t(n), 0);
  double dp[4];
  int32_t ip[6];
  if (std::fread(dp, 8, 4, f) == 4) {
    if (std::fread(ip, 4, 6, f) != 6 || std::fread(I.prior.data(), 1, size_t(n), f) != size_t(n)) return 2;
    I.conf = DadaConf{dp[0], dp[1], dp[2], dp[3], 0.42, ip[0] != 0, ip[1] != 0, uint32_t(ip[2]), uint32_t(ip[3]),
                      ip[4] > 0 ? size_t(ip[4]) : size_t(n)};
    I.conf.fp32 = ip[5] != 0;
  }
  std::fclose(f);
  std::vector<uint32_t> offs(n);
  uint32_t w = 0;
  for (int t = 0; t < n; ++t) {
    offs[t] = w;
    w += lens[t];
  }
  I.seqb.resize(tot);
  I.qualb.resize(tot);
  I.in.seq = I.seqb.data();
  I.in.qual = I.qualb.data();
  uint32_t bt, bp;
  encode_uniques(0, n, seq.data(), offs.data(), lens.data(), ab.data(), nullptr, qs.data(), I.in, &bt, &bp);
  if (bt != 0xffffffffu) return 3;
  I.ncol2 = ncol;
  I.errx = extend_err(err.data(), ncol, I.in.qmax, I.ncol2);
  ThreadGather G(world);
  std::vector<std::string> outs(static_cast<size_t>(world));
  std::vector<int> rcs(static_cast<size_t>(world), 0);
  std::vector<std::thread> th;
  for (int r = 1; r < world; ++r)
    th.emplace_back([&, r] { rcs[size_t(r)] = run_rank(I, r, world, G, outs[size_t(r)], fail_rank, fail_call); });
  rcs[0] = run_rank(I, 0, world, G, outs[0], fail_rank, fail_call);
  for (auto& t : th) t.join();
  if (fail_rank >= 0) {  // every rank failed at the same exchange
    for (int r = 0; r < world; ++r) {
      std::printf("rank %d rc %d %s\n", r, rcs[size_t(r)], outs[size_t(r)].c_str());
      const std::string& o = outs[size_t(r)];
      if (rcs[size_t(r)] != 6 || o.substr(0, o.find(':')) != outs[0].substr(0, outs[0].find(':'))) return 7;
    }
    return 0;
  }
  for (int r = 0; r < world; ++r) {
    if (rcs[size_t(r)]) return rcs[size_t(r)];
    if (outs[size_t(r)] != outs[0]) return 5;
  }
  std::fputs(outs[0].c_str(), stdout);
  return 0;
}

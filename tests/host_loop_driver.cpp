// Test driver (CPU only): the product's clustering loop (SampleState: absorb,
// shuffle, p-update, bud, final pass) driven by the oracle's compare in place
// of the GPU kernels, on one sample read from a file. Prints the result tables
// for tests/test_host_loop.py to hold against the oracle's full run_dada. The
// kernel launchers are stubs: nothing here touches a device.
#include "dgpu_host.cpp"

#include <cstdio>
#include <cstring>

namespace dgpu {
void launch_profiles(const uint8_t*, const uint32_t*, const uint32_t*, uint32_t, int, uint8_t*, uint8_t*,
                     cudaStream_t) {}
void launch_profiles_sparse(const uint8_t*, const uint32_t*, const uint32_t*, uint32_t, uint32_t, uint16_t*,
                            uint8_t*, uint32_t*, uint8_t*, cudaStream_t) {}
void launch_compare(const CompareLaunch&, cudaStream_t, cudaEvent_t*) {}
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

static void hex_row(const char* name, const double* v, size_t n) {
  std::printf("%s", name);
  for (size_t k = 0; k < n; ++k) {
    uint64_t b;
    std::memcpy(&b, &v[k], 8);
    std::printf(" %016llx", static_cast<unsigned long long>(b));
  }
  std::printf("\n");
}

template <class T>
static void int_row(const char* name, const std::vector<T>& v) {
  std::printf("%s", name);
  for (const T& x : v) std::printf(" %lld", static_cast<long long>(x));
  std::printf("\n");
}

// input: n, total bytes, ncol (int32); lens u32[n]; bases char[total];
// abund u32[n]; Phred sums u32[total]; err f64[16 * ncol]
int main(int argc, char** argv) {
  if (argc < 2) return 2;
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
  std::fclose(f);
  std::vector<uint32_t> offs(n);
  uint32_t w = 0;
  for (int t = 0; t < n; ++t) {
    offs[t] = w;
    w += lens[t];
  }
  std::vector<uint8_t> seqb(tot), qualb(tot);
  EncodedView in;
  in.seq = seqb.data();
  in.qual = qualb.data();
  uint32_t bt, bp;
  encode_uniques(0, n, seq.data(), offs.data(), lens.data(), ab.data(), nullptr, qs.data(), in, &bt, &bp);
  if (bt != 0xffffffffu) return 3;
  int ncol2 = ncol;
  std::vector<double> errx = extend_err(err.data(), ncol, in.qmax, ncol2);
  const orc_align_params ap{5, -4, -8, -8, 1, 0.42, 5, 16, 1, 1};
  void* sess = orc_c_b_new(n, in.seq, in.off.data(), in.len.data(), in.qual, in.reads.data(), nullptr, 5, 1, 1e-40,
                           1e-4, 1);
  DadaConf conf{1e-40, 1e-4, 1e-40, 1.0, 0.42, false, true, 1, 1, size_t(n)};
  std::vector<uint8_t> lock(n, 0), prior(n, 0), pushed(n, 0);
  SampleState S;
  S.init(n, 0, in.reads.data(), prior.data(), lock.data(), &conf);
  std::vector<uint32_t> ci_(n), ch(n);
  std::vector<double> cl(n), em(n);
  int64_t ci = 0;
  while (ci >= 0) {
    if (ci > 0 && orc_c_b_add_center(sess, int(S.clusters[size_t(ci)].center)) != ci) return 4;
    for (int r = 0; r < n; ++r)
      if (lock[r] && !pushed[r]) {
        orc_c_b_set_lock(sess, r, 1);
        pushed[r] = 1;
      }
    orc_align_params p = ap;
    p.kdist_cutoff = ci == 0 ? 1.0 : 0.42;
    double self;
    uint64_t cnt[9];
    const int ns = orc_c_b_compare(sess, int(ci), errx.data(), ncol2, &p, 1, 2, ci_.data(), cl.data(), ch.data(),
                                   em.data(), &self, cnt);
    // the host half of the store, as SampleState::absorb does it
    Cluster& c = S.clusters[size_t(ci)];
    c.self_ = self;
    c.comp.clear();
    const uint32_t center = uint32_t(c.center);
    for (int k = 0; k < ns; ++k) {
      const Comp cp{uint32_t(ci), ci_[k], cl[k], ch[k]};
      c.comp.push_back(cp);
      if (ci == 0 || cp.index == center) S.set_rcomp(cp.index, cp);
    }
    for (const Comp& cp : c.comp) {
      const uint32_t raw = cp.index;
      S.add_cand(raw, uint32_t(ci), cp.lambda, cp.hamming);
      if (++S.ncand[raw] == 2) {
        S.clusters[S.raw_cluster[raw]].multi.put(S.raw_pos[raw], true);
        if (S.built) S.emax[raw] = S.compmax[raw].lambda * double(S.reads_used[S.compmax[raw].i]);
      }
    }
    ci = S.advance(size_t(ci));
  }
  dgpu_result* R = finish(S, SampleSeqs{in.seq, in.off.data(), in.len.data()});
  std::printf("nclust %zu\n", R->cl_reads.size());
  int_row("map", R->map);
  hex_row("pvals", R->pvals.data(), R->pvals.size());
  int_row("cl_reads", R->cl_reads);
  int_row("cl_birth_type", R->cl_birth_type);
  int_row("cl_birth_from", R->cl_birth_from);
  int_row("cl_mem_off", R->cl_mem_off);
  int_row("mem_raw", R->mem_raw);
  int_row("mem_hamming", R->mem_hamming);
  hex_row("mem_lambda", R->mem_lambda.data(), R->mem_lambda.size());
  hex_row("mem_pval", R->mem_pval.data(), R->mem_pval.size());
  hex_row("cl_birth_pval", R->cl_birth_pval.data(), R->cl_birth_pval.size());
  hex_row("cl_birth_fold", R->cl_birth_fold.data(), R->cl_birth_fold.size());
  hex_row("cl_birth_e", R->cl_birth_e.data(), R->cl_birth_e.size());
  delete R;
  return 0;
}

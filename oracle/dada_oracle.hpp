// CPU oracle for the dada2-rs `dada` compare step -- TEST INFRASTRUCTURE ONLY.
//
// This is a single-threaded-deterministic C++ restatement of the Rust reference
// (HPCBio/dada2-rs 0.2.0) used to certify the CUDA product path and to time the
// CPU baseline. It is never linked into, loaded by, or called from the product
// library; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
// use it, and only as the checker.
//
// Each function names the reference file:line it restates. The reference cannot
// be compiled here (it is Rust; no cargo/rustc), so the restatement is pinned
// against the reference's own unit tests and inline known-answer vectors
// (ported in tests/test_oracle_*.py).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace orc {

// src/nwalign.rs:27 -- sentinel in Sub::map for a reference position that
// aligns to a gap in the query.
constexpr uint16_t GAP_GLYPH = 9999;

// src/nwalign.rs:63-90 (the NW backend only; WFA is off by default).
struct AlignParams {
  int32_t match_score = 5;
  int32_t mismatch = -4;
  int32_t gap_p = -8;
  int32_t homo_gap_p = -8;
  bool use_kmers = true;
  double kdist_cutoff = 0.42;
  int32_t kmer_size = 5;
  int32_t band = 16;
  bool vectorized = true;
  bool gapless = true;
};

// src/nwalign.rs:96-103
struct VecScores {
  int16_t match_score, mismatch, gap_p, end_gap_p;
  int32_t band;
};

// src/containers.rs:14-20
struct Comparison {
  uint32_t i = 0;
  uint32_t index = 0;
  double lambda = 0.0;
  uint32_t hamming = 0;
};

// src/containers.rs:29-45 (q0/q1 omitted: nothing on the compare path reads them)
struct Sub {
  uint32_t len0 = 0;
  std::vector<uint16_t> map;
  std::vector<uint16_t> pos;
  std::vector<uint8_t> nt0, nt1;
  size_t nsubs() const { return pos.size(); }
};

// src/containers.rs:78-108
struct Raw {
  std::vector<uint8_t> seq;        // 1..4 (A,C,G,T)
  std::vector<uint8_t> qual;       // rounded mean Phred
  bool has_qual = false;
  bool prior = false;
  // src/kmers.rs:137-147 resident 8-bit screen: dense for k<8, sparse for k>=8
  bool has_kmer8 = false;
  bool kmer8_sparse = false;
  std::vector<uint8_t> kmer8;
  std::vector<std::pair<uint16_t, uint8_t>> kmer8_sp;
  bool has_kord = false;
  std::vector<uint16_t> kord;
  uint32_t reads = 0;
  uint32_t index = 0;
  double p = 0.0;
  Comparison comp;
  bool lock = false;
  bool correct = true;
  size_t len() const { return seq.size(); }
};

// src/containers.rs:188-194
struct BudCand {
  double p;
  uint32_t reads;
  size_t r;
  size_t raw_idx;
};

enum BirthType : int32_t { BIRTH_INITIAL = 0, BIRTH_ABUNDANCE = 1, BIRTH_PRIOR = 2, BIRTH_SINGLETON = 3 };

// src/containers.rs:198-263
struct Bi {
  std::vector<uint8_t> seq;
  int64_t center = -1;
  std::vector<size_t> raws;
  uint32_t reads = 0;
  uint32_t i = 0;
  bool update_e = true;
  bool check_locks = true;
  double self_ = 0.0;
  int32_t birth_type = BIRTH_INITIAL;
  uint32_t birth_from = 0;
  double birth_pval = 0.0;
  double birth_fold = 1.0;
  double birth_e = 0.0;
  Comparison birth_comp;
  std::vector<Comparison> comp;
  bool has_bud_min = false, has_bud_min_prior = false;
  BudCand bud_min{}, bud_min_prior{};
};

// src/containers.rs:277-330
struct B {
  std::vector<Raw> raws;
  std::vector<Bi> clusters;
  uint32_t reads = 0;
  uint64_t nalign = 0;
  uint64_t nshroud = 0;
  double omega_a = 0.0, omega_p = 0.0;
  bool use_quals = true;
  std::vector<uint32_t> raw_cluster;
  std::vector<double> e_minmax;
};

// Alignment scratch (src/nwalign.rs:118-164), minus the timers.
struct AlignBuf {
  std::vector<int32_t> d32;
  std::vector<uint8_t> p32;
  std::vector<int16_t> d16;
  std::vector<uint8_t> p8;
  std::vector<int16_t> diag_buf;
  std::vector<uint8_t> homo1, homo2;
  std::vector<uint8_t> al0, al1;
};

// Which aligner raw_align_dp picked (src/nwalign.rs:1315-1414).
enum AlignMethod : int32_t { M_NONE = 0, M_GAPLESS = 1, M_VECTORIZED = 2, M_HOMO = 3, M_ENDSFREE = 4 };

// ---- kmers.rs ----
size_t n_kmers(int k);
std::vector<uint16_t> assign_kmer(const uint8_t* seq, size_t len, int k);
std::vector<uint8_t> assign_kmer8(const uint8_t* seq, size_t len, int k);
std::vector<std::pair<uint16_t, uint8_t>> assign_kmer8_sparse(const uint8_t* seq, size_t len, int k);
std::vector<uint16_t> assign_kmer_order(const uint8_t* seq, size_t len, int k);
void raw_assign_kmers(Raw& raw, int k);
double kmer_dist(const uint16_t* kv1, size_t len1, const uint16_t* kv2, size_t len2, int k, size_t n);
double kmer_dist8(const uint8_t* kv1, size_t len1, const uint8_t* kv2, size_t len2, int k, size_t n);
double kmer_dist8_sparse(const std::vector<std::pair<uint16_t, uint8_t>>& kv1, size_t len1,
                         const std::vector<std::pair<uint16_t, uint8_t>>& kv2, size_t len2, int k);
double kord_dist(const uint16_t* kord1, size_t len1, const uint16_t* kord2, size_t len2, int k);

// ---- nwalign.rs ----
void align_endsfree(const uint8_t* s1, size_t len1, const uint8_t* s2, size_t len2, int32_t match,
                    int32_t mismatch, int32_t gap_p, int32_t band, AlignBuf& buf);
void align_endsfree_homo(const uint8_t* s1, size_t len1, const uint8_t* s2, size_t len2,
                         const AlignParams& p, AlignBuf& buf);
void align_gapless(const uint8_t* s1, size_t len1, const uint8_t* s2, size_t len2, AlignBuf& buf);
void align_vectorized(const uint8_t* s1, size_t len1, const uint8_t* s2, size_t len2,
                      const VecScores& sc, AlignBuf& buf);
// Full-matrix variant kept by the reference's tests as the byte-identity spec
// for the rolling kernel (src/nwalign.rs:2375-2719).
void align_vectorized_full(const uint8_t* s1, size_t len1, const uint8_t* s2, size_t len2,
                           const VecScores& sc, AlignBuf& buf);
Sub al2subs(const std::vector<uint8_t>& al0, const std::vector<uint8_t>& al1);
// Returns false when the k-mer screen shrouds the pair. `method`, `kdist`,
// `kodist` report what the screen and dispatcher saw.
bool raw_align(const Raw& raw1, const Raw& raw2, const AlignParams& p, AlignBuf& buf,
               int32_t* method, double* kdist, double* kodist);
bool sub_new(const Raw& raw0, const Raw& raw1, const AlignParams& p, AlignBuf& buf, Sub& out,
             int32_t* method);

// ---- pval.rs ----
double compute_lambda(const Raw& raw, const Sub* sub, const double* err_mat, size_t ncol,
                      bool use_quals);
double calc_pA(uint32_t reads, double e_reads, bool prior);
double gamma_lr(double a, double x);
double ln_gamma_lanczos(double x);
double get_pA(uint32_t reads, bool prior, double lambda, uint32_t hamming, uint32_t bi_reads,
              bool detect_singletons);
uint64_t b_p_update(B& b, bool greedy, bool detect_singletons, double min_fold,
                    uint32_t min_hamming, uint32_t min_abund);

// ---- containers.rs ----
void b_new(B& b, std::vector<Raw>&& raws, double omega_a, double omega_p, bool use_quals);
void b_init(B& b);
size_t b_add_cluster(B& b, Bi&& bi);
void bi_add_raw(B& b, size_t bi_idx, size_t raw_idx);
size_t bi_pop_raw(B& b, size_t bi_idx, size_t r);
void bi_census(B& b, size_t i);
void bi_assign_center(B& b, size_t i);

// ---- cluster.rs ----
// Per-raw result of the compare map (src/cluster.rs:279-330).
struct CompareItem {
  double lambda;
  uint32_t hamming;  // UINT32_MAX = shrouded or skipped
  bool skipped;
  int32_t method;
};
struct CompareStats {
  uint64_t screened = 0, aligned = 0, stored = 0;
  uint64_t gapless = 0, vectorized = 0, homo = 0, endsfree = 0;
};
// The map alone: fills `items` (size nraw). nthreads<=1 runs serially.
void compare_map(const B& b, size_t i, const double* err_mat, size_t ncol, const AlignParams& p,
                 bool greedy, int nthreads, std::vector<CompareItem>& items);
// src/cluster.rs:239-423: map + serial store.
CompareStats b_compare_parallel(B& b, size_t i, const double* err_mat, size_t ncol,
                                const AlignParams& p, bool greedy, int nthreads);

struct Cand {
  uint32_t ci;
  double lambda;
  uint32_t hamming;
};
using CandIndex = std::vector<std::vector<Cand>>;
void index_add_cluster(CandIndex& index, const B& b, size_t ci);

struct ShuffleCarry {
  std::vector<Comparison> compmax;
  std::vector<double> emax;
  std::vector<uint32_t> reads_used;
  std::vector<uint8_t> in_affected;
  std::vector<size_t> affected;
  std::vector<uint8_t> dirty_cluster;
  std::vector<uint32_t> dirty_list;
  std::vector<uint8_t> reads_fell;
  std::vector<uint32_t> reads_fell_list;
  bool built = false;
  void grow_to(size_t n);
};
struct ShuffleResult {
  size_t moves = 0;
  size_t calls = 0;
};
ShuffleResult b_shuffle_converge(B& b, const CandIndex& index, size_t max_shuffle,
                                 ShuffleCarry& carry);
// Returns the new cluster index, or -1 when nothing buds.
int64_t b_bud_incremental(B& b, double min_fold, uint32_t min_hamming, uint32_t min_abund);

// ---- dada.rs ----
struct DadaParams {
  AlignParams align;
  std::vector<double> err_mat;
  size_t err_ncol = 0;
  double omega_a = 1e-40, omega_p = 1e-4, omega_c = 1e-40;
  bool detect_singletons = false;
  size_t max_clust = 0;
  double min_fold = 1.0;
  uint32_t min_hamming = 1, min_abund = 1;
  bool use_quals = true;
  bool greedy = true;
  int nthreads = 1;
  bool transitions = false;  // also compute the DadaAux transition counts (src/dada.rs:609-640)
};
struct RawInput {
  std::string seq;  // ASCII
  uint32_t abundance = 0;
  bool prior = false;
  bool has_quals = false;
  std::vector<uint32_t> quals;  // per-position Phred sums
};
struct ClusterSummary {
  std::vector<uint8_t> sequence;
  uint32_t reads;
  std::vector<uint32_t> members, member_hammings;
  std::vector<double> member_lambdas, member_pvals;
  int32_t birth_type;
  uint32_t birth_from;
  double birth_pval, birth_fold, birth_e;
  uint32_t birth_hamming;
};
struct DadaRunStats {
  uint64_t compare_calls = 0;
  uint64_t cmp_scanned = 0;  // sum of nraw over compare calls (src/dada.rs:862,969)
  uint64_t screened = 0, aligned = 0, stored = 0;
  uint64_t gapless = 0, vectorized = 0, homo = 0, endsfree = 0;
  uint64_t shuffle_calls = 0, shuffle_moves = 0;
  double t_compare = 0.0, t_total = 0.0;  // seconds
  double t_shuffle = 0.0, t_pupdate = 0.0, t_bud = 0.0;
};
struct DadaResult {
  std::vector<ClusterSummary> clusters;
  std::vector<int64_t> map;  // -1 = None
  std::vector<double> pvals;
  uint64_t nalign = 0, nshroud = 0;
  uint32_t nraw = 0;
  DadaRunStats stats;
  // with DadaParams::transitions: 16 x transitions_ncol counts (src/error.rs:194-249)
  std::vector<uint32_t> transitions;
  size_t transitions_ncol = 0;
};
// Returns an empty string on success, else the validation error message.
std::string dada_uniques(const std::vector<RawInput>& inputs, const DadaParams& params,
                         DadaResult& out);

// ---- learn_errors.rs / error_models.rs / loess.rs (oracle_learn.cpp) ----
struct ErrFunSpec {
  int kind = 0;     // 0 loess, 1 noqual, 2 binned quality, 3 PacBio
  int surface = 0;  // loess: 0 direct, 1 interpolate
  double cell = 0.2;
  double max_error_rate = 0.25, min_error_rate = 1e-7;
  double pseudocount = 1.0;
  std::vector<double> bins;  // binned quality: the anchor quality scores, ascending
};
struct LearnResult {
  size_t nq = 0, passes = 0;
  bool converged = false;
  std::vector<uint32_t> trans;
  std::vector<double> err_in, err_out;
};
std::string errfun_apply(const ErrFunSpec& e, const std::vector<uint32_t>& trans, size_t nq,
                         std::vector<double>& err);
std::vector<uint32_t> build_trans_mat(const std::vector<RawInput>& inputs, const DadaResult& res,
                                      const AlignParams& ap, size_t nq);
std::string learn_errors(const std::vector<std::vector<RawInput>>& samples, DadaParams params,
                         const ErrFunSpec& ef, size_t max_consist, LearnResult& out);

}  // namespace orc

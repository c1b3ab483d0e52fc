// C entry points of the CPU oracle -- TEST INFRASTRUCTURE ONLY (loaded by
// oracle/oracle.py for tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline). Plain pointers and sizes; no ownership crosses the boundary except
// the opaque handles, which the caller frees with the matching *_free call.
#include <algorithm>
#include <cstring>
#include <thread>

#include "dada_oracle.hpp"

using namespace orc;

extern "C" {

typedef struct {
  int32_t match_score, mismatch, gap_p, homo_gap_p;
  int32_t use_kmers;
  double kdist_cutoff;
  int32_t kmer_size, band, vectorized, gapless;
} orc_align_params;

typedef struct {
  orc_align_params align;
  double omega_a, omega_p, omega_c;
  int32_t detect_singletons, max_clust;
  double min_fold;
  uint32_t min_hamming, min_abund;
  int32_t use_quals, greedy, nthreads;
  int32_t transitions;
} orc_dada_params;

typedef struct {
  uint32_t* cl_reads;
  int32_t* cl_birth_type;
  uint32_t* cl_birth_from;
  double* cl_birth_pval;
  double* cl_birth_fold;
  double* cl_birth_e;
  uint32_t* cl_birth_hamming;
  uint32_t* cl_seq_off;  // nclust + 1
  uint8_t* cl_seq;
  uint32_t* cl_mem_off;  // nclust + 1
  uint32_t* mem_raw;
  uint32_t* mem_hamming;
  double* mem_lambda;
  double* mem_pval;
  int32_t* map;  // -1 = not corrected to any cluster
  double* pvals;
  uint64_t* counters;  // 16 slots
  double* times;       // 4 slots
} orc_dada_out;

static AlignParams to_params(const orc_align_params* p) {
  AlignParams a;
  a.match_score = p->match_score;
  a.mismatch = p->mismatch;
  a.gap_p = p->gap_p;
  a.homo_gap_p = p->homo_gap_p;
  a.use_kmers = p->use_kmers != 0;
  a.kdist_cutoff = p->kdist_cutoff;
  a.kmer_size = p->kmer_size;
  a.band = p->band;
  a.vectorized = p->vectorized != 0;
  a.gapless = p->gapless != 0;
  return a;
}

int orc_c_hardware_threads(void) {
  unsigned n = std::thread::hardware_concurrency();
  return n == 0 ? 1 : int(n);
}

// ---------------- kmers ----------------
void orc_c_assign_kmer(const uint8_t* seq, size_t len, int k, uint16_t* out) {
  std::vector<uint16_t> v = assign_kmer(seq, len, k);
  std::memcpy(out, v.data(), v.size() * 2);
}
void orc_c_assign_kmer8(const uint8_t* seq, size_t len, int k, uint8_t* out) {
  std::vector<uint8_t> v = assign_kmer8(seq, len, k);
  std::memcpy(out, v.data(), v.size());
}
size_t orc_c_assign_kmer8_sparse(const uint8_t* seq, size_t len, int k, uint16_t* idx, uint8_t* cnt) {
  auto v = assign_kmer8_sparse(seq, len, k);
  for (size_t t = 0; t < v.size(); ++t) {
    idx[t] = v[t].first;
    cnt[t] = v[t].second;
  }
  return v.size();
}
void orc_c_assign_kmer_order(const uint8_t* seq, size_t len, int k, uint16_t* out) {
  std::vector<uint16_t> v = assign_kmer_order(seq, len, k);
  std::memcpy(out, v.data(), v.size() * 2);
}
double orc_c_kmer_dist(const uint16_t* a, size_t l1, const uint16_t* b, size_t l2, int k) {
  return kmer_dist(a, l1, b, l2, k, n_kmers(k));
}
double orc_c_kmer_dist8(const uint8_t* a, size_t l1, const uint8_t* b, size_t l2, int k) {
  return kmer_dist8(a, l1, b, l2, k, n_kmers(k));
}
double orc_c_kmer_dist8_sparse(const uint16_t* ia, const uint8_t* ca, size_t na, size_t l1,
                               const uint16_t* ib, const uint8_t* cb, size_t nb, size_t l2, int k) {
  std::vector<std::pair<uint16_t, uint8_t>> a(na), b(nb);
  for (size_t t = 0; t < na; ++t) a[t] = {ia[t], ca[t]};
  for (size_t t = 0; t < nb; ++t) b[t] = {ib[t], cb[t]};
  return kmer_dist8_sparse(a, l1, b, l2, k);
}
double orc_c_kord_dist(const uint16_t* a, size_t l1, const uint16_t* b, size_t l2, int k) {
  return kord_dist(a, l1, b, l2, k);
}

// ---------------- aligners ----------------
// which: 0 vectorized (rolling), 1 vectorized full-matrix, 2 ends-free i32,
// 3 ends-free homopolymer, 4 gapless. Buffers need len1+len2 bytes.
// Returns the alignment length.
int orc_c_align(int which, const uint8_t* s1, size_t l1, const uint8_t* s2, size_t l2, int match,
                int mismatch, int gap, int homo_gap, int end_gap, int band, uint8_t* al0, uint8_t* al1) {
  AlignBuf buf;
  if (which == 0 || which == 1) {
    VecScores sc{int16_t(match), int16_t(mismatch), int16_t(gap), int16_t(end_gap), band};
    if (which == 0) align_vectorized(s1, l1, s2, l2, sc, buf);
    else align_vectorized_full(s1, l1, s2, l2, sc, buf);
  } else if (which == 2) {
    align_endsfree(s1, l1, s2, l2, match, mismatch, gap, band, buf);
  } else if (which == 3) {
    AlignParams p;
    p.match_score = match;
    p.mismatch = mismatch;
    p.gap_p = gap;
    p.homo_gap_p = homo_gap;
    p.band = band;
    align_endsfree_homo(s1, l1, s2, l2, p, buf);
  } else {
    align_gapless(s1, l1, s2, l2, buf);
  }
  std::memcpy(al0, buf.al0.data(), buf.al0.size());
  std::memcpy(al1, buf.al1.data(), buf.al1.size());
  return int(buf.al0.size());
}

// One buffer reused across a list of alignments (the reference's buffer-reuse
// test). Alignment t of `n` reads seqs at offsets; outputs are concatenated.
int orc_c_align_vectorized_reuse(int n, const uint8_t* s1cat, const uint32_t* s1off,
                                 const uint32_t* s1len, const uint8_t* s2cat, const uint32_t* s2off,
                                 const uint32_t* s2len, int match, int mismatch, int gap, int end_gap,
                                 int band, uint8_t* al0cat, uint8_t* al1cat, uint32_t* alen) {
  AlignBuf buf;
  size_t w = 0;
  for (int t = 0; t < n; ++t) {
    VecScores sc{int16_t(match), int16_t(mismatch), int16_t(gap), int16_t(end_gap), band};
    align_vectorized(s1cat + s1off[t], s1len[t], s2cat + s2off[t], s2len[t], sc, buf);
    std::memcpy(al0cat + w, buf.al0.data(), buf.al0.size());
    std::memcpy(al1cat + w, buf.al1.data(), buf.al1.size());
    alen[t] = uint32_t(buf.al0.size());
    w += buf.al0.size();
  }
  return int(w);
}

// raw_align on two encoded sequences with k-mer vectors built at params.kmer_size.
// Returns the method (0 = shrouded).
int orc_c_raw_align(const uint8_t* s1, size_t l1, const uint8_t* s2, size_t l2,
                    const orc_align_params* pp, uint8_t* al0, uint8_t* al1, int* alen, double* kdist,
                    double* kodist) {
  AlignParams p = to_params(pp);
  Raw r1, r2;
  r1.seq.assign(s1, s1 + l1);
  r2.seq.assign(s2, s2 + l2);
  if (p.use_kmers) {
    raw_assign_kmers(r1, p.kmer_size);
    raw_assign_kmers(r2, p.kmer_size);
  }
  AlignBuf buf;
  int32_t method = M_NONE;
  bool ok = raw_align(r1, r2, p, buf, &method, kdist, kodist);
  if (!ok) {
    *alen = 0;
    return 0;
  }
  std::memcpy(al0, buf.al0.data(), buf.al0.size());
  std::memcpy(al1, buf.al1.data(), buf.al1.size());
  *alen = int(buf.al0.size());
  return method;
}

// al2subs; map needs len0 slots, pos/nt0/nt1 need min(alen) slots. Returns nsubs.
int orc_c_al2subs(const uint8_t* al0, const uint8_t* al1, int alen, uint32_t* len0, uint16_t* map,
                  uint16_t* pos, uint8_t* nt0, uint8_t* nt1) {
  std::vector<uint8_t> a(al0, al0 + alen), b(al1, al1 + alen);
  Sub s = al2subs(a, b);
  *len0 = s.len0;
  std::copy(s.map.begin(), s.map.end(), map);
  std::copy(s.pos.begin(), s.pos.end(), pos);
  std::copy(s.nt0.begin(), s.nt0.end(), nt0);
  std::copy(s.nt1.begin(), s.nt1.end(), nt1);
  return int(s.nsubs());
}

double orc_c_calc_pA(uint32_t reads, double e_reads, int prior) { return calc_pA(reads, e_reads, prior != 0); }
double orc_c_gamma_lr(double a, double x) { return gamma_lr(a, x); }
double orc_c_ln_gamma(double x) { return ln_gamma_lanczos(x); }
double orc_c_get_pA(uint32_t reads, int prior, double lambda, uint32_t hamming, uint32_t bi_reads,
                    int detect_singletons) {
  return get_pA(reads, prior != 0, lambda, hamming, bi_reads, detect_singletons != 0);
}

// ---------------- compare session (a B with raws and cluster 0) ----------------
struct OrcSession {
  B b;
};

void* orc_c_b_new(int nraw, const uint8_t* seqcat, const uint32_t* off, const uint32_t* len,
                  const uint8_t* qualcat, const uint32_t* reads, const uint8_t* prior, int k,
                  int use_kmers, double omega_a, double omega_p, int use_quals) {
  std::vector<Raw> raws(static_cast<size_t>(nraw));
  for (int t = 0; t < nraw; ++t) {
    Raw& r = raws[size_t(t)];
    r.seq.assign(seqcat + off[t], seqcat + off[t] + len[t]);
    if (qualcat) {
      r.qual.assign(qualcat + off[t], qualcat + off[t] + len[t]);
      r.has_qual = true;
    }
    r.reads = reads[t];
    r.prior = prior ? prior[t] != 0 : false;
    if (use_kmers) raw_assign_kmers(r, k);
  }
  OrcSession* s = new OrcSession();
  b_new(s->b, std::move(raws), omega_a, omega_p, use_quals != 0);
  return s;
}
void orc_c_b_free(void* h) { delete static_cast<OrcSession*>(h); }
int orc_c_b_center(void* h, int ci) { return int(static_cast<OrcSession*>(h)->b.clusters[size_t(ci)].center); }
void orc_c_b_set_center(void* h, int ci, int center) {
  OrcSession* s = static_cast<OrcSession*>(h);
  s->b.clusters[size_t(ci)].center = center;
}
void orc_c_b_set_lock(void* h, int raw, int lock) { static_cast<OrcSession*>(h)->b.raws[size_t(raw)].lock = lock != 0; }
// Adds an empty cluster centred on `center` (membership untouched); returns its index.
int orc_c_b_add_center(void* h, int center) {
  OrcSession* s = static_cast<OrcSession*>(h);
  Bi bi;
  bi.center = center;
  bi.seq = s->b.raws[size_t(center)].seq;
  return int(b_add_cluster(s->b, std::move(bi)));
}

void orc_c_compare_map(void* h, int ci, const double* err, int ncol, const orc_align_params* pp,
                       int greedy, int nthreads, double* lambda, uint32_t* hamming, uint8_t* skipped,
                       int32_t* method) {
  OrcSession* s = static_cast<OrcSession*>(h);
  std::vector<CompareItem> items;
  compare_map(s->b, size_t(ci), err, size_t(ncol), to_params(pp), greedy != 0, nthreads, items);
  for (size_t t = 0; t < items.size(); ++t) {
    lambda[t] = items[t].lambda;
    hamming[t] = items[t].hamming;
    skipped[t] = items[t].skipped ? 1 : 0;
    method[t] = items[t].method;
  }
}

// map + store; returns the number stored. comps_* need nraw slots.
// counters: [nalign, nshroud, screened, aligned, stored, gapless, vectorized, homo, endsfree]
int orc_c_b_compare(void* h, int ci, const double* err, int ncol, const orc_align_params* pp, int greedy,
                    int nthreads, uint32_t* comp_index, double* comp_lambda, uint32_t* comp_hamming,
                    double* e_minmax, double* self_out, uint64_t* counters) {
  OrcSession* s = static_cast<OrcSession*>(h);
  size_t before = s->b.clusters[size_t(ci)].comp.size();
  CompareStats st = b_compare_parallel(s->b, size_t(ci), err, size_t(ncol), to_params(pp), greedy != 0, nthreads);
  const std::vector<Comparison>& cv = s->b.clusters[size_t(ci)].comp;
  for (size_t t = before; t < cv.size(); ++t) {
    comp_index[t - before] = cv[t].index;
    comp_lambda[t - before] = cv[t].lambda;
    comp_hamming[t - before] = cv[t].hamming;
  }
  std::copy(s->b.e_minmax.begin(), s->b.e_minmax.end(), e_minmax);
  *self_out = s->b.clusters[size_t(ci)].self_;
  uint64_t c[9] = {s->b.nalign, s->b.nshroud, st.screened, st.aligned, st.stored,
                   st.gapless, st.vectorized, st.homo, st.endsfree};
  std::copy(c, c + 9, counters);
  return int(cv.size() - before);
}

// ---------------- full dada ----------------
struct OrcDada {
  DadaResult res;
};

void* orc_c_dada(int nraw, const char* seqcat, const uint32_t* off, const uint32_t* len,
                 const uint32_t* abund, const uint8_t* prior, const uint32_t* qualcat,
                 const orc_dada_params* pp, const double* err, int ncol, char* errbuf, int errcap) {
  std::vector<RawInput> in(static_cast<size_t>(nraw));
  for (int t = 0; t < nraw; ++t) {
    RawInput& r = in[size_t(t)];
    r.seq.assign(seqcat + off[t], seqcat + off[t] + len[t]);
    r.abundance = abund[t];
    r.prior = prior ? prior[t] != 0 : false;
    if (qualcat) {
      r.has_quals = true;
      r.quals.assign(qualcat + off[t], qualcat + off[t] + len[t]);
    }
  }
  DadaParams dp;
  dp.align = to_params(&pp->align);
  dp.err_mat.assign(err, err + 16 * size_t(ncol));
  dp.err_ncol = size_t(ncol);
  dp.omega_a = pp->omega_a;
  dp.omega_p = pp->omega_p;
  dp.omega_c = pp->omega_c;
  dp.detect_singletons = pp->detect_singletons != 0;
  dp.max_clust = size_t(pp->max_clust);
  dp.min_fold = pp->min_fold;
  dp.min_hamming = pp->min_hamming;
  dp.min_abund = pp->min_abund;
  dp.use_quals = pp->use_quals != 0;
  dp.greedy = pp->greedy != 0;
  dp.nthreads = pp->nthreads;
  dp.transitions = pp->transitions != 0;
  OrcDada* d = new OrcDada();
  std::string e = dada_uniques(in, dp, d->res);
  if (!e.empty()) {
    if (errbuf && errcap > 0) {
      std::strncpy(errbuf, e.c_str(), size_t(errcap - 1));
      errbuf[errcap - 1] = 0;
    }
    delete d;
    return nullptr;
  }
  return d;
}

void orc_c_dada_free(void* h) { delete static_cast<OrcDada*>(h); }

// ---------------- learn-errors (oracle_learn.cpp) ----------------
struct orc_errfun {
  int32_t kind, surface;
  double cell, max_error_rate, min_error_rate, pseudocount;
  const double* bins;
  int32_t nbins;
};
static ErrFunSpec to_errfun(const orc_errfun* e) {
  ErrFunSpec s;
  s.kind = e->kind;
  s.surface = e->surface;
  s.cell = e->cell;
  s.max_error_rate = e->max_error_rate;
  s.min_error_rate = e->min_error_rate;
  s.pseudocount = e->pseudocount;
  if (e->bins && e->nbins > 0) s.bins.assign(e->bins, e->bins + e->nbins);
  return s;
}
int orc_c_errfun_apply(const orc_errfun* e, const uint32_t* trans, int nq, double* out, char* errbuf, int errcap) {
  std::vector<uint32_t> t(trans, trans + 16 * size_t(nq));
  std::vector<double> err;
  const std::string m = errfun_apply(to_errfun(e), t, size_t(nq), err);
  if (!m.empty()) {
    if (errbuf && errcap > 0) {
      std::strncpy(errbuf, m.c_str(), size_t(errcap - 1));
      errbuf[errcap - 1] = 0;
    }
    return -1;
  }
  std::copy(err.begin(), err.end(), out);
  return 0;
}
// Samples as in orc_c_dada, sample s owning uniques [start[s], start[s+1]).
// info: [0] nq, [1] passes, [2] converged. trans/err_in/err_out need 16 x
// nq_cap slots; returns nq, or -1 with the message in errbuf.
int orc_c_learn_errors(int nsamples, const uint32_t* start, const char* seqcat, const uint32_t* off,
                       const uint32_t* len, const uint32_t* abund, const uint32_t* qualcat, const orc_dada_params* pp,
                       const orc_errfun* ef, int max_consist, int nq_cap, int32_t* info, uint32_t* trans,
                       double* err_in, double* err_out, char* errbuf, int errcap) {
  std::vector<std::vector<RawInput>> samples(static_cast<size_t>(nsamples));
  for (int s = 0; s < nsamples; ++s)
    for (uint32_t t = start[s]; t < start[s + 1]; ++t) {
      RawInput r;
      r.seq.assign(seqcat + off[t], seqcat + off[t] + len[t]);
      r.abundance = abund[t];
      if (qualcat) {
        r.has_quals = true;
        r.quals.assign(qualcat + off[t], qualcat + off[t] + len[t]);
      }
      samples[size_t(s)].push_back(std::move(r));
    }
  DadaParams dp;
  dp.align = to_params(&pp->align);
  dp.omega_a = pp->omega_a;
  dp.omega_p = pp->omega_p;
  dp.omega_c = pp->omega_c;
  dp.detect_singletons = pp->detect_singletons != 0;
  dp.max_clust = size_t(pp->max_clust);
  dp.min_fold = pp->min_fold;
  dp.min_hamming = pp->min_hamming;
  dp.min_abund = pp->min_abund;
  dp.use_quals = pp->use_quals != 0;
  dp.greedy = pp->greedy != 0;
  dp.nthreads = pp->nthreads;
  LearnResult lr;
  const std::string m = learn_errors(samples, dp, to_errfun(ef), size_t(max_consist), lr);
  if (!m.empty() || int(lr.nq) > nq_cap) {
    const std::string msg = m.empty() ? std::string("nq beyond nq_cap") : m;
    if (errbuf && errcap > 0) {
      std::strncpy(errbuf, msg.c_str(), size_t(errcap - 1));
      errbuf[errcap - 1] = 0;
    }
    return -1;
  }
  info[0] = int32_t(lr.nq);
  info[1] = int32_t(lr.passes);
  info[2] = lr.converged ? 1 : 0;
  std::copy(lr.trans.begin(), lr.trans.end(), trans);
  std::copy(lr.err_in.begin(), lr.err_in.end(), err_in);
  std::copy(lr.err_out.begin(), lr.err_out.end(), err_out);
  return int(lr.nq);
}

// Transition counts of a run made with transitions set: returns the column
// count and copies 16 x ncol values to out (when non-null); 0 if none.
int orc_c_dada_transitions(void* h, uint32_t* out) {
  const DadaResult& r = static_cast<OrcDada*>(h)->res;
  if (out) std::copy(r.transitions.begin(), r.transitions.end(), out);
  return int(r.transitions_ncol);
}

// sizes: [nclust, nraw, total members, total center-sequence bytes]
void orc_c_dada_sizes(void* h, int64_t* sizes) {
  const DadaResult& r = static_cast<OrcDada*>(h)->res;
  int64_t mem = 0, seq = 0;
  for (const ClusterSummary& c : r.clusters) {
    mem += int64_t(c.members.size());
    seq += int64_t(c.sequence.size());
  }
  sizes[0] = int64_t(r.clusters.size());
  sizes[1] = int64_t(r.nraw);
  sizes[2] = mem;
  sizes[3] = seq;
}

void orc_c_dada_fill(void* h, const orc_dada_out* o) {
  const DadaResult& r = static_cast<OrcDada*>(h)->res;
  uint32_t so = 0, mo = 0;
  for (size_t ci = 0; ci < r.clusters.size(); ++ci) {
    const ClusterSummary& c = r.clusters[ci];
    o->cl_reads[ci] = c.reads;
    o->cl_birth_type[ci] = c.birth_type;
    o->cl_birth_from[ci] = c.birth_from;
    o->cl_birth_pval[ci] = c.birth_pval;
    o->cl_birth_fold[ci] = c.birth_fold;
    o->cl_birth_e[ci] = c.birth_e;
    o->cl_birth_hamming[ci] = c.birth_hamming;
    o->cl_seq_off[ci] = so;
    std::copy(c.sequence.begin(), c.sequence.end(), o->cl_seq + so);
    so += uint32_t(c.sequence.size());
    o->cl_mem_off[ci] = mo;
    for (size_t t = 0; t < c.members.size(); ++t) {
      o->mem_raw[mo + t] = c.members[t];
      o->mem_hamming[mo + t] = c.member_hammings[t];
      o->mem_lambda[mo + t] = c.member_lambdas[t];
      o->mem_pval[mo + t] = c.member_pvals[t];
    }
    mo += uint32_t(c.members.size());
  }
  o->cl_seq_off[r.clusters.size()] = so;
  o->cl_mem_off[r.clusters.size()] = mo;
  for (size_t t = 0; t < r.map.size(); ++t) {
    o->map[t] = int32_t(r.map[t]);
    o->pvals[t] = r.pvals[t];
  }
  const DadaRunStats& s = r.stats;
  uint64_t c[16] = {r.nalign, s.compare_calls, s.cmp_scanned, s.screened, s.aligned, s.stored,
                    s.gapless, s.vectorized, s.homo, s.endsfree, s.shuffle_calls, s.shuffle_moves,
                    r.nshroud, 0, 0, 0};
  std::copy(c, c + 16, o->counters);
  o->times[0] = s.t_compare;
  o->times[1] = s.t_total;
  o->times[2] = s.t_shuffle + s.t_pupdate + s.t_bud;
  o->times[3] = s.t_pupdate;
}

}  // extern "C"

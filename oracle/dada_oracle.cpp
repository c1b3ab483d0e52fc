// CPU oracle for the dada2-rs `dada` compare step -- TEST INFRASTRUCTURE ONLY.
// See dada_oracle.hpp for the contract. Every routine cites the Rust reference
// (HPCBio/dada2-rs 0.2.0) file:line it restates. Compiled with
// -ffp-contract=off so FP64 expressions round exactly as the Rust code does.
#include "dada_oracle.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <thread>

namespace orc {

[[noreturn]] static void die(const char* what) {
  std::fprintf(stderr, "oracle invariant violated: %s\n", what);
  std::abort();
}
#define ORC_CHECK(c, msg) \
  do {                    \
    if (!(c)) die(msg);   \
  } while (0)

// ===========================================================================
// kmers.rs
// ===========================================================================

size_t n_kmers(int k) { return size_t(1) << (2 * k); }  // src/kmers.rs:49-51

// src/kmers.rs:55-66 -- base-4 index of (nt-1); -1 if any nt is not 1..4.
static inline int64_t encode_kmer(const uint8_t* w, int k) {
  int64_t kmer = 0;
  for (int t = 0; t < k; ++t) {
    unsigned nt = w[t];
    if (nt < 1 || nt > 4) return -1;
    kmer = 4 * kmer + (nt - 1);
  }
  return kmer;
}

// src/kmers.rs:79-89 -- u16 counts over every k-window, saturating.
std::vector<uint16_t> assign_kmer(const uint8_t* seq, size_t len, int k) {
  std::vector<uint16_t> kv(n_kmers(k), 0);
  if (len < size_t(k)) return kv;
  for (size_t s = 0; s + k <= len; ++s) {
    int64_t idx = encode_kmer(seq + s, k);
    if (idx >= 0 && kv[idx] != 0xFFFF) kv[idx]++;
  }
  return kv;
}

// src/kmers.rs:96-101
std::vector<uint8_t> assign_kmer8(const uint8_t* seq, size_t len, int k) {
  std::vector<uint16_t> kv = assign_kmer(seq, len, k);
  std::vector<uint8_t> out(kv.size());
  for (size_t t = 0; t < kv.size(); ++t) out[t] = uint8_t(std::min<uint16_t>(kv[t], 255));
  return out;
}

// src/kmers.rs:113-120
std::vector<std::pair<uint16_t, uint8_t>> assign_kmer8_sparse(const uint8_t* seq, size_t len, int k) {
  std::vector<uint16_t> kv = assign_kmer(seq, len, k);
  std::vector<std::pair<uint16_t, uint8_t>> out;
  for (size_t t = 0; t < kv.size(); ++t)
    if (kv[t] > 0) out.emplace_back(uint16_t(t), uint8_t(std::min<uint16_t>(kv[t], 255)));
  return out;
}

// src/kmers.rs:129-135 -- invalid windows give 0.
std::vector<uint16_t> assign_kmer_order(const uint8_t* seq, size_t len, int k) {
  std::vector<uint16_t> out;
  if (len < size_t(k)) return out;
  out.reserve(len - k + 1);
  for (size_t s = 0; s + k <= len; ++s) {
    int64_t idx = encode_kmer(seq + s, k);
    out.push_back(uint16_t(idx < 0 ? 0 : idx));
  }
  return out;
}

// src/kmers.rs:213-221 (SPARSE_KMER_MIN = 8, src/kmers.rs:45)
void raw_assign_kmers(Raw& raw, int k) {
  if (k >= 8) {
    raw.kmer8_sparse = true;
    raw.kmer8_sp = assign_kmer8_sparse(raw.seq.data(), raw.seq.size(), k);
  } else {
    raw.kmer8_sparse = false;
    raw.kmer8 = assign_kmer8(raw.seq.data(), raw.seq.size(), k);
  }
  raw.has_kmer8 = true;
  raw.kord = assign_kmer_order(raw.seq.data(), raw.seq.size(), k);
  raw.has_kord = true;
}

// src/kmers.rs:233-241
double kmer_dist(const uint16_t* kv1, size_t len1, const uint16_t* kv2, size_t len2, int k, size_t n) {
  uint32_t dotsum = 0;
  for (size_t t = 0; t < n; ++t) dotsum += std::min(kv1[t], kv2[t]);
  double scale = double(std::min(len1, len2) - size_t(k) + 1);
  return 1.0 - double(dotsum) / scale;
}

// src/kmers.rs:254-269 -- -1.0 when any element-wise min is 255.
double kmer_dist8(const uint8_t* kv1, size_t len1, const uint8_t* kv2, size_t len2, int k, size_t n) {
  uint32_t dotsum = 0;
  bool overflow = false;
  for (size_t t = 0; t < n; ++t) {
    uint8_t m = std::min(kv1[t], kv2[t]);
    if (m == 255) overflow = true;
    dotsum += m;
  }
  if (overflow) return -1.0;
  double scale = double(std::min(len1, len2) - size_t(k) + 1);
  return 1.0 - double(dotsum) / scale;
}

// src/kmers.rs:280-308 -- merge-join over ascending (index,count) lists.
double kmer_dist8_sparse(const std::vector<std::pair<uint16_t, uint8_t>>& kv1, size_t len1,
                         const std::vector<std::pair<uint16_t, uint8_t>>& kv2, size_t len2, int k) {
  uint32_t dotsum = 0;
  size_t a = 0, b = 0;
  while (a < kv1.size() && b < kv2.size()) {
    if (kv1[a].first < kv2[b].first) {
      ++a;
    } else if (kv1[a].first > kv2[b].first) {
      ++b;
    } else {
      uint8_t m = std::min(kv1[a].second, kv2[b].second);
      if (m == 255) return -1.0;
      dotsum += m;
      ++a;
      ++b;
    }
  }
  double scale = double(std::min(len1, len2) - size_t(k) + 1);
  return 1.0 - double(dotsum) / scale;
}

// src/kmers.rs:314-328
double kord_dist(const uint16_t* kord1, size_t len1, const uint16_t* kord2, size_t len2, int k) {
  if (len1 != len2) return -1.0;
  size_t km1 = k > 0 ? size_t(k - 1) : 0;
  if (len1 < km1) return -1.0;
  size_t klen = len1 - km1;
  if (klen == 0) return -1.0;
  uint32_t dotsum = 0;
  for (size_t t = 0; t < klen; ++t) dotsum += (kord1[t] == kord2[t]) ? 1u : 0u;
  return 1.0 - double(dotsum) / double(klen);
}

// ===========================================================================
// nwalign.rs
// ===========================================================================

static inline bool is_nt(uint8_t b) { return b >= 1 && b <= 5; }  // src/nwalign.rs:204-206

// src/nwalign.rs:211-227 -- true inside runs of >= 3 identical bytes.
static void homopolymer_mask(const uint8_t* seq, size_t n, std::vector<uint8_t>& mask) {
  mask.assign(n, 0);
  size_t run_start = 0;
  while (run_start < n) {
    size_t run_end = run_start + 1;
    while (run_end < n && seq[run_end] == seq[run_start]) ++run_end;
    if (run_end - run_start >= 3)
      for (size_t t = run_start; t < run_end; ++t) mask[t] = 1;
    run_start = run_end;
  }
}

// src/nwalign.rs:234-273 -- pointer codes 1 diag, 2 left (gap in s1), 3 up.
static void traceback_rowmajor(const uint8_t* p, size_t ncol, const uint8_t* s1, const uint8_t* s2,
                               size_t len1, size_t len2, std::vector<uint8_t>& al0,
                               std::vector<uint8_t>& al1) {
  al0.clear();
  al1.clear();
  size_t i = len1, j = len2;
  while (i > 0 || j > 0) {
    uint8_t v = p[i * ncol + j];
    if (v == 1) {
      ORC_CHECK(i > 0 && j > 0, "traceback diag at edge");
      al0.push_back(s1[i - 1]);
      al1.push_back(s2[j - 1]);
      --i;
      --j;
    } else if (v == 2) {
      ORC_CHECK(j > 0, "traceback left at j=0");
      al0.push_back('-');
      al1.push_back(s2[j - 1]);
      --j;
    } else if (v == 3) {
      ORC_CHECK(i > 0, "traceback up at i=0");
      al0.push_back(s1[i - 1]);
      al1.push_back('-');
      --i;
    } else {
      die("nwalign traceback: invalid pointer value");
    }
  }
  std::reverse(al0.begin(), al0.end());
  std::reverse(al1.begin(), al1.end());
}

// src/nwalign.rs:276-284
static void band_adjust(size_t len1, size_t len2, int32_t band, int32_t& lband, int32_t& rband) {
  if (len2 > len1) {
    lband = band;
    rband = band + int32_t(len2 - len1);
  } else if (len1 > len2) {
    lband = band + int32_t(len1 - len2);
    rband = band;
  } else {
    lband = band;
    rband = band;
  }
}

// src/nwalign.rs:287-308 (BAND_SENTINEL = -9999, src/nwalign.rs:30)
static void fill_band_sentinels(int32_t* d, size_t ncol, size_t len1, size_t len2, int32_t lband,
                                int32_t rband, int32_t band) {
  if (band >= 0 && (band < int32_t(len1) || band < int32_t(len2))) {
    for (size_t i = 0; i <= len1; ++i) {
      int64_t li = int64_t(i) - lband - 1;
      if (li >= 0) d[i * ncol + size_t(li)] = -9999;
      int64_t ri = int64_t(i) + rband + 1;
      if (ri <= int64_t(len2)) d[i * ncol + size_t(ri)] = -9999;
    }
  }
}

// Shared body of align_endsfree_with_buf (src/nwalign.rs:336-417) and
// align_endsfree_homo_with_buf (src/nwalign.rs:435-528). When `homo` is false
// both gap penalties equal gap_p and the masks are ignored.
static void endsfree_core(const uint8_t* s1, size_t len1, const uint8_t* s2, size_t len2,
                          int32_t match, int32_t mismatch, int32_t gap_p, int32_t homo_gap_p,
                          int32_t band, bool homo, AlignBuf& buf) {
  size_t ncol = len2 + 1, nrow = len1 + 1;
  if (homo) {
    homopolymer_mask(s1, len1, buf.homo1);
    homopolymer_mask(s2, len2, buf.homo2);
  }
  buf.d32.assign(nrow * ncol, 0);
  buf.p32.assign(nrow * ncol, 0);
  int32_t* d = buf.d32.data();
  uint8_t* p = buf.p32.data();
  for (size_t i = 0; i <= len1; ++i) p[i * ncol] = 3;
  for (size_t j = 0; j <= len2; ++j) p[j] = 2;
  int32_t lband, rband;
  band_adjust(len1, len2, band, lband, rband);
  fill_band_sentinels(d, ncol, len1, len2, lband, rband, band);
  for (size_t i = 1; i <= len1; ++i) {
    size_t l = band >= 0 ? size_t(std::max<int64_t>(int64_t(i) - lband, 1)) : 1;
    size_t r = band >= 0 ? size_t(std::min<int64_t>(int64_t(i) + rband, int64_t(len2))) : len2;
    for (size_t j = l; j <= r; ++j) {
      int32_t left, up;
      if (i == len1) left = d[i * ncol + j - 1];
      else if (homo && buf.homo2[j - 1]) left = d[i * ncol + j - 1] + homo_gap_p;
      else left = d[i * ncol + j - 1] + gap_p;
      if (j == len2) up = d[(i - 1) * ncol + j];
      else if (homo && buf.homo1[i - 1]) up = d[(i - 1) * ncol + j] + homo_gap_p;
      else up = d[(i - 1) * ncol + j] + gap_p;
      int32_t diag = d[(i - 1) * ncol + j - 1] + (s1[i - 1] == s2[j - 1] ? match : mismatch);
      if (up >= diag && up >= left) {
        d[i * ncol + j] = up;
        p[i * ncol + j] = 3;
      } else if (left >= diag) {
        d[i * ncol + j] = left;
        p[i * ncol + j] = 2;
      } else {
        d[i * ncol + j] = diag;
        p[i * ncol + j] = 1;
      }
    }
  }
  traceback_rowmajor(p, ncol, s1, s2, len1, len2, buf.al0, buf.al1);
}

void align_endsfree(const uint8_t* s1, size_t len1, const uint8_t* s2, size_t len2, int32_t match,
                    int32_t mismatch, int32_t gap_p, int32_t band, AlignBuf& buf) {
  endsfree_core(s1, len1, s2, len2, match, mismatch, gap_p, gap_p, band, false, buf);
}

void align_endsfree_homo(const uint8_t* s1, size_t len1, const uint8_t* s2, size_t len2,
                         const AlignParams& p, AlignBuf& buf) {
  endsfree_core(s1, len1, s2, len2, p.match_score, p.mismatch, p.gap_p, p.homo_gap_p, p.band, true,
                buf);
}

// src/nwalign.rs:645-655
void align_gapless(const uint8_t* s1, size_t len1, const uint8_t* s2, size_t len2, AlignBuf& buf) {
  size_t len = std::max(len1, len2);
  buf.al0.resize(len);
  buf.al1.resize(len);
  for (size_t t = 0; t < len; ++t) {
    buf.al0[t] = t < len1 ? s1[t] : '-';
    buf.al1[t] = t < len2 ? s2[t] : '-';
  }
}

// i16 saturating add (Rust i16::saturating_add).
static inline int16_t sadd16(int16_t a, int16_t b) {
  int32_t s = int32_t(a) + int32_t(b);
  if (s > 32767) s = 32767;
  if (s < -32768) s = -32768;
  return int16_t(s);
}

// src/nwalign.rs:665-739 -- one anti-diagonal. Precedence up>=left>=diag,
// or left>=up>=diag when the inputs were swapped; diag wins only when strictly
// greater.
static inline void dploop(int16_t* d_cur, uint8_t* p_cur, const int16_t* d_prev,
                          const int16_t* diag_buf, size_t left_off, size_t up_off, size_t out_off,
                          size_t col_min, size_t n, int16_t gap_p, bool swap) {
  for (size_t k = 0; k < n; ++k) {
    int16_t l = sadd16(d_prev[left_off + k], gap_p);
    int16_t u = sadd16(d_prev[up_off + k], gap_p);
    int16_t dg = diag_buf[col_min + k];
    int16_t entry;
    uint8_t pe;
    if (swap) {
      if (l >= u) { entry = l; pe = 2; } else { entry = u; pe = 3; }
    } else {
      if (u >= l) { entry = u; pe = 3; } else { entry = l; pe = 2; }
    }
    if (dg > entry) { entry = dg; pe = 1; }
    d_cur[out_off + k] = entry;
    p_cur[out_off + k] = pe;
  }
}

static inline size_t sat_sub1(size_t v) { return v == 0 ? 0 : v - 1; }

// Geometry of the compressed anti-diagonal layout (src/nwalign.rs:775-787).
struct VecGeom {
  bool swap;
  const uint8_t *s1, *s2;
  size_t len1, len2;
  int32_t band;
  size_t bu, start_col, ncol, nrow;
  int16_t fill_val;
};

static VecGeom vec_geom(const uint8_t* s1_in, size_t l1, const uint8_t* s2_in, size_t l2,
                        const VecScores& sc) {
  VecGeom g;
  g.swap = l1 > l2;
  g.s1 = g.swap ? s2_in : s1_in;
  g.s2 = g.swap ? s1_in : s2_in;
  g.len1 = g.swap ? l2 : l1;
  g.len2 = g.swap ? l1 : l2;
  g.band = sc.band < 0 ? int32_t(g.len2) : sc.band;
  g.bu = size_t(g.band);
  g.start_col = 1 + (std::min(g.bu, g.len1) + 1) / 2;
  g.ncol = 2 + g.start_col + std::min(g.bu + g.len2 - g.len1, g.len2) / 2;
  g.nrow = g.len1 + g.len2 + 1;
  int16_t min_score = std::min<int16_t>(std::min<int16_t>(std::min(sc.mismatch, sc.gap_p), sc.match_score), 0);
  g.fill_val = int16_t(uint16_t(uint16_t(0x8000) - uint16_t(min_score)));  // i16::MIN.wrapping_sub
  return g;
}

// src/nwalign.rs:1090-1139 -- traceback through the compressed p matrix.
static void vec_traceback(const VecGeom& g, const uint8_t* p, AlignBuf& buf) {
  std::vector<uint8_t>& al0 = buf.al0;
  std::vector<uint8_t>& al1 = buf.al1;
  al0.clear();
  al1.clear();
  size_t i = g.len1, j = g.len2;
  while (i > 0 || j > 0) {
    int64_t col_signed = 2 * int64_t(g.start_col) + int64_t(j) - int64_t(i);
    ORC_CHECK(col_signed >= 0, "vectorized traceback: negative column");
    size_t col = size_t(col_signed / 2);
    ORC_CHECK((i + j) * g.ncol + col < g.ncol * g.nrow, "vectorized traceback out of range");
    uint8_t v = p[(i + j) * g.ncol + col];
    if (v == 1) {
      ORC_CHECK(i > 0 && j > 0, "vec traceback diag at edge");
      al0.push_back(g.s1[i - 1]);
      al1.push_back(g.s2[j - 1]);
      --i;
      --j;
    } else if (v == 2) {
      ORC_CHECK(j > 0, "vec traceback left at j=0");
      al0.push_back('-');
      al1.push_back(g.s2[j - 1]);
      --j;
    } else if (v == 3) {
      ORC_CHECK(i > 0, "vec traceback up at i=0");
      al0.push_back(g.s1[i - 1]);
      al1.push_back('-');
      --i;
    } else {
      die("vectorized traceback: invalid pointer");
    }
  }
  std::reverse(al0.begin(), al0.end());
  std::reverse(al1.begin(), al1.end());
  if (g.swap) std::swap(buf.al0, buf.al1);
}

// The per-row band bookkeeping shared by both vectorized variants
// (src/nwalign.rs:980-1079 and 2566-2663).
struct VecState {
  size_t col_min, col_max;
  int64_t i_max, j_min;  // j_min carries the reference's wrapping usize as -1
  bool even, recalc_left, recalc_right;
};

static inline void vec_band_transition(const VecGeom& g, size_t row, VecState& s) {
  if (row == std::min(g.bu, g.len1)) {
    s.col_min = sat_sub1(s.col_min);
    s.i_max += 1;
    s.j_min -= 1;
  }
  if (row == std::min(g.bu + g.len2 - g.len1, g.len2)) s.col_max += 1;
}

static inline void vec_advance(const VecGeom& g, size_t row, VecState& s) {
  int32_t band_mod2 = g.band % 2;
  if (int32_t(row) < g.band && int32_t(row) < int32_t(g.len1)) {
    if (s.even) s.col_min = sat_sub1(s.col_min);
    s.i_max += 1;
  } else if (s.i_max < int64_t(g.len1) - 1) {
    if (band_mod2 == 0) {
      if (s.even) s.j_min += 1;
      else s.i_max += 1;
    } else if (s.even) {
      s.col_min = sat_sub1(s.col_min);
      s.i_max += 1;
    } else {
      s.col_min += 1;
      s.j_min += 1;
    }
  } else {
    if (!s.even) s.col_min += 1;
    s.j_min += 1;
  }
  size_t top_limit = std::min(g.bu + g.len2 - g.len1, g.len2);
  if (row < top_limit) {
    if (!s.even) s.col_max += 1;
  } else if ((row + 1) / 2 + s.col_max - g.start_col < g.len2) {
    size_t full_band = g.bu + g.len2 - g.len1;
    if (full_band % 2 == 0) {
      if (s.even) s.col_max = sat_sub1(s.col_max);
      else s.col_max += 1;
    }
  } else if (s.even) {
    s.col_max = sat_sub1(s.col_max);
  }
}

// Fill diag_buf[col_min .. col_min+n) from the row-2 scores (src/nwalign.rs:910-954).
static inline void vec_diag_fill(const VecGeom& g, const VecState& s, size_t n, const int16_t* d_prev2,
                                 int16_t* diag_buf, int16_t match, int16_t mismatch) {
  int64_t nn = int64_t(n);
  int64_t k_lo = std::clamp<int64_t>(s.i_max - int64_t(g.len1) + 1, 0, nn);
  int64_t k_hi = std::clamp<int64_t>(std::min<int64_t>(s.i_max + 1, int64_t(g.len2) - s.j_min), 0, nn);
  k_hi = std::max(k_hi, k_lo);
  for (int64_t k = 0; k < nn; ++k) {
    size_t c = s.col_min + size_t(k);
    if (k < k_lo || k >= k_hi) {
      diag_buf[c] = sadd16(d_prev2[c], g.fill_val);
    } else {
      int64_t si = s.i_max - k, sj = s.j_min + k;
      ORC_CHECK(si >= 0 && si < int64_t(g.len1) && sj >= 0 && sj < int64_t(g.len2),
                "vectorized diag fill out of range");
      int16_t sc = g.s1[si] == g.s2[sj] ? match : mismatch;
      diag_buf[c] = sadd16(d_prev2[c], sc);
    }
  }
}

// src/nwalign.rs:761-1140 -- the shipping 3-row rolling i16 kernel.
void align_vectorized(const uint8_t* s1_in, size_t l1, const uint8_t* s2_in, size_t l2,
                      const VecScores& sc, AlignBuf& buf) {
  VecGeom g = vec_geom(s1_in, l1, s2_in, l2, sc);
  const size_t ncol = g.ncol, nrow = g.nrow;
  const int16_t fill = g.fill_val, egp = sc.end_gap_p, gap = sc.gap_p;
  buf.d16.assign(ncol * 3, 0);
  buf.p8.assign(ncol * nrow, 0);
  buf.diag_buf.assign(ncol, 0);
  uint8_t* p = buf.p8.data();
  int16_t* diag_buf = buf.diag_buf.data();
  int16_t* slots[3] = {buf.d16.data(), buf.d16.data() + ncol, buf.d16.data() + 2 * ncol};
  const size_t left_fill_limit = 1 + std::min(g.bu, g.len1);
  const size_t top_fill_limit = 1 + std::min(g.bu + g.len2 - g.len1, g.len2);
  auto left_col = [&](size_t row) {
    size_t a = g.start_col - 1, b = (row - 1) / 2;
    return a > b ? a - b : 0;
  };
  auto top_col = [&](size_t row) { return g.start_col + row / 2; };
  for (size_t row = 0; row < 2; ++row) {
    int16_t* slot = slots[row];
    slot[0] = fill;
    slot[1] = fill;
    slot[ncol - 2] = fill;
    slot[ncol - 1] = fill;
    if (row == 0) {
      slot[g.start_col] = 0;
    } else {
      if (row < left_fill_limit) {
        slot[left_col(row)] = egp;
        p[row * ncol + left_col(row)] = 3;
      }
      if (row < top_fill_limit) {
        slot[top_col(row)] = egp;
        p[row * ncol + top_col(row)] = 2;
      }
    }
  }
  p[g.start_col] = 0;
  int16_t row_free = egp;

  VecState s{g.start_col, g.start_col, 0, 0, true, false, false};
  for (size_t row = 2; row <= g.len1 + g.len2; ++row) {
    ORC_CHECK(s.col_max >= s.col_min && s.col_max < ncol, "vectorized band range");
    size_t n = s.col_max - s.col_min + 1;
    row_free = sadd16(row_free, egp);
    int16_t* cur = slots[2];
    cur[0] = fill;
    cur[1] = fill;
    cur[ncol - 2] = fill;
    cur[ncol - 1] = fill;
    if (row < left_fill_limit) {
      cur[left_col(row)] = row_free;
      p[row * ncol + left_col(row)] = 3;
    }
    if (row < top_fill_limit) {
      cur[top_col(row)] = row_free;
      p[row * ncol + top_col(row)] = 2;
    }
    vec_diag_fill(g, s, n, slots[0], diag_buf, sc.match_score, sc.mismatch);
    size_t even_off = s.even ? 1 : 0;
    ORC_CHECK(s.col_min >= even_off, "vectorized left offset underflow");
    size_t left_off = s.col_min - even_off;
    size_t up_off = s.col_min + 1 - even_off;
    ORC_CHECK(up_off + n <= ncol, "vectorized up offset overflow");
    dploop(cur, p + row * ncol, slots[1], diag_buf, left_off, up_off, s.col_min, s.col_min, n, gap,
           g.swap);
    vec_band_transition(g, row, s);
    if (egp > gap) {
      if (s.recalc_left) {
        int16_t d_free = sadd16(slots[1][left_off], egp);
        int16_t cv = cur[s.col_min];
        uint8_t pc = p[row * ncol + s.col_min];
        if (d_free > cv) {
          cur[s.col_min] = d_free;
          p[row * ncol + s.col_min] = 2;
        } else if (!(d_free != cv || (!g.swap && pc != 1) || (g.swap && pc == 2))) {
          p[row * ncol + s.col_min] = 2;
        }
      }
      if (s.i_max == int64_t(g.len1) - 1) s.recalc_left = true;
      if (s.recalc_right) {
        size_t idx = up_off + s.col_max - s.col_min;
        ORC_CHECK(idx < ncol, "recalc_right index");
        int16_t d_free = sadd16(slots[1][idx], egp);
        int16_t cv = cur[s.col_max];
        uint8_t pc = p[row * ncol + s.col_max];
        if (d_free > cv) {
          cur[s.col_max] = d_free;
          p[row * ncol + s.col_max] = 3;
        } else if (!(d_free != cv || (!g.swap && pc == 3) || (g.swap && pc != 1))) {
          p[row * ncol + s.col_max] = 3;
        }
      }
      if ((row + 1) / 2 + s.col_max - g.start_col == g.len2) s.recalc_right = true;
    }
    vec_advance(g, row, s);
    int16_t* t = slots[0];
    slots[0] = slots[1];
    slots[1] = slots[2];
    slots[2] = t;
    s.even = !s.even;
  }
  vec_traceback(g, p, buf);
}

// src/nwalign.rs:2375-2719 -- full-matrix reference used only by the
// reference's byte-identity fuzz test.
void align_vectorized_full(const uint8_t* s1_in, size_t l1, const uint8_t* s2_in, size_t l2,
                           const VecScores& sc, AlignBuf& buf) {
  VecGeom g = vec_geom(s1_in, l1, s2_in, l2, sc);
  const size_t ncol = g.ncol, nrow = g.nrow;
  const int16_t fill = g.fill_val, egp = sc.end_gap_p, gap = sc.gap_p;
  std::vector<int16_t> d(ncol * nrow, 0);
  buf.p8.assign(ncol * nrow, 0);
  buf.diag_buf.assign(ncol, 0);
  uint8_t* p = buf.p8.data();
  int16_t* diag_buf = buf.diag_buf.data();
  for (size_t row = 0; row < nrow; ++row) {
    d[row * ncol] = fill;
    d[row * ncol + 1] = fill;
    d[row * ncol + ncol - 2] = fill;
    d[row * ncol + ncol - 1] = fill;
  }
  d[g.start_col] = 0;
  p[g.start_col] = 0;
  {
    size_t row = 1, col = g.start_col - 1;
    int16_t d_free = egp;
    size_t limit = 1 + std::min(g.bu, g.len1);
    while (row < limit) {
      d[row * ncol + col] = d_free;
      p[row * ncol + col] = 3;
      if (row % 2 == 0) col = sat_sub1(col);
      ++row;
      d_free = sadd16(d_free, egp);
    }
  }
  {
    size_t row = 1, col = g.start_col;
    int16_t d_free = egp;
    size_t limit = 1 + std::min(g.bu + g.len2 - g.len1, g.len2);
    while (row < limit) {
      d[row * ncol + col] = d_free;
      p[row * ncol + col] = 2;
      if (row % 2 == 1) ++col;
      ++row;
      d_free = sadd16(d_free, egp);
    }
  }
  VecState s{g.start_col, g.start_col, 0, 0, true, false, false};
  for (size_t row = 2; row <= g.len1 + g.len2; ++row) {
    ORC_CHECK(s.col_max >= s.col_min && s.col_max < ncol, "full vectorized band range");
    size_t n = s.col_max - s.col_min + 1;
    vec_diag_fill(g, s, n, &d[(row - 2) * ncol], diag_buf, sc.match_score, sc.mismatch);
    size_t even_off = s.even ? 1 : 0;
    size_t prev_base = (row - 1) * ncol;
    size_t left_off = prev_base + s.col_min - even_off;
    size_t up_off = prev_base + s.col_min + 1 - even_off;
    dploop(&d[row * ncol], p + row * ncol, &d[prev_base], diag_buf, left_off - prev_base,
           up_off - prev_base, s.col_min, s.col_min, n, gap, g.swap);
    vec_band_transition(g, row, s);
    if (egp > gap) {
      if (s.recalc_left) {
        int16_t d_free = sadd16(d[left_off], egp);
        int16_t cv = d[row * ncol + s.col_min];
        uint8_t pc = p[row * ncol + s.col_min];
        if (d_free > cv) {
          d[row * ncol + s.col_min] = d_free;
          p[row * ncol + s.col_min] = 2;
        } else if (!(d_free != cv || (!g.swap && pc != 1) || (g.swap && pc == 2))) {
          p[row * ncol + s.col_min] = 2;
        }
      }
      if (s.i_max == int64_t(g.len1) - 1) s.recalc_left = true;
      if (s.recalc_right) {
        int16_t d_free = sadd16(d[up_off + s.col_max - s.col_min], egp);
        int16_t cv = d[row * ncol + s.col_max];
        uint8_t pc = p[row * ncol + s.col_max];
        if (d_free > cv) {
          d[row * ncol + s.col_max] = d_free;
          p[row * ncol + s.col_max] = 3;
        } else if (!(d_free != cv || (!g.swap && pc == 3) || (g.swap && pc != 1))) {
          p[row * ncol + s.col_max] = 3;
        }
      }
      if ((row + 1) / 2 + s.col_max - g.start_col == g.len2) s.recalc_right = true;
    }
    vec_advance(g, row, s);
    s.even = !s.even;
  }
  vec_traceback(g, p, buf);
}

// src/nwalign.rs:1169-1224
Sub al2subs(const std::vector<uint8_t>& al0, const std::vector<uint8_t>& al1) {
  ORC_CHECK(al0.size() == al1.size(), "al2subs: unequal alignment rows");
  Sub s;
  size_t alen = al0.size();
  uint32_t len0 = 0;
  for (size_t t = 0; t < alen; ++t)
    if (is_nt(al0[t])) ++len0;
  s.len0 = len0;
  s.map.assign(len0, GAP_GLYPH);
  int64_t i0 = -1, i1 = -1;
  for (size_t t = 0; t < alen; ++t) {
    bool nt0 = is_nt(al0[t]), nt1 = is_nt(al1[t]);
    if (nt0) ++i0;
    if (nt1) ++i1;
    if (nt0) s.map[size_t(i0)] = nt1 ? uint16_t(i1) : GAP_GLYPH;
    if (nt0 && nt1 && al0[t] != al1[t] && al0[t] != 5 && al1[t] != 5) {
      s.pos.push_back(uint16_t(i0));
      s.nt0.push_back(al0[t]);
      s.nt1.push_back(al1[t]);
    }
  }
  return s;
}

// src/nwalign.rs:1244-1414 (raw_align_with_buf + raw_align_dp).
bool raw_align(const Raw& raw1, const Raw& raw2, const AlignParams& p, AlignBuf& buf,
               int32_t* method, double* kdist_out, double* kodist_out) {
  double kdist = 0.0, kodist = -1.0;
  if (p.use_kmers) {
    const int k = p.kmer_size;
    if (raw1.has_kmer8 && raw2.has_kmer8) {
      double d8 = raw1.kmer8_sparse
                      ? kmer_dist8_sparse(raw1.kmer8_sp, raw1.len(), raw2.kmer8_sp, raw2.len(), k)
                      : kmer_dist8(raw1.kmer8.data(), raw1.len(), raw2.kmer8.data(), raw2.len(), k,
                                   raw1.kmer8.size());
      if (d8 < 0.0) {
        std::vector<uint16_t> v1 = assign_kmer(raw1.seq.data(), raw1.len(), k);
        std::vector<uint16_t> v2 = assign_kmer(raw2.seq.data(), raw2.len(), k);
        kdist = kmer_dist(v1.data(), raw1.len(), v2.data(), raw2.len(), k, v1.size());
      } else {
        kdist = d8;
      }
    } else {
      kdist = 0.0;
    }
    if (p.gapless && raw1.has_kord && raw2.has_kord)
      kodist = kord_dist(raw1.kord.data(), raw1.len(), raw2.kord.data(), raw2.len(), k);
  }
  if (kdist_out) *kdist_out = kdist;
  if (kodist_out) *kodist_out = kodist;
  if (p.use_kmers && kdist > p.kdist_cutoff) {
    if (method) *method = M_NONE;
    return false;
  }
  const uint8_t *a = raw1.seq.data(), *b = raw2.seq.data();
  size_t la = raw1.len(), lb = raw2.len();
  if (p.band == 0 || (p.gapless && std::fabs(kodist - kdist) < std::numeric_limits<double>::epsilon())) {
    align_gapless(a, la, b, lb, buf);
    if (method) *method = M_GAPLESS;
    return true;
  }
  bool use_homo = p.homo_gap_p != p.gap_p && p.homo_gap_p <= 0;
  bool too_long = la > 3500 || lb > 3500;
  if (p.vectorized && !too_long && !use_homo) {
    VecScores sc{int16_t(p.match_score), int16_t(p.mismatch), int16_t(p.gap_p), 0, p.band};
    align_vectorized(a, la, b, lb, sc, buf);
    if (method) *method = M_VECTORIZED;
    return true;
  }
  if (use_homo) {
    align_endsfree_homo(a, la, b, lb, p, buf);
    if (method) *method = M_HOMO;
    return true;
  }
  align_endsfree(a, la, b, lb, p.match_score, p.mismatch, p.gap_p, p.band, buf);
  if (method) *method = M_ENDSFREE;
  return true;
}

// src/nwalign.rs:1429-1455 (quality mapping omitted: compute_lambda does not read q0/q1).
bool sub_new(const Raw& raw0, const Raw& raw1, const AlignParams& p, AlignBuf& buf, Sub& out,
             int32_t* method) {
  if (!raw_align(raw0, raw1, p, buf, method, nullptr, nullptr)) return false;
  out = al2subs(buf.al0, buf.al1);
  return true;
}

// ===========================================================================
// pval.rs
// ===========================================================================

// src/pval.rs:253-320 -- ordered left-to-right FP64 product over raw positions.
double compute_lambda(const Raw& raw, const Sub* sub, const double* err_mat, size_t ncol,
                      bool use_quals) {
  if (!sub) return 0.0;
  size_t len = raw.len();
  std::vector<size_t> tvec(len), qind(len);
  for (size_t pos = 0; pos < len; ++pos) {
    unsigned nt = raw.seq[pos];
    ORC_CHECK(nt >= 1 && nt <= 4, "non-ACGT nucleotide reached compute_lambda");
    size_t nti = nt - 1;
    tvec[pos] = nti * 4 + nti;
    qind[pos] = (use_quals && raw.has_qual) ? raw.qual[pos] : 0;
  }
  for (size_t s = 0; s < sub->nsubs(); ++s) {
    size_t pos0 = sub->pos[s];
    size_t pos1 = sub->map[pos0];
    ORC_CHECK(pos1 < len, "sub pos1 beyond raw length");
    size_t n0 = sub->nt0[s] ? sub->nt0[s] - 1 : 0;
    size_t n1 = sub->nt1[s] ? sub->nt1[s] - 1 : 0;
    tvec[pos1] = n0 * 4 + n1;
  }
  double lambda = 1.0;
  for (size_t pos = 0; pos < len; ++pos) lambda = lambda * err_mat[tvec[pos] * ncol + qind[pos]];
  return lambda;
}

// lnGamma as statrs 0.18.0 documents its `ln_gamma`: the Lanczos
// approximation with the parameters of G. R. Pugh, "An Analysis of the Lanczos
// Gamma Approximation" (PhD thesis, UBC 2004, p. 116): r = 10.900511 and the
// eleven coefficients d_0..d_10 below, evaluated for x >= 0.5 as
//   ln(d_0 + sum_{k=1..10} d_k / (x + k - 1)) + ln(2 sqrt(e / pi))
//     + (x - 0.5) ln((x - 0.5 + r) / e),
// the sum accumulated left to right from d_0, each term's divisor formed as
// (x + k) - 1, and e the double nearest Euler's number. Calc_pA only needs
// a >= 1 (a = reads), so the reflection branch for x < 0.5 is not restated.
// Not the C library's lgamma: the two differ by a few ulps (ln_gamma(1) is
// -4.4e-16 here, not 0), which moves p-values by ulps.
double ln_gamma_lanczos(double x) {
  static const double kR = 10.900511;
  static const double kD[11] = {
      2.48574089138753565546e-5,  1.05142378581721974210,     -3.45687097222016235469,
      4.51227709466894823700,     -2.98285225323576655721,    1.05639711577126713077,
      -1.95428773191645869583e-1, 1.70970543404441224307e-2,  -5.71926117404305781283e-4,
      4.63399473359905636708e-6,  -2.71994908488607703910e-9};
  static const double kLn2SqrtEOverPi = 0.6207822376352452;  // ln(2 sqrt(e / pi))
  static const double kE = 2.718281828459045;
  double s = kD[0];
  for (int k = 1; k <= 10; ++k) s = s + kD[k] / (x + double(k) - 1.0);
  return std::log(s) + kLn2SqrtEOverPi + (x - 0.5) * std::log((x - 0.5 + kR) / kE);
}

// Regularised lower incomplete gamma P(a, x). statrs 0.18.0's
// `Poisson::sf(k) = gamma_lr(k + 1, lambda)` (the call site is src/pval.rs:219-223)
// follows the published Cephes igam/igamc method (S. Moshier): a power series
// when x <= 1 or x <= a, otherwise 1 - (Legendre continued fraction for the
// upper tail), with the exponent prefactor a*ln(x) - x - lnGamma(a) tested for
// underflow first, lnGamma being ln_gamma_lanczos above. Before that, statrs
// answers 0.0 for an x within its default accuracy (10 * 2^-53) of zero. No
// reference test fixes calc_pA values, so bit-level agreement with statrs
// rests on this restatement of its documented method.
double gamma_lr(double a, double x) {
  const double eps = 1e-15;
  const double big = 4503599627370496.0;            // 2^52
  const double big_inv = 2.22044604925031308085e-16;  // 2^-52
  const double zero_acc = 1.1102230246251565e-15;     // 10 * 2^-53
  if (std::isnan(a) || std::isnan(x)) return std::numeric_limits<double>::quiet_NaN();
  if (std::fabs(a) < zero_acc) return 1.0;
  if (std::fabs(x) < zero_acc) return 0.0;
  double ax = a * std::log(x) - x - ln_gamma_lanczos(a);
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
  double p3 = 1.0, q3 = x, p2 = x + 1.0, q2 = z * x;
  double ans = p2 / q2;
  for (;;) {
    y += 1.0;
    z += 2.0;
    c += 1.0;
    double yc = y * c;
    double pn = p2 * z - p3 * yc;
    double qn = q2 * z - q3 * yc;
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
      double nextans = pn / qn;
      double err = std::fabs((ans - nextans) / nextans);
      ans = nextans;
      if (err <= eps) break;
    }
  }
  return 1.0 - std::exp(ax) * ans;
}

// src/pval.rs:329-353
static double poisson_upper_tail_direct(uint32_t reads, double lambda) {
  double k = double(reads);
  double log_lambda = std::log(lambda);
  double log_kfact = 0.0;
  for (uint32_t t = 1; t <= reads; ++t) log_kfact += std::log(double(t));
  double log_leading = -lambda + k * log_lambda - log_kfact;
  double series_sum = 1.0, term = 1.0;
  for (uint32_t jj = 1; jj < 10000u; ++jj) {
    term *= lambda / (k + double(jj));
    if (!std::isfinite(term) || term <= 0.0) break;
    double new_sum = series_sum + term;
    if (new_sum == series_sum) break;
    series_sum = new_sum;
  }
  return std::exp(log_leading + std::log(series_sum));
}

// src/pval.rs:208-241 (TAIL_APPROX_CUTOFF = 1e-7, src/pval.rs:18)
double calc_pA(uint32_t reads, double e_reads, bool prior) {
  ORC_CHECK(reads > 0, "calc_pA: reads must be > 0");
  if (!(e_reads > 0.0)) return 1.0;  // Poisson::new rejects lambda <= 0 / NaN
  double pval = gamma_lr(double(reads - 1) + 1.0, e_reads);
  if (pval == 0.0 && e_reads > 0.0) pval = poisson_upper_tail_direct(reads, e_reads);
  if (prior) return pval;
  double norm = 1.0 - std::exp(-e_reads);
  if (norm < 1e-7) norm = e_reads - 0.5 * e_reads * e_reads;
  return pval / norm;
}

// src/pval.rs:376-398
double get_pA(uint32_t reads, bool prior, double lambda, uint32_t hamming, uint32_t bi_reads,
              bool detect_singletons) {
  if (reads == 1 && !prior && !detect_singletons) return 1.0;
  if (hamming == 0) return 1.0;
  if (lambda == 0.0) return 0.0;
  double e_reads = lambda * double(bi_reads);
  return calc_pA(reads, e_reads, prior || detect_singletons);
}

// src/pval.rs:45-130 -- reprice dirty clusters, refresh their bud caches, and
// apply greedy locks once per new cluster.
uint64_t b_p_update(B& b, bool greedy, bool detect_singletons, double min_fold,
                    uint32_t min_hamming, uint32_t min_abund) {
  uint64_t repriced = 0;
  for (size_t i = 0; i < b.clusters.size(); ++i) {
    Bi& bi = b.clusters[i];
    if (bi.update_e) {
      uint32_t bi_reads = bi.reads;
      bool have = false, have_prior = false;
      BudCand bm{}, bmp{};
      for (size_t r = 0; r < bi.raws.size(); ++r) {
        size_t raw_idx = bi.raws[r];
        Raw& raw = b.raws[raw_idx];
        double p = get_pA(raw.reads, raw.prior, raw.comp.lambda, raw.comp.hamming, bi_reads,
                          detect_singletons);
        raw.p = p;
        ++repriced;
        if (r == 0) continue;
        if (raw.reads < min_abund || raw.comp.hamming < min_hamming) continue;
        bool fold_ok = min_fold <= 1.0 || double(raw.reads) >= min_fold * raw.comp.lambda * double(bi_reads);
        if (!fold_ok) continue;
        BudCand cand{p, raw.reads, r, raw_idx};
        if (!have || p < bm.p || (p == bm.p && cand.reads > bm.reads)) {
          bm = cand;
          have = true;
        }
        if (raw.prior && (!have_prior || p < bmp.p || (p == bmp.p && cand.reads > bmp.reads))) {
          bmp = cand;
          have_prior = true;
        }
      }
      bi.has_bud_min = have;
      bi.bud_min = bm;
      bi.has_bud_min_prior = have_prior;
      bi.bud_min_prior = bmp;
      bi.update_e = false;
    }
    if (greedy && bi.check_locks) {
      int64_t center = bi.center;
      uint32_t center_reads = center >= 0 ? b.raws[size_t(center)].reads : 0;
      for (size_t raw_idx : bi.raws) {
        double e_from_center = double(center_reads) * b.raws[raw_idx].comp.lambda;
        if (e_from_center > double(b.raws[raw_idx].reads)) b.raws[raw_idx].lock = true;
        if (int64_t(raw_idx) == center) b.raws[raw_idx].lock = true;
      }
      bi.check_locks = false;
    }
  }
  return repriced;
}

// ===========================================================================
// containers.rs
// ===========================================================================

static Bi new_bi() { return Bi(); }  // src/containers.rs:241-263

// src/containers.rs:337-359
void b_new(B& b, std::vector<Raw>&& raws, double omega_a, double omega_p, bool use_quals) {
  b.raws = std::move(raws);
  b.reads = 0;
  for (size_t t = 0; t < b.raws.size(); ++t) {
    b.reads += b.raws[t].reads;
    b.raws[t].index = uint32_t(t);
  }
  b.e_minmax.assign(b.raws.size(), -999.0);
  b.omega_a = omega_a;
  b.omega_p = omega_p;
  b.use_quals = use_quals;
  b_init(b);
}

// src/containers.rs:363-390
void b_init(B& b) {
  b.clusters.clear();
  Bi bi = new_bi();
  bi.birth_type = BIRTH_INITIAL;
  bi.birth_e = double(b.reads);
  b.clusters.push_back(std::move(bi));
  b.nalign = 0;
  b.nshroud = 0;
  b.raw_cluster.assign(b.raws.size(), 0);
  for (size_t t = 0; t < b.raws.size(); ++t) {
    b.clusters[0].raws.push_back(b.raws[t].index);
    b.clusters[0].reads += b.raws[t].reads;
  }
  b.clusters[0].update_e = true;
  bi_census(b, 0);
  bi_assign_center(b, 0);
}

size_t b_add_cluster(B& b, Bi&& bi) {  // src/containers.rs:394-399
  size_t idx = b.clusters.size();
  bi.i = uint32_t(idx);
  b.clusters.push_back(std::move(bi));
  return idx;
}

void bi_add_raw(B& b, size_t bi_idx, size_t raw_idx) {  // src/containers.rs:403-415
  uint32_t reads = b.raws[raw_idx].reads;
  if (raw_idx < b.raw_cluster.size()) b.raw_cluster[raw_idx] = uint32_t(bi_idx);
  b.clusters[bi_idx].raws.push_back(raw_idx);
  b.clusters[bi_idx].reads += reads;
  b.clusters[bi_idx].update_e = true;
}

size_t bi_pop_raw(B& b, size_t bi_idx, size_t r) {  // src/containers.rs:424-435 (swap_remove)
  std::vector<size_t>& rs = b.clusters[bi_idx].raws;
  ORC_CHECK(r < rs.size(), "bi_pop_raw: index out of range");
  size_t raw_idx = rs[r];
  rs[r] = rs.back();
  rs.pop_back();
  b.clusters[bi_idx].reads -= b.raws[raw_idx].reads;
  b.clusters[bi_idx].update_e = true;
  return raw_idx;
}

void bi_census(B& b, size_t i) {  // src/containers.rs:439-445
  uint32_t reads = 0;
  for (size_t ri : b.clusters[i].raws) reads += b.raws[ri].reads;
  b.clusters[i].reads = reads;
}

// src/containers.rs:450-463 -- max_by_key keeps the LAST maximum on ties.
void bi_assign_center(B& b, size_t i) {
  Bi& bi = b.clusters[i];
  if (bi.raws.empty()) return;
  size_t best = bi.raws[0];
  for (size_t ri : bi.raws)
    if (b.raws[ri].reads >= b.raws[best].reads) best = ri;
  bi.center = int64_t(best);
  bi.seq = b.raws[best].seq;
}

// ===========================================================================
// cluster.rs
// ===========================================================================

static void compare_one(const B& b, size_t center_idx, uint32_t center_reads, size_t index,
                        const double* err_mat, size_t ncol, const AlignParams& p, bool greedy,
                        AlignBuf& buf, CompareItem& out) {
  const Raw& raw = b.raws[index];
  if (greedy && (raw.reads > center_reads || raw.lock)) {
    out = CompareItem{compute_lambda(raw, nullptr, err_mat, ncol, b.use_quals), UINT32_MAX, true, M_NONE};
    return;
  }
  Sub sub;
  int32_t method = M_NONE;
  bool ok = sub_new(b.raws[center_idx], raw, p, buf, sub, &method);
  double lambda = compute_lambda(raw, ok ? &sub : nullptr, err_mat, ncol, b.use_quals);
  out = CompareItem{lambda, ok ? uint32_t(sub.nsubs()) : UINT32_MAX, false, method};
}

// src/cluster.rs:279-330 -- the parallel map (rayon with_max_len(32) becomes
// 32-raw chunks pulled from an atomic counter).
void compare_map(const B& b, size_t i, const double* err_mat, size_t ncol, const AlignParams& p,
                 bool greedy, int nthreads, std::vector<CompareItem>& items) {
  ORC_CHECK(b.clusters[i].center >= 0, "b_compare: cluster has no center");
  size_t center_idx = size_t(b.clusters[i].center);
  uint32_t center_reads = b.raws[center_idx].reads;
  size_t nraw = b.raws.size();
  items.assign(nraw, CompareItem{0.0, UINT32_MAX, false, M_NONE});
  if (nthreads <= 1) {
    AlignBuf buf;
    for (size_t t = 0; t < nraw; ++t)
      compare_one(b, center_idx, center_reads, t, err_mat, ncol, p, greedy, buf, items[t]);
    return;
  }
  const size_t grain = 32;
  std::atomic<size_t> next{0};
  auto worker = [&]() {
    AlignBuf buf;
    for (;;) {
      size_t lo = next.fetch_add(grain);
      if (lo >= nraw) break;
      size_t hi = std::min(nraw, lo + grain);
      for (size_t t = lo; t < hi; ++t)
        compare_one(b, center_idx, center_reads, t, err_mat, ncol, p, greedy, buf, items[t]);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
}

// src/cluster.rs:239-423 (map) + 351-397 (serial store).
CompareStats b_compare_parallel(B& b, size_t i, const double* err_mat, size_t ncol,
                                const AlignParams& p, bool greedy, int nthreads) {
  std::vector<CompareItem> items;
  compare_map(b, i, err_mat, ncol, p, greedy, nthreads, items);
  size_t center_idx = size_t(b.clusters[i].center);
  uint32_t center_reads = b.raws[center_idx].reads;
  double total_reads = double(b.reads);
  CompareStats st;
  for (size_t index = 0; index < items.size(); ++index) {
    const CompareItem& it = items[index];
    if (!it.skipped) {
      ++st.screened;
      ++b.nalign;
      if (it.hamming == UINT32_MAX) ++b.nshroud;
      else ++st.aligned;
    }
    switch (it.method) {
      case M_GAPLESS: ++st.gapless; break;
      case M_VECTORIZED: ++st.vectorized; break;
      case M_HOMO: ++st.homo; break;
      case M_ENDSFREE: ++st.endsfree; break;
      default: break;
    }
    if (index == center_idx) b.clusters[i].self_ = it.lambda;
    if (it.lambda * total_reads > b.e_minmax[index]) {
      double new_e = it.lambda * double(center_reads);
      if (new_e > b.e_minmax[index]) b.e_minmax[index] = new_e;
      Comparison comp{uint32_t(i), uint32_t(index), it.lambda, it.hamming == UINT32_MAX ? 0u : it.hamming};
      b.clusters[i].comp.push_back(comp);
      ++st.stored;
      if (i == 0 || index == center_idx) b.raws[index].comp = comp;
    }
  }
  return st;
}

// src/cluster.rs:731-739
void index_add_cluster(CandIndex& index, const B& b, size_t ci) {
  for (const Comparison& c : b.clusters[ci].comp)
    index[c.index].push_back(Cand{uint32_t(ci), c.lambda, c.hamming});
}

void ShuffleCarry::grow_to(size_t n) {  // src/cluster.rs:891-895
  reads_used.resize(n, 0);
  dirty_cluster.resize(n, 0);
  reads_fell.resize(n, 0);
}

// src/cluster.rs:748-767 -- descending walk because bi_pop_raw swap-removes.
static size_t move_pass_cluster(B& b, size_t ci, const std::vector<Comparison>& compmax) {
  size_t moves = 0;
  size_t r = b.clusters[ci].raws.size();
  while (r > 0) {
    --r;
    size_t raw_idx = b.clusters[ci].raws[r];
    size_t best_ci = compmax[raw_idx].i;
    if (best_ci != ci) {
      if (b.clusters[ci].center == int64_t(raw_idx)) continue;
      bi_pop_raw(b, ci, r);
      bi_add_raw(b, best_ci, raw_idx);
      b.raws[raw_idx].comp = compmax[raw_idx];
      ++moves;
    }
  }
  return moves;
}

// src/cluster.rs:781-783
static inline bool beats(double e, double e_cur, uint32_t ci, uint32_t ci_cur) {
  return e > e_cur || (e == e_cur && ci < ci_cur);
}

// src/cluster.rs:792-810
static void record_change(size_t raw, uint32_t new_ci, const std::vector<Comparison>& compmax,
                          const B& b, ShuffleCarry& c) {
  if (new_ci == compmax[raw].i) return;
  uint32_t cur = b.raw_cluster[raw];
  if (cur != UINT32_MAX && !c.dirty_cluster[cur]) {
    c.dirty_cluster[cur] = 1;
    c.dirty_list.push_back(cur);
  }
}

// src/cluster.rs:819-835
static Comparison best_from_cands_scored(const std::vector<Cand>& cands, size_t raw,
                                         const std::vector<Bi>& clusters, double& best_e) {
  best_e = -std::numeric_limits<double>::infinity();
  Comparison best;
  for (const Cand& c : cands) {
    double e = c.lambda * double(clusters[c.ci].reads);
    if (e > best_e) {
      best_e = e;
      best = Comparison{c.ci, uint32_t(raw), c.lambda, c.hamming};
    }
  }
  return best;
}

// src/cluster.rs:908-1320 (default arms: carry on, prune on, incremental reconcile).
ShuffleResult b_shuffle_converge(B& b, const CandIndex& index, size_t max_shuffle, ShuffleCarry& carry) {
  size_t nraw = b.raws.size();
  bool carried = carry.built;
  if (!carried) {
    carry.compmax.assign(nraw, Comparison());
    carry.emax.assign(nraw, -std::numeric_limits<double>::infinity());
    carry.reads_used.clear();
    carry.dirty_cluster.clear();
    carry.reads_fell.clear();
    carry.grow_to(b.clusters.size());
    for (const Bi& bi : b.clusters) {
      double ci_reads = double(bi.reads);
      for (const Comparison& comp : bi.comp) {
        double e = comp.lambda * ci_reads;
        if (e > carry.emax[comp.index]) {
          carry.emax[comp.index] = e;
          carry.compmax[comp.index] = comp;
        }
      }
    }
    for (size_t ci = 0; ci < b.clusters.size(); ++ci) carry.reads_used[ci] = b.clusters[ci].reads;
    carry.built = true;
  } else {
    carry.grow_to(b.clusters.size());
  }
  carry.in_affected.resize(nraw, 0);

  bool after_reconcile = false;
  bool skip_move = carried;
  size_t total_moves = 0, nshuffle = 0;
  for (;;) {
    if (skip_move) {
      skip_move = false;
      ++nshuffle;
    } else {
      size_t moves = 0;
      if (after_reconcile) {
        std::sort(carry.dirty_list.begin(), carry.dirty_list.end());
        for (size_t k = 0; k < carry.dirty_list.size(); ++k)
          moves += move_pass_cluster(b, carry.dirty_list[k], carry.compmax);
      } else {
        for (size_t ci = 0; ci < b.clusters.size(); ++ci) moves += move_pass_cluster(b, ci, carry.compmax);
      }
      for (uint32_t ci : carry.dirty_list) carry.dirty_cluster[ci] = 0;
      carry.dirty_list.clear();
      carry.dirty_cluster.resize(b.clusters.size(), 0);
      total_moves += moves;
      ++nshuffle;
      if (moves == 0 || nshuffle >= max_shuffle) break;
    }
    // Reconcile pass A1: clusters whose reads fell mark their best-holders for a rescan.
    carry.reads_fell.resize(b.clusters.size(), 0);
    for (size_t ci = 0; ci < carry.reads_used.size(); ++ci) {
      if (b.clusters[ci].reads < carry.reads_used[ci] && !carry.reads_fell[ci]) {
        carry.reads_fell[ci] = 1;
        carry.reads_fell_list.push_back(uint32_t(ci));
      }
    }
    for (uint32_t ci : carry.reads_fell_list) {
      for (const Comparison& comp : b.clusters[ci].comp) {
        size_t raw = comp.index;
        if (carry.compmax[raw].i == ci && !carry.in_affected[raw]) {
          carry.in_affected[raw] = 1;
          carry.affected.push_back(raw);
        }
      }
    }
    // Pass A2: changed clusters in ascending order, incremental test.
    for (size_t ci = 0; ci < b.clusters.size(); ++ci) {
      uint32_t new_reads = b.clusters[ci].reads;
      if (new_reads == carry.reads_used[ci]) continue;
      double reads_f = double(new_reads);
      for (const Comparison& comp : b.clusters[ci].comp) {
        size_t raw = comp.index;
        if (carry.in_affected[raw]) continue;
        double e = comp.lambda * reads_f;
        if (carry.compmax[raw].i == uint32_t(ci)) {
          carry.emax[raw] = e;
        } else if (beats(e, carry.emax[raw], uint32_t(ci), carry.compmax[raw].i)) {
          carry.emax[raw] = e;
          record_change(raw, uint32_t(ci), carry.compmax, b, carry);
          carry.compmax[raw] = comp;
        }
      }
      carry.reads_used[ci] = new_reads;
    }
    // Pass B: full candidate rescan for the marked raws.
    for (size_t raw : carry.affected) {
      double new_e;
      Comparison nb = best_from_cands_scored(index[raw], raw, b.clusters, new_e);
      if (nb.i != carry.compmax[raw].i) record_change(raw, nb.i, carry.compmax, b, carry);
      carry.compmax[raw] = nb;
      carry.emax[raw] = new_e;
      carry.in_affected[raw] = 0;
    }
    carry.affected.clear();
    for (uint32_t ci : carry.reads_fell_list) carry.reads_fell[ci] = 0;
    carry.reads_fell_list.clear();
    after_reconcile = true;
  }
  return ShuffleResult{total_moves, nshuffle};
}

// Pops raw (ci, r) into a new cluster (src/cluster.rs:1566-1621, the shared bud tail).
static size_t bud_tail(B& b, size_t ci, size_t r, size_t raw_idx, double pval, int32_t type) {
  double expected = b.raws[raw_idx].comp.lambda * double(b.clusters[ci].reads);
  Comparison birth_comp = b.raws[raw_idx].comp;
  double birth_fold = double(b.raws[raw_idx].reads) / std::max(expected, std::numeric_limits<double>::min());
  bi_pop_raw(b, ci, r);
  Bi nb = new_bi();
  nb.birth_type = type;
  if (type == BIRTH_ABUNDANCE) nb.birth_from = uint32_t(ci);
  nb.birth_pval = pval;
  nb.birth_fold = birth_fold;
  nb.birth_e = expected;
  nb.birth_comp = birth_comp;
  size_t new_ci = b_add_cluster(b, std::move(nb));
  bi_add_raw(b, new_ci, raw_idx);
  bi_assign_center(b, new_ci);
  return new_ci;
}

// src/cluster.rs:1501-1640
int64_t b_bud_incremental(B& b, double /*min_fold*/, uint32_t /*min_hamming*/, uint32_t /*min_abund*/) {
  double nraw = double(b.raws.size());
  ORC_CHECK(b.clusters[0].center >= 0, "b_bud: cluster 0 has no center");
  size_t init_center = size_t(b.clusters[0].center);
  bool have = false, have_prior = false;
  size_t m_ci = 0, m_r = 0, m_raw = 0, mp_ci = 0, mp_r = 0, mp_raw = 0;
  double min_p = b.raws[init_center].p, min_p_prior = b.raws[init_center].p;
  uint32_t min_reads = b.raws[init_center].reads, min_reads_prior = b.raws[init_center].reads;
  for (size_t ci = 0; ci < b.clusters.size(); ++ci) {
    const Bi& bi = b.clusters[ci];
    if (bi.has_bud_min) {
      const BudCand& c = bi.bud_min;
      if (c.p < min_p || (c.p == min_p && c.reads > min_reads)) {
        have = true;
        m_ci = ci;
        m_r = c.r;
        m_raw = c.raw_idx;
        min_p = c.p;
        min_reads = c.reads;
      }
    }
    if (bi.has_bud_min_prior) {
      const BudCand& c = bi.bud_min_prior;
      if (c.p < min_p_prior || (c.p == min_p_prior && c.reads > min_reads_prior)) {
        have_prior = true;
        mp_ci = ci;
        mp_r = c.r;
        mp_raw = c.raw_idx;
        min_p_prior = c.p;
        min_reads_prior = c.reads;
      }
    }
  }
  double p_a = min_p * nraw;
  double p_p = min_p_prior;
  if (p_a < b.omega_a && have) return int64_t(bud_tail(b, m_ci, m_r, m_raw, p_a, BIRTH_ABUNDANCE));
  if (p_p < b.omega_p && have_prior) return int64_t(bud_tail(b, mp_ci, mp_r, mp_raw, p_p, BIRTH_PRIOR));
  return -1;
}

// ===========================================================================
// dada.rs
// ===========================================================================

static uint8_t nt_encode(char c) {  // src/misc.rs:346-356
  switch (c) {
    case 'A': case 'a': return 1;
    case 'C': case 'c': return 2;
    case 'G': case 'g': return 3;
    case 'T': case 't': case 'U': case 'u': return 4;
    case 'N': case 'n': return 5;
    case '-': return '-';
    default: return 0;
  }
}

static void accumulate(DadaRunStats& rs, const CompareStats& st, size_t nraw) {
  rs.compare_calls++;
  rs.cmp_scanned += nraw;
  rs.screened += st.screened;
  rs.aligned += st.aligned;
  rs.stored += st.stored;
  rs.gapless += st.gapless;
  rs.vectorized += st.vectorized;
  rs.homo += st.homo;
  rs.endsfree += st.endsfree;
}

// src/dada.rs:749-1110 (timers and verbose reporting omitted).
static void run_dada(B& bb, std::vector<Raw>&& raws, const DadaParams& params, const double* err,
                     size_t ncol, DadaRunStats& rs) {
  b_new(bb, std::move(raws), params.omega_a, params.omega_p, params.use_quals);
  AlignParams init_params = params.align;
  init_params.kdist_cutoff = 1.0;
  auto t0 = std::chrono::steady_clock::now();
  CompareStats st = b_compare_parallel(bb, 0, err, ncol, init_params, params.greedy, params.nthreads);
  accumulate(rs, st, bb.raws.size());
  rs.t_compare += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  CandIndex cand(bb.raws.size());
  index_add_cluster(cand, bb, 0);
  b_p_update(bb, params.greedy, params.detect_singletons, params.min_fold, params.min_hamming,
             params.min_abund);
  size_t max_clust = params.max_clust == 0 ? bb.raws.size() : params.max_clust;
  ShuffleCarry carry;
  auto since = [](std::chrono::steady_clock::time_point a) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
  };
  while (bb.clusters.size() < max_clust) {
    t0 = std::chrono::steady_clock::now();
    int64_t newi = b_bud_incremental(bb, params.min_fold, params.min_hamming, params.min_abund);
    rs.t_bud += since(t0);
    if (newi < 0) break;
    t0 = std::chrono::steady_clock::now();
    st = b_compare_parallel(bb, size_t(newi), err, ncol, params.align, params.greedy, params.nthreads);
    accumulate(rs, st, bb.raws.size());
    rs.t_compare += since(t0);
    t0 = std::chrono::steady_clock::now();
    index_add_cluster(cand, bb, size_t(newi));
    ShuffleResult sr = b_shuffle_converge(bb, cand, 10, carry);
    rs.shuffle_calls += sr.calls;
    rs.shuffle_moves += sr.moves;
    rs.t_shuffle += since(t0);
    t0 = std::chrono::steady_clock::now();
    b_p_update(bb, params.greedy, params.detect_singletons, params.min_fold, params.min_hamming,
               params.min_abund);
    rs.t_pupdate += since(t0);
  }
}

// src/dada.rs:243-592 (aux outputs and the learn-errors Raw cache omitted).
std::string dada_uniques(const std::vector<RawInput>& inputs, const DadaParams& params, DadaResult& out) {
  auto t_start = std::chrono::steady_clock::now();
  size_t nraw = inputs.size();
  if (nraw == 0) return "Zero input sequences.";
  size_t maxlen = 0, minlen = SIZE_MAX;
  for (const RawInput& r : inputs) {
    maxlen = std::max(maxlen, r.seq.size());
    minlen = std::min(minlen, r.seq.size());
  }
  if (maxlen >= 9999) return "Input sequences exceed the maximum allowed length (9999).";
  int k = params.align.kmer_size;
  if (k < 3 || k > 8) return "kmer_size out of supported range (3..=8).";
  if (minlen <= size_t(k)) return "All input sequences must be longer than the k-mer size.";
  for (size_t i = 0; i < nraw; ++i) {
    for (char c : inputs[i].seq) {
      if (!(c == 'A' || c == 'C' || c == 'G' || c == 'T' || c == 'U' || c == 'a' || c == 'c' ||
            c == 'g' || c == 't' || c == 'u'))
        return "Sequence " + std::to_string(i) + " contains a non-ACGT base.";
    }
  }
  if (params.err_mat.size() != 16 * params.err_ncol) return "Error matrix length does not match 16 x ncol.";
  bool has_quals = false;
  for (const RawInput& r : inputs) has_quals = has_quals || r.has_quals;
  if (has_quals) {
    for (size_t i = 0; i < nraw; ++i)
      if (inputs[i].has_quals && inputs[i].quals.size() != inputs[i].seq.size())
        return "Sequence " + std::to_string(i) + ": quality length does not match sequence length.";
  }
  // src/dada.rs:337-384 -- extend the error model by repeating its last column.
  std::vector<double> err = params.err_mat;
  size_t ncol = params.err_ncol;
  if (has_quals && params.err_ncol > 0) {
    size_t qmax = 0;
    for (const RawInput& r : inputs) {
      if (!r.has_quals) continue;
      double c = double(std::max<uint32_t>(r.abundance, 1));
      for (uint32_t s : r.quals) qmax = std::max(qmax, size_t(std::llround(std::round(double(s) / c))));
    }
    if (qmax >= params.err_ncol) {
      size_t old = params.err_ncol, nn = qmax + 1;
      std::vector<double> ext(16 * nn, 0.0);
      for (size_t t = 0; t < 16; ++t) {
        for (size_t q = 0; q < old; ++q) ext[t * nn + q] = params.err_mat[t * old + q];
        for (size_t q = old; q < nn; ++q) ext[t * nn + q] = params.err_mat[t * old + old - 1];
      }
      err.swap(ext);
      ncol = nn;
    }
  }
  std::vector<Raw> raws(nraw);
  for (size_t i = 0; i < nraw; ++i) {
    Raw& raw = raws[i];
    const RawInput& in = inputs[i];
    raw.seq.resize(in.seq.size());
    for (size_t t = 0; t < in.seq.size(); ++t) raw.seq[t] = nt_encode(in.seq[t]);
    raw.reads = in.abundance;
    raw.prior = in.prior;
    if (has_quals && in.has_quals) {  // src/containers.rs:128-137
      double c = double(in.abundance);
      raw.qual.resize(in.quals.size());
      for (size_t t = 0; t < in.quals.size(); ++t) {
        double q = std::round(double(in.quals[t]) / c);
        raw.qual[t] = q >= 255.0 ? 255 : (q > 0.0 ? uint8_t(q) : 0);
      }
      raw.has_qual = true;
    }
    raw.index = uint32_t(i);
    if (params.align.use_kmers) raw_assign_kmers(raw, k);
  }
  B bb;
  out = DadaResult();
  run_dada(bb, std::move(raws), params, err.data(), ncol, out.stats);
  // src/dada.rs:502-533 -- final p-values and the read-to-cluster map.
  out.pvals.assign(nraw, 0.0);
  for (size_t ci = 0; ci < bb.clusters.size(); ++ci) {
    const Bi& bi = bb.clusters[ci];
    for (size_t raw_idx : bi.raws) {
      Raw& raw = bb.raws[raw_idx];
      double p;
      bool correct;
      if (int64_t(raw_idx) == bi.center) {
        p = 1.0;
        correct = true;
      } else {
        p = calc_pA(raw.reads, raw.comp.lambda * double(bi.reads), true);
        correct = p >= params.omega_c;
      }
      raw.p = p;
      raw.correct = correct;
      out.pvals[raw.index] = p;
    }
  }
  out.map.assign(nraw, -1);
  for (size_t ci = 0; ci < bb.clusters.size(); ++ci)
    for (size_t raw_idx : bb.clusters[ci].raws)
      if (bb.raws[raw_idx].correct) out.map[bb.raws[raw_idx].index] = int64_t(ci);
  for (const Bi& bi : bb.clusters) {
    ClusterSummary cs;
    cs.sequence = bi.seq;
    cs.reads = bi.reads;
    for (size_t raw_idx : bi.raws) {
      cs.members.push_back(uint32_t(raw_idx));
      cs.member_hammings.push_back(bb.raws[raw_idx].comp.hamming);
      cs.member_lambdas.push_back(bb.raws[raw_idx].comp.lambda);
      cs.member_pvals.push_back(bb.raws[raw_idx].p);
    }
    cs.birth_type = bi.birth_type;
    cs.birth_from = bi.birth_from;
    cs.birth_pval = bi.birth_pval;
    cs.birth_fold = bi.birth_fold;
    cs.birth_e = bi.birth_e;
    cs.birth_hamming = bi.birth_comp.hamming;
    out.clusters.push_back(std::move(cs));
  }
  if (params.transitions) {
    // src/dada.rs:609-617, 648-673: every raw realigned against its cluster's
    // center with the k-mer screen off; then src/error.rs:194-249: for each
    // correct member, every center position aligned to a raw base adds the
    // raw's reads at (4*(center nt) + raw nt, the raw's quality there).
    AlignParams fa = params.align;
    fa.use_kmers = false;
    fa.kdist_cutoff = 1.0;
    const size_t tncol = has_quals ? ncol : 1;
    out.transitions.assign(16 * tncol, 0u);
    out.transitions_ncol = tncol;
    AlignBuf buf;
    for (const Bi& bi : bb.clusters) {
      if (bi.center < 0) continue;
      const Raw& cr = bb.raws[size_t(bi.center)];
      for (size_t raw_idx : bi.raws) {
        const Raw& raw = bb.raws[raw_idx];
        if (!raw.correct) continue;
        Sub sub;
        int32_t method = 0;
        if (!sub_new(cr, raw, fa, buf, sub, &method)) continue;
        for (size_t pos0 = 0; pos0 < cr.seq.size(); ++pos0) {
          if (sub.map[pos0] == GAP_GLYPH) continue;
          const size_t pos1 = sub.map[pos0];
          const size_t nti0 = cr.seq[pos0] ? cr.seq[pos0] - 1u : 0u;
          const size_t nti1 = raw.seq[pos1] ? raw.seq[pos1] - 1u : 0u;
          const size_t qual = has_quals ? (raw.has_qual ? raw.qual[pos1] : 0u) : 0u;
          const size_t t = 4 * nti0 + nti1;
          if (t < 16 && qual < tncol) out.transitions[t * tncol + qual] += raw.reads;
        }
      }
    }
  }
  out.nalign = bb.nalign;
  out.nshroud = bb.nshroud;
  out.nraw = uint32_t(nraw);
  out.stats.t_total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  return std::string();
}

}  // namespace orc

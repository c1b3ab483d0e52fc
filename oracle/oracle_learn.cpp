// Oracle (test infrastructure only; never linked into the product): a CPU
// restatement of dada2-rs 0.2.0's learn-errors loop, used to check the
// product's GPU learn-errors run bit for bit.
//
//   learn_errors       src/learn_errors.rs:739-1020 (init pass 525-616,
//                      detect_nq 494-506, convergence by equality with any
//                      earlier input matrix)
//   build_trans_mat    src/learn_errors.rs:618-738 (center stubs without
//                      k-mer vectors, so no screen and never gapless; q =
//                      min(round(sum / reads), nq - 1); saturating u32 counts)
//   accumulate_trans   src/error_models.rs:495-515 (wrapping u32 sums)
//   loess_errfun       src/error_models.rs:119-210, noqual_errfun 212-261,
//                      expand_err_matrix
//   loess_predict etc. src/loess.rs:29-500
// Parity with the reference is pinned by the reference's own property tests
// (tests/test_learn_errfun.py) but not to its bits: fit_local_at sorts each
// neighbourhood with sort_unstable_by in the reference, and the summation
// order of equally distant points there is the sort's; here ties keep
// ascending x. The product follows the same rule.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <string>
#include <vector>

#include "dada_oracle.hpp"

namespace orc {
namespace {

struct Fit {
  bool ok = false;
  std::vector<double> c;
};

// Gaussian elimination, partial pivoting on the last largest magnitude.
Fit gauss(std::vector<double> a, std::vector<double> b, size_t n) {
  Fit f;
  for (size_t col = 0; col < n; ++col) {
    size_t piv = col;
    for (size_t r = col + 1; r < n; ++r)
      if (std::fabs(a[r * n + col]) >= std::fabs(a[piv * n + col])) piv = r;
    if (piv != col) {
      for (size_t k = 0; k < n; ++k) std::swap(a[col * n + k], a[piv * n + k]);
      std::swap(b[col], b[piv]);
    }
    const double pv = a[col * n + col];
    if (std::fabs(pv) < 1e-12) return f;
    for (size_t row = col + 1; row < n; ++row) {
      const double m = a[row * n + col] / pv;
      a[row * n + col] = 0.0;
      for (size_t k = col + 1; k < n; ++k) a[row * n + k] -= a[col * n + k] * m;
      b[row] -= b[col] * m;
    }
  }
  f.c.assign(n, 0.0);
  for (size_t ii = n; ii-- > 0;) {
    double s = b[ii];
    for (size_t j = ii + 1; j < n; ++j) s -= a[ii * n + j] * f.c[j];
    if (std::fabs(a[ii * n + ii]) < 1e-12) return Fit{};
    f.c[ii] = s / a[ii * n + ii];
  }
  f.ok = true;
  return f;
}

Fit local_fit(double x0, const std::vector<size_t>& valid, const std::vector<double>& x, const std::vector<double>& y,
              const std::vector<double>& w, size_t nloc, size_t p) {
  std::vector<std::pair<double, size_t>> d;
  for (size_t i : valid) d.emplace_back(std::fabs(x[i] - x0), i);
  std::stable_sort(d.begin(), d.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  const double dmax = d[nloc - 1].first;
  std::vector<std::pair<size_t, double>> pts;
  for (size_t t = 0; t < nloc; ++t) {
    const double u = dmax > 0.0 ? d[t].first / dmax : 0.0;
    double tri = 0.0;
    if (u < 1.0) {
      const double v = 1.0 - u * u * u;
      tri = v * v * v;
    }
    const double wt = tri * w[d[t].second];
    if (wt > 0.0) pts.emplace_back(d[t].second, wt);
  }
  std::vector<double> xs;
  for (const auto& e : pts) xs.push_back(x[e.first]);
  std::sort(xs.begin(), xs.end());
  const size_t nd = size_t(std::unique(xs.begin(), xs.end()) - xs.begin());
  for (size_t pe = std::min({p, pts.size(), nd}); pe >= 1; --pe) {
    std::vector<double> ata(pe * pe, 0.0), atb(pe, 0.0), r(pe, 1.0);
    for (const auto& e : pts) {
      const double xi = x[e.first], yi = y[e.first], wt = e.second;
      double xp = xi;
      for (size_t j = 1; j < pe; ++j) {
        r[j] = xp;
        xp *= xi;
      }
      for (size_t j = 0; j < pe; ++j) {
        atb[j] += wt * r[j] * yi;
        for (size_t k = 0; k < pe; ++k) ata[j * pe + k] += wt * r[j] * r[k];
      }
    }
    Fit f = gauss(ata, atb, pe);
    if (f.ok) return f;
  }
  return Fit{};
}

void poly(const std::vector<double>& c, double x, double* v, double* dv) {
  double acc = 0.0, xp = 1.0;
  for (double ci : c) {
    acc += ci * xp;
    xp *= x;
  }
  double der = 0.0, xq = 1.0;
  for (size_t j = 1; j < c.size(); ++j) {
    der += double(j) * c[j] * xq;
    xq *= x;
  }
  *v = acc;
  if (dv) *dv = der;
}

// src/loess.rs:341-466; NaN stands for None.
std::vector<double> loess(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& w,
                          int surface, double cell) {
  const double span = 0.75;
  const size_t degree = 2, n = x.size();
  std::vector<double> out(n, std::numeric_limits<double>::quiet_NaN());
  std::vector<size_t> valid;
  for (size_t i = 0; i < n; ++i)
    if (std::isfinite(y[i]) && w[i] > 0.0) valid.push_back(i);
  const size_t nv = valid.size();
  const size_t eff = std::min(degree, nv ? nv - 1 : 0);
  if (nv <= eff) return out;
  const size_t nloc = std::min(std::max(size_t(std::floor(span * double(nv))), eff + 1), nv);
  const size_t p = eff + 1;
  double lo = std::numeric_limits<double>::infinity(), hi = -lo;
  for (size_t i : valid) {
    lo = std::min(lo, x[i]);
    hi = std::max(hi, x[i]);
  }
  if (surface == 0) {
    for (size_t k = 0; k < n; ++k) {
      if (x[k] < lo || x[k] > hi) continue;
      Fit f = local_fit(x[k], valid, x, y, w, nloc, p);
      if (f.ok) poly(f.c, x[k], &out[k], nullptr);
    }
    return out;
  }
  const size_t thr = std::max(size_t(std::floor(cell * span * double(nv))), p);
  std::vector<double> sx;
  for (size_t i : valid) sx.push_back(x[i]);
  std::sort(sx.begin(), sx.end());
  std::vector<double> vx = {sx.front(), sx.back()};
  std::vector<std::pair<size_t, size_t>> todo = {{0, sx.size() - 1}};
  while (!todo.empty()) {
    auto [l, u] = todo.back();
    todo.pop_back();
    if (u - l + 1 <= thr) continue;
    const size_t m = (l + u) / 2;
    if (m == l || m == u) continue;
    vx.push_back(sx[m]);
    todo.push_back({l, m});
    todo.push_back({m + 1, u});
  }
  std::sort(vx.begin(), vx.end());
  vx.erase(std::unique(vx.begin(), vx.end()), vx.end());
  std::vector<Fit> vf;
  for (double v : vx) vf.push_back(local_fit(v, valid, x, y, w, nloc, p));
  for (size_t k = 0; k < n; ++k) {
    const double x0 = x[k];
    if (x0 < lo || x0 > hi) continue;
    const size_t up = size_t(std::upper_bound(vx.begin(), vx.end(), x0) - vx.begin());
    size_t a_i = up == 0 ? 0 : (up >= vx.size() ? vx.size() - 2 : up - 1);
    size_t b_i = up == 0 ? std::min<size_t>(1, vx.size() - 1) : (up >= vx.size() ? vx.size() - 1 : up);
    if (vx.size() == 1) a_i = b_i = 0;  // one vertex: the reference's index underflows (it panics)
    if (!vf[a_i].ok || !vf[b_i].ok) continue;
    const double a = vx[a_i], b = vx[b_i];
    double fa, da, fb, db;
    poly(vf[a_i].c, a, &fa, &da);
    poly(vf[b_i].c, b, &fb, &db);
    if (a == b) {
      out[k] = fa;
      continue;
    }
    const double h = (x0 - a) / (b - a), g = 1.0 - h;
    out[k] = g * g * (1.0 + 2.0 * h) * fa + h * h * (3.0 - 2.0 * h) * fb +
             (h * g * g * da + h * h * (h - 1.0) * db) * (b - a);
  }
  return out;
}

void fill_ends(std::vector<double>& v) {
  size_t first = v.size(), last = v.size();
  for (size_t i = 0; i < v.size(); ++i)
    if (!std::isnan(v[i])) {
      if (first == v.size()) first = i;
      last = i;
    }
  if (first == v.size()) return;
  for (size_t i = 0; i < first; ++i) v[i] = v[first];
  for (size_t i = last + 1; i < v.size(); ++i) v[i] = v[last];
}

double clampr(double r, const ErrFunSpec& e) {
  if (r < e.min_error_rate) return e.min_error_rate;
  if (r > e.max_error_rate) return e.max_error_rate;
  return r;
}

void expand12(const std::vector<double>& off, size_t nq, std::vector<double>& err) {
  err.assign(16 * nq, 0.0);
  const size_t rows[4][3] = {{1, 2, 3}, {4, 6, 7}, {8, 9, 11}, {12, 13, 14}};
  const size_t diag[4] = {0, 5, 10, 15};
  for (size_t g = 0; g < 4; ++g)
    for (size_t q = 0; q < nq; ++q) {
      const double a = off[(3 * g) * nq + q], b = off[(3 * g + 1) * nq + q], c = off[(3 * g + 2) * nq + q];
      err[rows[g][0] * nq + q] = a;
      err[rows[g][1] * nq + q] = b;
      err[rows[g][2] * nq + q] = c;
      err[diag[g] * nq + q] = 1.0 - a - b - c;
    }
}

}  // namespace

// loess_errfun (src/error_models.rs:119-210) over the nq columns of trans.
static std::string loess_fit(const ErrFunSpec& e, const std::vector<uint32_t>& trans, size_t nq,
                             std::vector<double>& err) {
  std::vector<double> off(12 * nq, 0.0);
  std::vector<double> x(nq), tot(nq), yl(nq);
  for (size_t q = 0; q < nq; ++q) x[q] = double(q);
  size_t o = 0, failed = 0;
  for (size_t i = 0; i < 4; ++i) {
    for (size_t q = 0; q < nq; ++q)
      tot[q] = double(trans[(i * 4) * nq + q]) + double(trans[(i * 4 + 1) * nq + q]) +
               double(trans[(i * 4 + 2) * nq + q]) + double(trans[(i * 4 + 3) * nq + q]);
    for (size_t j = 0; j < 4; ++j) {
      if (i == j) continue;
      for (size_t q = 0; q < nq; ++q)
        yl[q] = tot[q] == 0.0 ? std::numeric_limits<double>::quiet_NaN()
                              : std::log10((double(trans[(i * 4 + j) * nq + q]) + 1.0) / tot[q]);
      std::vector<double> pr = loess(x, yl, tot, e.surface, e.cell);
      fill_ends(pr);
      bool any = false;
      for (double v : pr) any = any || std::isfinite(v);
      if (!any) ++failed;
      for (size_t q = 0; q < nq; ++q)
        off[o * nq + q] = clampr(std::isfinite(pr[q]) ? std::pow(10.0, pr[q]) : e.min_error_rate, e);
      ++o;
    }
  }
  if (failed == 12) return "LOESS fit failed for all 12 transitions";
  expand12(off, nq, err);
  return std::string();
}

// A quality anchor as Rust's `f64 as usize` gives it: NaN and negatives to 0,
// truncation toward zero otherwise (saturating).
static size_t anchor_index(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 18446744073709551615.0) return std::numeric_limits<size_t>::max();
  return size_t(v);
}

// Rust's `{}` of an f64 for the messages: integral values without a point.
static std::string rust_f64(double v) {
  if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
  if (std::isnan(v)) return "NaN";
  char b[64];
  if (v == std::floor(v) && std::fabs(v) < 1e15) std::snprintf(b, sizeof b, "%.0f", v);
  else std::snprintf(b, sizeof b, "%.17g", v);
  return b;
}

// binned_qual_errfun (src/error_models.rs:263-396): per off-diagonal
// transition, the observed rate at each anchor quality, linear between
// adjacent anchors, flat beyond the outer ones; quality scores are 0..nq-1
// (src/learn_errors.rs:87). Unsorted anchors, on which the reference's
// unsigned step count underflows, are refused.
static std::string binned_fit(const ErrFunSpec& e, const std::vector<uint32_t>& trans, size_t nq,
                              std::vector<double>& err) {
  double qmin = std::numeric_limits<double>::infinity(), qmax = -qmin;
  bool observed = false;
  for (size_t q = 0; q < nq; ++q) {
    double t = 0.0;
    for (size_t r = 0; r < 16; ++r) t += double(trans[r * nq + q]);
    if (t > 0.0) {
      observed = true;
      qmin = std::min(qmin, double(q));
      qmax = std::max(qmax, double(q));
    }
  }
  if (!observed) return "No observed transitions";
  double bmin = std::numeric_limits<double>::infinity(), bmax = -bmin;
  for (double b : e.bins) {
    bmax = std::max(bmax, b);
    bmin = std::min(bmin, b);
  }
  if (qmax > bmax)
    return "Input data contains quality score " + rust_f64(qmax) + " higher than max binned value " + rust_f64(bmax);
  if (qmin < bmin)
    return "Input data contains quality score " + rust_f64(qmin) + " lower than min binned value " + rust_f64(bmin);
  std::vector<double> off(12 * nq, 0.0);
  size_t o = 0;
  for (size_t i = 0; i < 4; ++i) {
    std::vector<double> tot(nq, 0.0);
    for (size_t q = 0; q < nq; ++q)
      for (size_t j = 0; j < 4; ++j) tot[q] += double(trans[(i * 4 + j) * nq + q]);
    for (size_t j = 0; j < 4; ++j) {
      if (i == j) continue;
      std::vector<double> p(nq), pred(nq, std::numeric_limits<double>::quiet_NaN());
      for (size_t q = 0; q < nq; ++q)
        p[q] = tot[q] > 0.0 ? double(trans[(i * 4 + j) * nq + q]) / tot[q] : std::numeric_limits<double>::quiet_NaN();
      for (size_t k = 0; k + 1 < e.bins.size(); ++k) {
        const size_t lo = anchor_index(e.bins[k]), hi = anchor_index(e.bins[k + 1]);
        if (lo >= nq || hi >= nq) continue;
        if (hi < lo) return "binned quality scores must be ascending";
        const double lp = p[lo], hp = p[hi];
        if (!std::isfinite(lp) || !std::isfinite(hp)) continue;
        const size_t steps = hi - lo + 1;
        for (size_t s = 0; s < steps; ++s) {
          const double t = steps > 1 ? double(s) / double(steps - 1) : 0.0;
          pred[lo + s] = lp * (1.0 - t) + hp * t;
        }
      }
      fill_ends(pred);
      for (size_t q = 0; q < nq; ++q) off[o * nq + q] = std::isfinite(pred[q]) ? clampr(pred[q], e) : e.min_error_rate;
      ++o;
    }
  }
  expand12(off, nq, err);
  return std::string();
}

// pacbio_errfun (src/error_models.rs:408-462): with a Q93 column (quality
// scores 0..nq-1, so nq = 94), LOESS over columns 0..92 and (count + 1) /
// (source total + 4) for every entry of column 93; otherwise LOESS.
static std::string pacbio_fit(const ErrFunSpec& e, const std::vector<uint32_t>& trans, size_t nq,
                              std::vector<double>& err) {
  if (nq != 94) return loess_fit(e, trans, nq, err);
  const size_t sub = nq - 1;
  std::vector<uint32_t> ts(16 * sub);
  for (size_t r = 0; r < 16; ++r)
    for (size_t q = 0; q < sub; ++q) ts[r * sub + q] = trans[r * nq + q];
  std::vector<double> es;
  const std::string m = loess_fit(e, ts, sub, es);
  if (!m.empty()) return m;
  err.assign(16 * nq, 0.0);
  for (size_t r = 0; r < 16; ++r)
    for (size_t q = 0; q < sub; ++q) err[r * nq + q] = es[r * sub + q];
  for (size_t i = 0; i < 4; ++i) {
    double t93 = 0.0;
    for (size_t j = 0; j < 4; ++j) t93 += double(trans[(i * 4 + j) * nq + sub]);
    for (size_t j = 0; j < 4; ++j) err[(i * 4 + j) * nq + sub] = (double(trans[(i * 4 + j) * nq + sub]) + 1.0) / (t93 + 4.0);
  }
  return std::string();
}

std::string errfun_apply(const ErrFunSpec& e, const std::vector<uint32_t>& trans, size_t nq, std::vector<double>& err) {
  std::vector<double> off(12 * nq, 0.0);
  if (e.kind == 1) {  // noqual
    double obs[16];
    for (size_t r = 0; r < 16; ++r) {
      double s = 0.0;
      for (size_t q = 0; q < nq; ++q) s += double(trans[r * nq + q]);
      obs[r] = s + e.pseudocount;
    }
    size_t o = 0;
    for (size_t i = 0; i < 4; ++i) {
      const double tot = obs[i * 4] + obs[i * 4 + 1] + obs[i * 4 + 2] + obs[i * 4 + 3];
      for (size_t j = 0; j < 4; ++j) {
        if (i == j) continue;
        const double rate = tot > 0.0 ? clampr(obs[i * 4 + j] / tot, e) : e.min_error_rate;
        for (size_t q = 0; q < nq; ++q) off[o * nq + q] = rate;
        ++o;
      }
    }
    expand12(off, nq, err);
    return std::string();
  }
  if (e.kind == 4) return "external_errfun runs a user command: not restated here";
  if (e.kind == 2) return binned_fit(e, trans, nq, err);
  if (e.kind == 3) return pacbio_fit(e, trans, nq, err);
  return loess_fit(e, trans, nq, err);
}

// src/learn_errors.rs:618-738
std::vector<uint32_t> build_trans_mat(const std::vector<RawInput>& inputs, const DadaResult& res,
                                      const AlignParams& ap, size_t nq) {
  std::vector<uint32_t> trans(16 * nq, 0u);
  std::vector<Raw> centers(res.clusters.size());
  for (size_t c = 0; c < centers.size(); ++c) centers[c].seq = res.clusters[c].sequence;
  AlignBuf buf;
  for (size_t i = 0; i < inputs.size(); ++i) {
    if (res.map[i] < 0 || !inputs[i].has_quals) continue;
    const RawInput& in = inputs[i];
    Raw q;
    q.seq.resize(in.seq.size());
    for (size_t t = 0; t < in.seq.size(); ++t) {
      const char ch = in.seq[t];
      q.seq[t] = ch == 'A' || ch == 'a' ? 1 : ch == 'C' || ch == 'c' ? 2 : ch == 'G' || ch == 'g' ? 3 : 4;
    }
    q.reads = in.abundance;
    if (!raw_align(centers[size_t(res.map[i])], q, ap, buf, nullptr, nullptr, nullptr)) continue;
    const double cnt = double(in.abundance);
    size_t qpos = 0;
    for (size_t k = 0; k < buf.al0.size(); ++k) {
      const uint8_t n0 = buf.al0[k], n1 = buf.al1[k];
      if (n0 >= 1 && n0 <= 4 && n1 >= 1 && n1 <= 4) {
        const size_t qq = std::min(size_t(std::round(double(in.quals[qpos]) / cnt)), nq - 1);
        uint32_t& cell = trans[(size_t(n0 - 1) * 4 + (n1 - 1)) * nq + qq];
        const uint64_t s = uint64_t(cell) + in.abundance;
        cell = s > 0xffffffffull ? 0xffffffffu : uint32_t(s);
      }
      if (n1 != '-') ++qpos;
    }
  }
  return trans;
}

// src/learn_errors.rs:494-506, 525-616, 739-1020
std::string learn_errors(const std::vector<std::vector<RawInput>>& samples, DadaParams params, const ErrFunSpec& ef,
                         size_t max_consist, LearnResult& out) {
  uint32_t qmax = 0;
  bool any_q = false;
  for (const auto& s : samples)
    for (const auto& r : s)
      if (r.has_quals)
        for (uint32_t v : r.quals) {
          any_q = true;
          qmax = std::max(qmax, uint32_t(std::round(double(v) / double(r.abundance))));
        }
  const size_t nq = (any_q ? size_t(qmax) : 40) + 1;
  out.nq = nq;
  params.err_ncol = nq;
  params.transitions = false;
  auto pass = [&](const std::vector<double>& err, std::vector<uint32_t>& acc) -> std::string {
    params.err_mat = err;
    acc.assign(16 * nq, 0u);
    for (const auto& s : samples) {
      DadaResult r;
      std::string m = dada_uniques(s, params, r);
      if (!m.empty()) return m;
      std::vector<uint32_t> t = build_trans_mat(s, r, params.align, nq);
      for (size_t b = 0; b < acc.size(); ++b) acc[b] += t[b];
    }
    return std::string();
  };
  std::vector<uint32_t> acc;
  const size_t keep = params.max_clust;
  params.max_clust = 1;
  std::string m = pass(std::vector<double>(16 * nq, 1.0), acc);
  params.max_clust = keep;
  if (!m.empty()) return m;
  std::vector<double> err;
  m = errfun_apply(ef, acc, nq, err);
  if (!m.empty()) return m;
  for (size_t r : {size_t(0), size_t(5), size_t(10), size_t(15)})
    for (size_t q = 0; q < nq; ++q) err[r * nq + q] = 1.0;
  out.trans.assign(16 * nq, 0u);
  out.err_in = err;
  out.err_out = err;
  out.passes = 0;
  out.converged = false;
  std::vector<std::vector<double>> seen;
  for (size_t it = 0; it < max_consist; ++it) {
    out.passes = it + 1;
    seen.push_back(err);
    m = pass(err, acc);
    if (!m.empty()) return m;
    std::vector<double> fit;
    m = errfun_apply(ef, acc, nq, fit);
    if (!m.empty()) return m;
    bool conv = false;
    for (const auto& h : seen) conv = conv || h == fit;
    out.err_in = err;
    out.trans = acc;
    out.err_out = fit;
    if (conv) {
      out.converged = true;
      break;
    }
    err = fit;
  }
  return std::string();
}

}  // namespace orc

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

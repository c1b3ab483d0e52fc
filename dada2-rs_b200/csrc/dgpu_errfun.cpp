// Error-model fits of the learn-errors loop: the 16 x nq error-rate matrix
// estimated from a 16 x nq transition-count matrix (row 4 * ref nt + query
// nt, column = quality score). Host code; the loop calls it once per pass.
//
// Restated from dada2-rs 0.2.0 with the same floating-point operations in
// the same order:
//   loess_errfun      src/error_models.rs:119-210 (log10 rates, weights =
//                     counts of the source nucleotide, span 0.75, degree 2,
//                     flat extrapolation, clamp to [min, max] error rate)
//   noqual_errfun     src/error_models.rs:212-261
//   expand_err_matrix src/error_models.rs (12 off-diagonal rows -> 16 rows,
//                     diagonal = 1 - the three off-diagonals)
//   loess_predict, fit_local_at, solve_linear, build_kd_vertices_1d,
//   eval_poly(_and_deriv), extrapolate_flat    src/loess.rs:29-500
// One deliberate difference: fit_local_at orders each neighbourhood by
// distance with a stable sort (ties in distance keep ascending x), where the
// reference uses sort_unstable_by. The neighbourhood and its weights are the
// same either way; only the summation order of equally distant points in the
// normal equations can differ, which moves a fitted rate by at most a few
// ulps.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "dada2_b200.h"

namespace dgpu {

void set_last_error(const char* msg);
int external_errfun_fit(const char* cmd, const uint32_t* trans, int nq, double* err, std::string* msg);

namespace {

// Gaussian elimination with partial pivoting on the row-major n x n matrix a
// (src/loess.rs:29-76). The pivot is the last row of largest magnitude in the
// column (Iterator::max_by keeps the last of equals); a pivot or diagonal
// below 1e-12 in magnitude makes the system singular.
bool solve_linear(std::vector<double>& a, std::vector<double>& b, int n, std::vector<double>& x) {
  for (int col = 0; col < n; ++col) {
    int pr = col;
    for (int r = col + 1; r < n; ++r)
      if (!(std::fabs(a[size_t(r) * n + col]) < std::fabs(a[size_t(pr) * n + col]))) pr = r;
    if (pr != col) {
      for (int k = 0; k < n; ++k) std::swap(a[size_t(col) * n + k], a[size_t(pr) * n + k]);
      std::swap(b[col], b[pr]);
    }
    const double pivot = a[size_t(col) * n + col];
    if (std::fabs(pivot) < 1e-12) return false;
    for (int row = col + 1; row < n; ++row) {
      const double f = a[size_t(row) * n + col] / pivot;
      a[size_t(row) * n + col] = 0.0;
      for (int k = col + 1; k < n; ++k) {
        const double v = a[size_t(col) * n + k] * f;
        a[size_t(row) * n + k] -= v;
      }
      const double bv = b[col] * f;
      b[row] -= bv;
    }
  }
  x.assign(n, 0.0);
  for (int i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int j = i + 1; j < n; ++j) s -= a[size_t(i) * n + j] * x[j];
    const double diag = a[size_t(i) * n + i];
    if (std::fabs(diag) < 1e-12) return false;
    x[i] = s / diag;
  }
  return true;
}

double cube(double u) { return u * u * u; }

// Local weighted polynomial at x0 over the n_local nearest valid points,
// tricube weights times the observation weights, degree lowered while the
// surviving points cannot support it (src/loess.rs:177-250).
bool fit_local_at(double x0, const std::vector<int>& valid, const std::vector<double>& xs,
                  const std::vector<double>& ys, const std::vector<double>& weights, int n_local, int p,
                  std::vector<double>& coeffs) {
  std::vector<std::pair<int, double>> dists;
  dists.reserve(valid.size());
  for (int i : valid) dists.emplace_back(i, std::fabs(xs[i] - x0));
  std::stable_sort(dists.begin(), dists.end(),
                   [](const std::pair<int, double>& a, const std::pair<int, double>& b) { return a.second < b.second; });
  const double max_dist = dists[size_t(n_local) - 1].second;
  std::vector<std::pair<int, double>> ws;
  for (int t = 0; t < n_local; ++t) {
    const int i = dists[t].first;
    const double d = dists[t].second;
    const double u = max_dist > 0.0 ? d / max_dist : 0.0;
    const double tri = u < 1.0 ? cube(1.0 - cube(u)) : 0.0;
    const double w = tri * weights[i];
    if (w > 0.0) ws.emplace_back(i, w);
  }
  std::vector<double> distinct;
  for (const auto& e : ws) distinct.push_back(xs[e.first]);
  std::sort(distinct.begin(), distinct.end());
  distinct.erase(std::unique(distinct.begin(), distinct.end()), distinct.end());
  int pe = std::min({p, int(ws.size()), int(distinct.size())});
  std::vector<double> xtx, xty, row;
  while (pe >= 1) {
    xtx.assign(size_t(pe) * pe, 0.0);
    xty.assign(pe, 0.0);
    row.assign(pe, 1.0);
    for (const auto& e : ws) {
      const double xi = xs[e.first], yi = ys[e.first], w = e.second;
      double xpow = xi;
      for (int j = 1; j < pe; ++j) {
        row[j] = xpow;
        xpow *= xi;
      }
      for (int j = 0; j < pe; ++j) {
        xty[j] += w * row[j] * yi;
        for (int k = 0; k < pe; ++k) xtx[size_t(j) * pe + k] += w * row[j] * row[k];
      }
    }
    if (solve_linear(xtx, xty, pe, coeffs)) return true;
    --pe;
  }
  return false;
}

double eval_poly(const std::vector<double>& c, double x) {
  double acc = 0.0, xpow = 1.0;
  for (double v : c) {
    acc += v * xpow;
    xpow *= x;
  }
  return acc;
}

void eval_poly_and_deriv(const std::vector<double>& c, double x, double* val, double* der) {
  double v = 0.0, xpow = 1.0;
  for (double cc : c) {
    v += cc * xpow;
    xpow *= x;
  }
  double d = 0.0, xd = 1.0;
  for (size_t j = 1; j < c.size(); ++j) {
    d += double(j) * c[j] * xd;
    xd *= x;
  }
  *val = v;
  *der = d;
}

// Vertices of the 1-D kd-tree partition of the sorted valid xs: a cell of
// more than `threshold` points splits at its median rank m = (l + u) / 2,
// the vertex being that point's x (src/loess.rs:271-305).
std::vector<double> kd_vertices(const std::vector<double>& sx, size_t threshold) {
  const size_t n = sx.size();
  std::vector<double> v = {sx[0], sx[n - 1]};
  std::vector<std::pair<size_t, size_t>> stack = {{0, n - 1}};
  while (!stack.empty()) {
    const auto [l, u] = stack.back();
    stack.pop_back();
    if (u - l + 1 <= threshold) continue;
    const size_t m = (l + u) / 2;
    if (m == l || m == u) continue;
    v.push_back(sx[m]);
    stack.emplace_back(l, m);
    stack.emplace_back(m + 1, u);
  }
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  return v;
}

// LOESS of ys on xs with observation weights (src/loess.rs:341-466): span
// 0.75 of the valid points (finite y, positive weight) as the neighbourhood,
// `degree`; NaN where no fit exists (outside the valid x range or singular).
std::vector<double> loess_predict(const std::vector<double>& xs, const std::vector<double>& ys,
                                  const std::vector<double>& weights, double span, int degree, int surface,
                                  double cell) {
  const int n = int(xs.size());
  const double nan = std::numeric_limits<double>::quiet_NaN();
  std::vector<double> out(n, nan);
  std::vector<int> valid;
  for (int i = 0; i < n; ++i)
    if (std::isfinite(ys[i]) && weights[i] > 0.0) valid.push_back(i);
  const int nv = int(valid.size());
  const int eff = std::min(degree, nv > 0 ? nv - 1 : 0);
  if (nv <= eff) return out;
  const int n_local = std::min(std::max(int(std::floor(span * double(nv))), eff + 1), nv);
  const int p = eff + 1;
  double x_min = std::numeric_limits<double>::infinity(), x_max = -std::numeric_limits<double>::infinity();
  for (int i : valid) {
    x_min = std::min(x_min, xs[i]);
    x_max = std::max(x_max, xs[i]);
  }
  std::vector<double> c;
  if (surface == 0) {  // direct: one local fit per query
    for (int k = 0; k < n; ++k) {
      const double x0 = xs[k];
      if (x0 < x_min || x0 > x_max) continue;
      if (fit_local_at(x0, valid, xs, ys, weights, n_local, p, c)) out[k] = eval_poly(c, x0);
    }
    return out;
  }
  // interpolate: fits at the kd-tree vertices, cubic Hermite blend between
  // the two vertices around each query (R's ehg128)
  size_t threshold = size_t(std::floor(cell * span * double(nv)));
  threshold = std::max(threshold, size_t(p));
  std::vector<double> sx;
  for (int i : valid) sx.push_back(xs[i]);
  std::sort(sx.begin(), sx.end());
  const std::vector<double> vert = kd_vertices(sx, threshold);
  std::vector<std::vector<double>> vc(vert.size());
  std::vector<uint8_t> vok(vert.size(), 0);
  for (size_t v = 0; v < vert.size(); ++v) vok[v] = fit_local_at(vert[v], valid, xs, ys, weights, n_local, p, vc[v]);
  for (int k = 0; k < n; ++k) {
    const double x0 = xs[k];
    if (x0 < x_min || x0 > x_max) continue;
    const size_t upper = size_t(std::upper_bound(vert.begin(), vert.end(), x0) - vert.begin());
    size_t lo, hi;
    if (vert.size() == 1) {  // one distinct valid x: the reference's index underflows (a panic)
      lo = hi = 0;
    } else if (upper == 0) {
      lo = 0;
      hi = std::min<size_t>(1, vert.size() - 1);
    } else if (upper >= vert.size()) {
      lo = vert.size() - 2;
      hi = vert.size() - 1;
    } else {
      lo = upper - 1;
      hi = upper;
    }
    if (!vok[lo] || !vok[hi]) continue;
    const double a = vert[lo], b = vert[hi];
    double fa, fpa, fb, fpb;
    eval_poly_and_deriv(vc[lo], a, &fa, &fpa);
    eval_poly_and_deriv(vc[hi], b, &fb, &fpb);
    if (a == b) {
      out[k] = fa;
      continue;
    }
    const double h = (x0 - a) / (b - a);
    const double omh = 1.0 - h;
    const double phi0 = omh * omh * (1.0 + 2.0 * h);
    const double phi1 = h * h * (3.0 - 2.0 * h);
    const double psi0 = h * omh * omh;
    const double psi1 = h * h * (h - 1.0);
    out[k] = phi0 * fa + phi1 * fb + (psi0 * fpa + psi1 * fpb) * (b - a);
  }
  return out;
}

// NaN ends filled with the first / last finite prediction (src/loess.rs:468-498).
void extrapolate_flat(std::vector<double>& v) {
  int first = -1, last = -1;
  for (int i = 0; i < int(v.size()); ++i)
    if (!std::isnan(v[i])) {
      if (first < 0) first = i;
      last = i;
    }
  if (first < 0) return;
  for (int i = 0; i < first; ++i) v[i] = v[first];
  for (int i = last + 1; i < int(v.size()); ++i) v[i] = v[last];
}

double clamp_rate(double r, const dgpu_errfun& ef) { return std::min(std::max(r, ef.min_error_rate), ef.max_error_rate); }

// 12 off-diagonal rows (A->C, A->G, A->T, C->A, C->G, C->T, G->A, G->C,
// G->T, T->A, T->C, T->G) to the 16-row matrix with each diagonal the
// remainder 1 - the three off-diagonals of its source nucleotide.
void expand(const std::vector<double>& off, int nq, double* err) {
  static const int dest[4][3] = {{1, 2, 3}, {4, 6, 7}, {8, 9, 11}, {12, 13, 14}};
  static const int diag[4] = {0, 5, 10, 15};
  for (int g = 0; g < 4; ++g)
    for (int q = 0; q < nq; ++q) {
      const double v0 = off[size_t(3 * g) * nq + q], v1 = off[size_t(3 * g + 1) * nq + q],
                   v2 = off[size_t(3 * g + 2) * nq + q];
      err[size_t(dest[g][0]) * nq + q] = v0;
      err[size_t(dest[g][1]) * nq + q] = v1;
      err[size_t(dest[g][2]) * nq + q] = v2;
      err[size_t(diag[g]) * nq + q] = 1.0 - v0 - v1 - v2;
    }
}

// LOESS per off-diagonal transition over the nq columns of trans (row 4i+j,
// column q) into err. Returns 0, or DGPU_E_INVALID with *msg when the fit
// fails for all twelve transitions (src/error_models.rs:186-201).
int loess_fit(const dgpu_errfun& ef, const uint32_t* trans, int nq, double* err, std::string* msg) {
  std::vector<double> off(size_t(12) * nq, 0.0);
  std::vector<double> xs(nq), tot(nq), rlogp(nq);
  for (int q = 0; q < nq; ++q) xs[q] = double(q);
  int orow = 0, failed = 0;
  for (int i = 0; i < 4; ++i) {
    for (int q = 0; q < nq; ++q) {
      double s = 0.0;
      for (int j = 0; j < 4; ++j) s += double(trans[size_t(i * 4 + j) * nq + q]);
      tot[q] = s;
    }
    for (int j = 0; j < 4; ++j) {
      if (i == j) continue;
      for (int q = 0; q < nq; ++q) {
        const double e = double(trans[size_t(i * 4 + j) * nq + q]);
        rlogp[q] = tot[q] == 0.0 ? std::numeric_limits<double>::quiet_NaN() : std::log10((e + 1.0) / tot[q]);
      }
      std::vector<double> pred = loess_predict(xs, rlogp, tot, 0.75, 2, ef.surface, ef.cell);
      extrapolate_flat(pred);
      bool any = false;
      for (double v : pred) any |= std::isfinite(v);
      failed += any ? 0 : 1;
      for (int q = 0; q < nq; ++q) {
        const double rate = std::isfinite(pred[q]) ? std::pow(10.0, pred[q]) : ef.min_error_rate;
        off[size_t(orow) * nq + q] = clamp_rate(rate, ef);
      }
      ++orow;
    }
  }
  if (failed == 12) {
    *msg = "LOESS fit failed for all 12 transitions (no transition has any observation)";
    return DGPU_E_INVALID;
  }
  expand(off, nq, err);
  return 0;
}

// An anchor quality as an index: what Rust's `f64 as usize` gives (NaN and
// negatives 0, truncation, saturation).
size_t anchor_col(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 18446744073709551615.0) return std::numeric_limits<size_t>::max();
  return size_t(v);
}

// An f64 as Rust's `{}` prints it, for the messages the reference returns.
std::string f64_text(double v) {
  if (std::isnan(v)) return "NaN";
  if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
  char b[64];
  if (std::fabs(v) < 1e15 && v == std::floor(v)) std::snprintf(b, sizeof b, "%.0f", v);
  else std::snprintf(b, sizeof b, "%.17g", v);
  return b;
}

// Piecewise-linear rates between anchor qualities (quality scores 0..nq-1).
int binned_fit(const dgpu_errfun& ef, const uint32_t* trans, int nq, double* err, std::string* msg) {
  const double inf = std::numeric_limits<double>::infinity();
  double lo_obs = inf, hi_obs = -inf;
  for (int q = 0; q < nq; ++q) {
    uint64_t c = 0;
    for (int r = 0; r < 16; ++r) c += trans[size_t(r) * nq + q];
    if (c) {
      lo_obs = std::min(lo_obs, double(q));
      hi_obs = std::max(hi_obs, double(q));
    }
  }
  if (hi_obs < lo_obs) {
    *msg = "No observed transitions";
    return DGPU_E_INVALID;
  }
  const int nb = ef.bins ? ef.nbins : 0;
  double bmin = inf, bmax = -inf;
  for (int k = 0; k < nb; ++k) {
    bmin = std::min(bmin, ef.bins[k]);
    bmax = std::max(bmax, ef.bins[k]);
  }
  if (hi_obs > bmax) {
    *msg = "Input data contains quality score " + f64_text(hi_obs) + " higher than max binned value " + f64_text(bmax);
    return DGPU_E_INVALID;
  }
  if (lo_obs < bmin) {
    *msg = "Input data contains quality score " + f64_text(lo_obs) + " lower than min binned value " + f64_text(bmin);
    return DGPU_E_INVALID;
  }
  const double nan = std::numeric_limits<double>::quiet_NaN();
  std::vector<double> off(size_t(12) * nq, 0.0), rate(nq), line(nq);
  int orow = 0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      if (i == j) continue;
      for (int q = 0; q < nq; ++q) {
        double t = 0.0;
        for (int k = 0; k < 4; ++k) t += double(trans[size_t(i * 4 + k) * nq + q]);
        rate[q] = t > 0.0 ? double(trans[size_t(i * 4 + j) * nq + q]) / t : nan;
      }
      std::fill(line.begin(), line.end(), nan);
      for (int k = 0; k + 1 < nb; ++k) {
        const size_t a = anchor_col(ef.bins[k]), b = anchor_col(ef.bins[k + 1]);
        if (a >= size_t(nq) || b >= size_t(nq)) continue;
        if (b < a) {
          *msg = "binned quality scores must be ascending";
          return DGPU_E_INVALID;
        }
        if (!std::isfinite(rate[a]) || !std::isfinite(rate[b])) continue;
        const size_t n = b - a + 1;
        for (size_t s = 0; s < n; ++s) {
          const double f = n > 1 ? double(s) / double(n - 1) : 0.0;
          line[a + s] = rate[a] * (1.0 - f) + rate[b] * f;
        }
      }
      extrapolate_flat(line);
      for (int q = 0; q < nq; ++q)
        off[size_t(orow) * nq + q] = std::isfinite(line[q]) ? clamp_rate(line[q], ef) : ef.min_error_rate;
      ++orow;
    }
  expand(off, nq, err);
  return 0;
}

// PacBio: LOESS below Q93 and a pseudocount estimate in the Q93 column.
int pacbio_fit(const dgpu_errfun& ef, const uint32_t* trans, int nq, double* err, std::string* msg) {
  if (nq != 94) return loess_fit(ef, trans, nq, err, msg);
  const int lo = 93;
  std::vector<uint32_t> below(size_t(16) * lo);
  for (int r = 0; r < 16; ++r)
    std::copy(trans + size_t(r) * nq, trans + size_t(r) * nq + lo, below.begin() + size_t(r) * lo);
  std::vector<double> fit(size_t(16) * lo);
  const int rc = loess_fit(ef, below.data(), lo, fit.data(), msg);
  if (rc) return rc;
  for (int r = 0; r < 16; ++r) std::copy(fit.begin() + size_t(r) * lo, fit.begin() + size_t(r + 1) * lo, err + size_t(r) * nq);
  for (int i = 0; i < 4; ++i) {
    double t = 0.0;
    for (int j = 0; j < 4; ++j) t += double(trans[size_t(i * 4 + j) * nq + lo]);
    for (int j = 0; j < 4; ++j)
      err[size_t(i * 4 + j) * nq + lo] = (double(trans[size_t(i * 4 + j) * nq + lo]) + 1.0) / (t + 4.0);
  }
  return 0;
}

}  // namespace

// The fit the learn-errors loop applies to its accumulated transition matrix
// (quality scores 0..nq-1, src/learn_errors.rs:84-100). Returns 0, or
// DGPU_E_INVALID with *msg where the reference's fit returns an error.
int errfun_apply(const dgpu_errfun& ef, const uint32_t* trans, int nq, double* err, std::string* msg) {
  if (ef.kind == DGPU_ERRFUN_NOQUAL) {
    std::vector<double> off(size_t(12) * nq, 0.0);
    double obs[16];
    for (int r = 0; r < 16; ++r) {
      double s = 0.0;
      for (int q = 0; q < nq; ++q) s += double(trans[size_t(r) * nq + q]);
      obs[r] = s + ef.pseudocount;
    }
    int orow = 0;
    for (int i = 0; i < 4; ++i) {
      double tot = 0.0;
      for (int j = 0; j < 4; ++j) tot += obs[i * 4 + j];
      for (int j = 0; j < 4; ++j) {
        if (i == j) continue;
        const double rate = tot > 0.0 ? clamp_rate(obs[i * 4 + j] / tot, ef) : ef.min_error_rate;
        for (int q = 0; q < nq; ++q) off[size_t(orow) * nq + q] = rate;
        ++orow;
      }
    }
    expand(off, nq, err);
    return 0;
  }
  if (ef.kind == DGPU_ERRFUN_LOESS) return loess_fit(ef, trans, nq, err, msg);
  if (ef.kind == DGPU_ERRFUN_BINNED) return binned_fit(ef, trans, nq, err, msg);
  if (ef.kind == DGPU_ERRFUN_PACBIO) return pacbio_fit(ef, trans, nq, err, msg);
  if (ef.kind == DGPU_ERRFUN_EXTERNAL) return external_errfun_fit(ef.cmd, trans, nq, err, msg);
  *msg = "unknown error function kind";
  return DGPU_E_INVALID;
}

}  // namespace dgpu

extern "C" int dgpu_errfun_apply(const dgpu_errfun* ef, const uint32_t* trans, int nq, double* err_out) {
  if (!ef || !trans || !err_out || nq <= 0) {
    dgpu::set_last_error("bad argument");
    return DGPU_E_INVALID;
  }
  std::string msg;
  const int rc = dgpu::errfun_apply(*ef, trans, nq, err_out, &msg);
  if (rc) dgpu::set_last_error(msg.c_str());
  return rc;
}

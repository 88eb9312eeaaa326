// host_analysis.cpp -- host FP64 analysis downstream of the glueball
// measurements: the periodic cosh effective mass with delete-one jackknife
// errors (glueball_effective_mass.rs:91-263), the correlated single-state
// fit with plateau-window selection (glueball_scalar_fit.rs:156-690) and the
// two-operator variational projection, a 2x2 generalized eigenproblem
// (glueball_scalar_variational.rs:132-975).
//
// These run on the host over correlators the device pipeline produced
// (N_cfg <= 64 configurations, N_t <= 64 slices: microseconds to
// milliseconds of sequential FP64).  Compiled with -ffp-contract=off so every
// a*b+c is two roundings, as in the reference; the reference's explicit
// fused multiply-adds (f64::mul_add) are std::fma here.  Every failure is
// the reference's fail-closed variant, checked in the reference's order.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

#include "../../include/ym_analysis.h"

namespace {

// ------------------------------------------------------------ shared pieces

bool fin(double v) { return std::isfinite(v); }   // (libm's finite() would clash)

// Rust's f64::acosh: ln(x + sqrt(x - 1) * sqrt(x + 1)) for x >= 1.
double rust_acosh(double x) {
    if (x < 1.0) return NAN;
    return std::log(x + std::sqrt(x - 1.0) * std::sqrt(x + 1.0));
}

// A jackknife replica set as the reference's &[Vec<f64>]: one pointer and
// one length per replica.
struct Replicas {
    const double *const *row;
    const int64_t *len;
    int64_t n;
};

// ------------------------------------------------ effective mass (phase 3D)

constexpr int64_t kMinReplicates = 3, kMaxReplicates = 64;   // glueball_effective_mass.rs:18-19
constexpr int64_t kMinTimeExtent = 4, kMaxTimeExtent = 64;    // glueball_effective_mass.rs:20-21

// validate_inputs (glueball_effective_mass.rs:91-134)
int32_t validate_effective_mass(const double *full, int64_t nt, const Replicas &jk,
                                const uint64_t *lags, int64_t n_lags) {
    if (nt < kMinTimeExtent) return YM_ERR_TIME_EXTENT_TOO_SMALL;
    if (nt > kMaxTimeExtent) return YM_ERR_TIME_EXTENT_TOO_LARGE;
    if (jk.n < kMinReplicates) return YM_ERR_TOO_FEW_JACKKNIFE_REPLICATES;
    if (jk.n > kMaxReplicates) return YM_ERR_TOO_MANY_JACKKNIFE_REPLICATES;
    if (n_lags <= 0) return YM_ERR_EMPTY_ANALYSIS_WINDOW;
    for (int64_t t = 0; t < nt; ++t)
        if (!fin(full[t])) return YM_ERR_NON_FINITE_CORRELATOR;
    for (int64_t r = 0; r < jk.n; ++r)
        if (jk.len[r] != nt) return YM_ERR_SHAPE_MISMATCH;
    for (int64_t r = 0; r < jk.n; ++r)
        for (int64_t t = 0; t < nt; ++t)
            if (!fin(jk.row[r][t])) return YM_ERR_NON_FINITE_CORRELATOR;
    const uint64_t ext = (uint64_t)nt;
    uint64_t previous = 0;
    for (int64_t i = 0; i < n_lags; ++i) {
        const uint64_t tau = lags[i];
        const bool doubled_reaches_midpoint = tau > UINT64_MAX / 2 || 2 * tau >= ext;
        if (tau == 0 || tau >= ext - 1 || doubled_reaches_midpoint || (i != 0 && tau <= previous))
            return YM_ERR_INVALID_ANALYSIS_LAG;
        previous = tau;
    }
    return YM_OK;
}

// cosh_effective_mass (glueball_effective_mass.rs:136-157)
int32_t cosh_mass(const double *c, uint64_t tau, double *out) {
    const double center = c[tau];
    if (center <= 0.0) return YM_ERR_NON_POSITIVE_CENTRAL_CORRELATOR;
    const double numerator = c[tau - 1] + c[tau + 1];
    const double denominator = 2.0 * center;
    const double argument = numerator / denominator;
    if (!fin(numerator) || !fin(denominator) || !fin(argument))
        return YM_ERR_NON_FINITE_STATISTIC;
    if (argument < 1.0) return YM_ERR_ACOSH_DOMAIN_VIOLATION;
    const double m = rust_acosh(argument);
    if (!fin(m)) return YM_ERR_NON_FINITE_STATISTIC;
    *out = m;
    return YM_OK;
}

// cosh_effective_mass_with_jackknife (glueball_effective_mass.rs:170-234)
int32_t effective_mass_series(const double *full, int64_t nt, const Replicas &jk,
                              const uint64_t *lags, int64_t n_lags, ym_effective_mass_point *points) {
    if (int32_t st = validate_effective_mass(full, nt, jk, lags, n_lags)) return st;
    std::vector<double> masses((size_t)jk.n);
    for (int64_t i = 0; i < n_lags; ++i) {
        const uint64_t tau = lags[i];
        double estimate;
        if (int32_t st = cosh_mass(full, tau, &estimate)) return st;
        double sum = 0.0;
        for (int64_t r = 0; r < jk.n; ++r) {
            if (int32_t st = cosh_mass(jk.row[r], tau, &masses[(size_t)r])) return st;
            sum += masses[(size_t)r];
            if (!fin(sum)) return YM_ERR_NON_FINITE_STATISTIC;
        }
        const double n = (double)jk.n;
        const double mean = sum / n;
        if (!fin(mean)) return YM_ERR_NON_FINITE_STATISTIC;
        double ssd = 0.0;
        for (double m : masses) {
            const double d = m - mean;
            ssd += d * d;
            if (!fin(ssd)) return YM_ERR_NON_FINITE_STATISTIC;
        }
        const double variance = ((n - 1.0) / n) * ssd;
        const double se = std::sqrt(variance);
        if (!fin(variance) || variance < 0.0 || !fin(se)) return YM_ERR_NON_FINITE_STATISTIC;
        points[i] = ym_effective_mass_point{(int64_t)tau, estimate, mean, se};
    }
    return YM_OK;
}

// analytic_periodic_single_state (glueball_effective_mass.rs:237-263)
int32_t single_state(int64_t nt, double mass, double amplitude, double *out) {
    if (nt < kMinTimeExtent || nt > kMaxTimeExtent || !fin(mass) || mass <= 0.0 ||
        !fin(amplitude) || amplitude <= 0.0)
        return YM_ERR_INVALID_FIXTURE_PARAMETER;
    for (int64_t tau = 0; tau < nt; ++tau) {
        const double left = std::exp(-mass * (double)tau);
        const double right = std::exp(-mass * (double)(nt - tau));
        const double v = amplitude * (left + right);
        if (!fin(v)) return YM_ERR_NON_FINITE_STATISTIC;
        out[tau] = v;
    }
    return YM_OK;
}

// ------------------------------------------------- correlated fit (phase 3E)

constexpr int64_t kMinWindowPoints = 3, kMaxWindowPoints = 8;   // glueball_scalar_fit.rs:15-16
constexpr int64_t kMaxCandidateWindows = 16;                    // glueball_scalar_fit.rs:17
constexpr double kPlateauMaxZ = 2.5;                             // glueball_scalar_fit.rs:18
constexpr double kMassGridMin = 0.05, kMassGridMax = 2.0;        // glueball_scalar_fit.rs:19-20
constexpr double kMassGridStep = 0.001;                          // glueball_scalar_fit.rs:21
constexpr int64_t kMassGridSteps = 1950;                         // glueball_scalar_fit.rs:22
constexpr double kPivotRelTolerance = 1.0e-12;                   // glueball_scalar_fit.rs:23

// FitWindow::point_count: end - start + 1, absent when end < start or the
// count overflows.
bool point_count(const ym_fit_window &w, uint64_t *count) {
    if (w.end < w.start || w.end - w.start == UINT64_MAX) return false;
    *count = w.end - w.start + 1;
    return true;
}

// validate_candidate_windows (glueball_scalar_fit.rs:156-182)
int32_t validate_windows(int64_t nt, const ym_fit_window *c, int64_t n) {
    if (n <= 0) return YM_ERR_EMPTY_CANDIDATE_WINDOWS;
    if (n > kMaxCandidateWindows) return YM_ERR_TOO_MANY_CANDIDATE_WINDOWS;
    for (int64_t i = 0; i < n; ++i) {
        uint64_t count;
        if (!point_count(c[i], &count)) return YM_ERR_INVALID_CANDIDATE_WINDOW;
        const bool end_reaches_midpoint = c[i].end > UINT64_MAX / 2 || 2 * c[i].end >= (uint64_t)nt;
        if (c[i].start == 0 || count < (uint64_t)kMinWindowPoints || count > (uint64_t)kMaxWindowPoints ||
            end_reaches_midpoint)
            return YM_ERR_INVALID_CANDIDATE_WINDOW;
        for (int64_t j = 0; j < i; ++j)
            if (c[j].start == c[i].start && c[j].end == c[i].end)
                return YM_ERR_DUPLICATE_CANDIDATE_WINDOW;
    }
    return YM_OK;
}

struct Plateau {
    ym_fit_window window;
    double weighted_mass, max_z;
};

// evaluate_plateau_window (glueball_scalar_fit.rs:197-237)
int32_t evaluate_plateau(const double *full, int64_t nt, const Replicas &jk, const ym_fit_window &w,
                         Plateau *out) {
    uint64_t count;
    if (!point_count(w, &count)) return YM_ERR_INVALID_CANDIDATE_WINDOW;
    std::vector<uint64_t> lags((size_t)count);
    for (uint64_t i = 0; i < count; ++i) lags[(size_t)i] = w.start + i;
    std::vector<ym_effective_mass_point> pts((size_t)count);
    if (int32_t st = effective_mass_series(full, nt, jk, lags.data(), (int64_t)count, pts.data()))
        return st;
    double wsum = 0.0, weights = 0.0;
    for (const auto &p : pts) {
        if (!fin(p.standard_error) || p.standard_error <= 0.0)
            return YM_ERR_DEGENERATE_PLATEAU_UNCERTAINTY;
        const double weight = 1.0 / (p.standard_error * p.standard_error);
        wsum += weight * p.full_estimate;
        weights += weight;
        if (!fin(wsum) || !fin(weights)) return YM_ERR_NON_FINITE_STATISTIC;
    }
    if (weights <= 0.0) return YM_ERR_NON_FINITE_STATISTIC;
    const double wm = wsum / weights;
    if (!fin(wm)) return YM_ERR_NON_FINITE_STATISTIC;
    double max_z = 0.0;
    for (const auto &p : pts) {
        const double z = std::fabs((p.full_estimate - wm) / p.standard_error);
        if (!fin(z)) return YM_ERR_NON_FINITE_STATISTIC;
        max_z = std::fmax(max_z, z);
    }
    *out = Plateau{w, wm, max_z};
    return YM_OK;
}

// choose_plateau_window (glueball_scalar_fit.rs:239-274): the longest
// passing window, ties to the later start.
int32_t choose_plateau(const double *full, int64_t nt, const Replicas &jk, const ym_fit_window *c,
                       int64_t n, Plateau *best) {
    if (int32_t st = validate_windows(nt, c, n)) return st;
    bool have = false;
    uint64_t best_count = 0;
    for (int64_t i = 0; i < n; ++i) {
        Plateau sel{};
        const int32_t st = evaluate_plateau(full, nt, jk, c[i], &sel);
        if (st == YM_ERR_DEGENERATE_PLATEAU_UNCERTAINTY) continue;
        if (st) return st;
        if (sel.max_z > kPlateauMaxZ) continue;
        uint64_t count = 0;
        point_count(c[i], &count);
        if (!have || count > best_count || (count == best_count && c[i].start > best->window.start)) {
            *best = sel;
            best_count = count;
            have = true;
        }
    }
    return have ? YM_OK : YM_ERR_NO_ACCEPTED_PLATEAU_WINDOW;
}

// A dense row-major n x n matrix.
struct Dense {
    int64_t n;
    std::vector<double> v;
    explicit Dense(int64_t size) : n(size), v((size_t)(size * size), 0.0) {}
    double &at(int64_t r, int64_t c) { return v[(size_t)(r * n + c)]; }
    double at(int64_t r, int64_t c) const { return v[(size_t)(r * n + c)]; }
};

// jackknife_covariance (glueball_scalar_fit.rs:276-322)
int32_t window_covariance(const Replicas &jk, const ym_fit_window &w, Dense *out) {
    uint64_t upoints;
    if (!point_count(w, &upoints)) return YM_ERR_INVALID_CANDIDATE_WINDOW;
    if ((uint64_t)jk.n <= upoints) return YM_ERR_INSUFFICIENT_REPLICATES_FOR_COVARIANCE;
    const int64_t points = (int64_t)upoints;
    std::vector<double> means((size_t)points, 0.0);
    for (int64_t r = 0; r < jk.n; ++r)
        for (int64_t c = 0; c < points; ++c) {
            const uint64_t tau = w.start + (uint64_t)c;
            if (tau >= (uint64_t)jk.len[r]) return YM_ERR_INVALID_CANDIDATE_WINDOW;
            const double v = jk.row[r][tau];
            if (!fin(v)) return YM_ERR_NON_FINITE_STATISTIC;
            means[(size_t)c] += v;
        }
    const double n = (double)jk.n;
    for (double &m : means) m /= n;
    Dense cov(points);
    for (int64_t r = 0; r < jk.n; ++r)
        for (int64_t a = 0; a < points; ++a) {
            const double left = jk.row[r][w.start + a] - means[(size_t)a];
            for (int64_t b = 0; b < points; ++b)
                cov.at(a, b) += left * (jk.row[r][w.start + b] - means[(size_t)b]);
        }
    const double factor = (n - 1.0) / n;
    for (double &x : cov.v) {
        x *= factor;
        if (!fin(x)) return YM_ERR_NON_FINITE_STATISTIC;
    }
    *out = std::move(cov);
    return YM_OK;
}

double max_abs_entry(const Dense &m) {
    double s = 0.0;
    for (double x : m.v) s = std::fmax(s, std::fabs(x));   // f64::max ignores NaN, as fmax does
    return s;
}

// validate_positive_definite (glueball_scalar_fit.rs:324-359): Cholesky
// with every pivot above 1e-12 of the largest entry.
int32_t check_positive_definite(const Dense &m) {
    const int64_t n = m.n;
    if (n == 0) return YM_ERR_COVARIANCE_NOT_POSITIVE_DEFINITE;
    const double scale = max_abs_entry(m);
    if (!fin(scale) || scale <= 0.0) return YM_ERR_COVARIANCE_NOT_POSITIVE_DEFINITE;
    Dense l(n);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t j = 0; j <= i; ++j) {
            double s = m.at(i, j);
            for (int64_t k = 0; k < j; ++k) s -= l.at(i, k) * l.at(j, k);
            if (i == j) {
                if (!fin(s) || s <= scale * kPivotRelTolerance)
                    return YM_ERR_COVARIANCE_NOT_POSITIVE_DEFINITE;
                l.at(i, j) = std::sqrt(s);
            } else {
                const double pivot = l.at(j, j);
                if (!fin(pivot) || pivot <= 0.0) return YM_ERR_COVARIANCE_NOT_POSITIVE_DEFINITE;
                l.at(i, j) = s / pivot;
            }
        }
    return YM_OK;
}

// invert_matrix (glueball_scalar_fit.rs:361-421): Gauss-Jordan on [M | 1]
// with partial pivoting (first strictly larger magnitude wins).
int32_t invert(const Dense &m, Dense *inverse) {
    if (int32_t st = check_positive_definite(m)) return st;
    const int64_t n = m.n, w = 2 * n;
    const double scale = max_abs_entry(m);
    std::vector<std::vector<double>> aug((size_t)n, std::vector<double>((size_t)w, 0.0));
    for (int64_t r = 0; r < n; ++r) {
        for (int64_t c = 0; c < n; ++c) aug[(size_t)r][(size_t)c] = m.at(r, c);
        aug[(size_t)r][(size_t)(n + r)] = 1.0;
    }
    for (int64_t col = 0; col < n; ++col) {
        int64_t pr = col;
        double pabs = std::fabs(aug[(size_t)col][(size_t)col]);
        for (int64_t r = col + 1; r < n; ++r) {
            const double cand = std::fabs(aug[(size_t)r][(size_t)col]);
            if (cand > pabs) {
                pabs = cand;
                pr = r;
            }
        }
        if (!fin(pabs) || pabs <= scale * kPivotRelTolerance) return YM_ERR_SINGULAR_COVARIANCE;
        if (pr != col) std::swap(aug[(size_t)pr], aug[(size_t)col]);
        std::vector<double> &prow = aug[(size_t)col];
        const double pivot = prow[(size_t)col];
        for (double &x : prow) x /= pivot;
        for (int64_t r = 0; r < n; ++r) {
            if (r == col) continue;
            std::vector<double> &row = aug[(size_t)r];
            const double f = row[(size_t)col];
            for (int64_t i = 0; i < w; ++i) row[(size_t)i] -= f * prow[(size_t)i];
        }
    }
    Dense out(n);
    for (int64_t r = 0; r < n; ++r)
        for (int64_t c = 0; c < n; ++c) {
            const double v = aug[(size_t)r][(size_t)(n + c)];
            if (!fin(v)) return YM_ERR_SINGULAR_COVARIANCE;
            out.at(r, c) = v;
        }
    *inverse = std::move(out);
    return YM_OK;
}

// quadratic_form (glueball_scalar_fit.rs:423-439): sum_r l_r (sum_c M_rc r_c)
int32_t quad(const double *l, const Dense &m, const double *r, double *out) {
    double s = 0.0;
    for (int64_t i = 0; i < m.n; ++i) {
        double inner = 0.0;
        for (int64_t c = 0; c < m.n; ++c) inner += m.at(i, c) * r[c];
        s += l[i] * inner;
    }
    if (!fin(s)) return YM_ERR_NON_FINITE_STATISTIC;
    *out = s;
    return YM_OK;
}

struct ProfileFit {
    double mass, amplitude, chi2;
};

// profile_grid_fit (glueball_scalar_fit.rs:470-526): for each grid mass the
// amplitude is the correlated least-squares optimum; keep the smallest
// chi^2, ties to the smaller mass.
int32_t profile_fit(int64_t nt, const ym_fit_window &w, const double *values, const Dense &inv,
                    ProfileFit *out) {
    const int64_t p = inv.n;
    for (int64_t i = 0; i < p; ++i)
        if (!fin(values[i])) return YM_ERR_NON_FINITE_STATISTIC;
    std::vector<double> basis((size_t)p), residual((size_t)p);
    bool have = false;
    ProfileFit best{0, 0, 0};
    for (int64_t g = 0; g <= kMassGridSteps; ++g) {
        const double mass = kMassGridMin + kMassGridStep * (double)g;
        if (mass > kMassGridMax + 1.0e-15) break;
        // periodic_basis (glueball_scalar_fit.rs:441-466)
        for (int64_t i = 0; i < p; ++i) {
            const uint64_t tau = w.start + (uint64_t)i;
            const double b = std::exp(-mass * (double)tau) + std::exp(-mass * (double)((uint64_t)nt - tau));
            if (!fin(b) || b <= 0.0) return YM_ERR_NON_FINITE_STATISTIC;
            basis[(size_t)i] = b;
        }
        double den, num, chi2;
        if (int32_t st = quad(basis.data(), inv, basis.data(), &den)) return st;
        if (den <= 0.0 || !fin(den)) continue;
        if (int32_t st = quad(basis.data(), inv, values, &num)) return st;
        const double amp = num / den;
        if (amp <= 0.0 || !fin(amp)) continue;
        for (int64_t i = 0; i < p; ++i) residual[(size_t)i] = values[i] - amp * basis[(size_t)i];
        if (int32_t st = quad(residual.data(), inv, residual.data(), &chi2)) return st;
        if (chi2 < 0.0 || !fin(chi2)) continue;
        if (!have || chi2 < best.chi2 || (chi2 == best.chi2 && mass < best.mass)) {
            best = ProfileFit{mass, amp, chi2};
            have = true;
        }
    }
    if (!have) return YM_ERR_NO_FINITE_GRID_FIT;
    *out = best;
    return YM_OK;
}

// window_values (glueball_scalar_fit.rs:528-546)
int32_t window_values(const double *v, int64_t len, const ym_fit_window &w, std::vector<double> *out) {
    uint64_t upoints;
    if (!point_count(w, &upoints)) return YM_ERR_INVALID_CANDIDATE_WINDOW;
    if (upoints > (uint64_t)len) return YM_ERR_INVALID_CANDIDATE_WINDOW;
    const int64_t points = (int64_t)upoints;
    out->assign((size_t)points, 0.0);
    for (int64_t i = 0; i < points; ++i) {
        const uint64_t tau = w.start + (uint64_t)i;
        if (tau >= (uint64_t)len) return YM_ERR_INVALID_CANDIDATE_WINDOW;
        if (!fin(v[tau])) return YM_ERR_NON_FINITE_STATISTIC;
        (*out)[(size_t)i] = v[tau];
    }
    return YM_OK;
}

// jackknife_standard_error (glueball_scalar_fit.rs:548-565)
int32_t jackknife_error(const std::vector<double> &v, double *mean_out, double *se_out) {
    if (v.empty()) return YM_ERR_NON_FINITE_STATISTIC;
    for (double x : v)
        if (!fin(x)) return YM_ERR_NON_FINITE_STATISTIC;
    const double n = (double)v.size();
    double s = 0.0;
    for (double x : v) s += x;
    const double mean = s / n;
    double ssd = 0.0;
    for (double x : v) {
        const double d = x - mean;
        ssd += d * d;
    }
    const double variance = ((n - 1.0) / n) * ssd;
    const double se = std::sqrt(variance);
    if (!fin(mean) || !fin(variance) || variance < 0.0 || !fin(se))
        return YM_ERR_NON_FINITE_STATISTIC;
    *mean_out = mean;
    *se_out = se;
    return YM_OK;
}

// maximum_off_diagonal_correlation (glueball_scalar_fit.rs:567-593)
int32_t max_off_diagonal(const Dense &cov, double *out) {
    double mx = 0.0;
    for (int64_t r = 0; r < cov.n; ++r) {
        const double drr = cov.at(r, r);
        if (drr <= 0.0 || !fin(drr)) return YM_ERR_COVARIANCE_NOT_POSITIVE_DEFINITE;
        const double rs = std::sqrt(drr);
        if (!fin(rs) || rs <= 0.0) return YM_ERR_COVARIANCE_NOT_POSITIVE_DEFINITE;
        for (int64_t c = 0; c < r; ++c) {
            const double dcc = cov.at(c, c);
            if (dcc <= 0.0 || !fin(dcc)) return YM_ERR_COVARIANCE_NOT_POSITIVE_DEFINITE;
            const double cs = std::sqrt(dcc);
            if (!fin(cs) || cs <= 0.0) return YM_ERR_COVARIANCE_NOT_POSITIVE_DEFINITE;
            const double corr = std::fabs((cov.at(r, c) / rs) / cs);
            if (!fin(corr)) return YM_ERR_NON_FINITE_STATISTIC;
            mx = std::fmax(mx, corr);
        }
    }
    *out = mx;
    return YM_OK;
}

// correlated_scalar_fit (glueball_scalar_fit.rs:595-650)
int32_t scalar_fit(const double *full, int64_t nt, const Replicas &jk, const ym_fit_window *cand,
                   int64_t n_cand, ym_scalar_fit_result *res) {
    Plateau sel{};
    if (int32_t st = choose_plateau(full, nt, jk, cand, n_cand, &sel)) return st;
    const ym_fit_window w = sel.window;
    Dense cov(0), inv(0);
    if (int32_t st = window_covariance(jk, w, &cov)) return st;
    if (int32_t st = invert(cov, &inv)) return st;
    double max_corr;
    if (int32_t st = max_off_diagonal(cov, &max_corr)) return st;
    std::vector<double> values;
    if (int32_t st = window_values(full, nt, w, &values)) return st;
    ProfileFit ff;
    if (int32_t st = profile_fit(nt, w, values.data(), inv, &ff)) return st;
    std::vector<double> masses, amplitudes;
    masses.reserve((size_t)jk.n);
    amplitudes.reserve((size_t)jk.n);
    for (int64_t r = 0; r < jk.n; ++r) {
        if (int32_t st = window_values(jk.row[r], jk.len[r], w, &values)) return st;
        ProfileFit f;
        if (int32_t st = profile_fit(nt, w, values.data(), inv, &f)) return st;
        masses.push_back(f.mass);
        amplitudes.push_back(f.amplitude);
    }
    double mass_mean, mass_se, amp_mean, amp_se;
    if (int32_t st = jackknife_error(masses, &mass_mean, &mass_se)) return st;
    if (int32_t st = jackknife_error(amplitudes, &amp_mean, &amp_se)) return st;
    uint64_t points = 0;
    point_count(w, &points);
    const int64_t dof = (int64_t)points - 2;
    const double chi2_dof = ff.chi2 / (double)dof;
    if (!fin(chi2_dof)) return YM_ERR_NON_FINITE_STATISTIC;
    res->time_extent = nt;
    res->jackknife_replicates = jk.n;
    res->selected_window = w;
    res->plateau_weighted_effective_mass = sel.weighted_mass;
    res->plateau_maximum_z = sel.max_z;
    res->fitted_mass = ff.mass;
    res->fitted_amplitude = ff.amplitude;
    res->chi_square = ff.chi2;
    res->degrees_of_freedom = dof;
    res->chi_square_per_dof = chi2_dof;
    res->mass_jackknife_mean = mass_mean;
    res->mass_standard_error = mass_se;
    res->amplitude_jackknife_mean = amp_mean;
    res->amplitude_standard_error = amp_se;
    res->maximum_off_diagonal_correlation = max_corr;
    return YM_OK;
}

// ------------------------------------------------- variational (phase 3J)

constexpr int64_t kMaxConfigurations = 64;          // glueball_correlators.rs:19
constexpr int64_t kVarMaxTimeExtent = 64;           // glueball_correlators.rs:20
constexpr double kSymmetryTolerance = 2.0e-12;      // glueball_scalar_variational.rs:26
constexpr double kNormalizationTolerance = 2.0e-12; // glueball_scalar_variational.rs:28
constexpr double kPdPivotTolerance = 1.0e-14;       // glueball_scalar_variational.rs:29

struct M2 {
    double a[2][2];
};

M2 load_m2(const double *p) { return M2{{{p[0], p[1]}, {p[2], p[3]}}}; }

bool m2_finite(const M2 &m) {
    return fin(m.a[0][0]) && fin(m.a[0][1]) && fin(m.a[1][0]) && fin(m.a[1][1]);
}

bool m2_equal(const M2 &x, const M2 &y) {
    return x.a[0][0] == y.a[0][0] && x.a[0][1] == y.a[0][1] && x.a[1][0] == y.a[1][0] &&
           x.a[1][1] == y.a[1][1];
}

// symmetry_within_tolerance (glueball_scalar_variational.rs:136-147)
bool symmetric_enough(const M2 &m) {
    const double residual = std::fabs(m.a[0][1] - m.a[1][0]);
    if (!fin(residual)) return false;
    const double scale = std::fmax(std::fmax(std::fabs(m.a[0][1]), std::fabs(m.a[1][0])), 1.0);
    return fin(scale) && residual <= kSymmetryTolerance * scale;
}

// stable_average (glueball_scalar_variational.rs:149-165): first + (second -
// first)/2, exact when both are the same bits.
int32_t stable_average(double x, double y, double *out) {
    if (!fin(x) || !fin(y)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    uint64_t bx, by;
    std::memcpy(&bx, &x, 8);
    std::memcpy(&by, &y, 8);
    if (bx == by) {
        *out = x;
        return YM_OK;
    }
    const double d = y - x;
    if (!fin(d)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    const double avg = x + 0.5 * d;
    if (!fin(avg)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    *out = avg;
    return YM_OK;
}

int32_t symmetrized(const M2 &m, M2 *out) {
    double cross;
    if (int32_t st = stable_average(m.a[0][1], m.a[1][0], &cross)) return st;
    *out = M2{{{m.a[0][0], cross}, {cross, m.a[1][1]}}};
    return YM_OK;
}

// validate_matrix_series (glueball_scalar_variational.rs:172-185)
int32_t validate_series(const double *mats, int64_t nt) {
    if (nt < 3 || nt > kVarMaxTimeExtent) return YM_ERR_CORRELATOR_SHAPE_MISMATCH;
    for (int64_t t = 0; t < nt; ++t) {
        const M2 m = load_m2(mats + 4 * t);
        if (!m2_finite(m)) return YM_ERR_NON_FINITE_ACCUMULATOR;
        if (!symmetric_enough(m)) return YM_ERR_MATRIX_NOT_SYMMETRIC;
    }
    return YM_OK;
}

// stable_divide_by_product (glueball_scalar_variational.rs:207-248):
// numerator / (p q) without forming p q, larger factor first.
int32_t divide_by_product(double num, double p, double q, double *out) {
    if (!fin(num) || !fin(p) || !fin(q) || p == 0.0 || q == 0.0)
        return YM_ERR_NON_FINITE_ACCUMULATOR;
    const double large = std::fabs(p) >= std::fabs(q) ? p : q;
    const double small = std::fabs(p) >= std::fabs(q) ? q : p;
    const double i1 = num / large, v1 = i1 / small;
    if (fin(i1) && fin(v1) && (i1 != 0.0 || num == 0.0)) {
        *out = v1;
        return YM_OK;
    }
    const double i2 = num / small, v2 = i2 / large;
    if (fin(i2) && fin(v2)) {
        *out = v2;
        return YM_OK;
    }
    return YM_ERR_NON_FINITE_ACCUMULATOR;
}

// compensated_symmetric_determinant (glueball_scalar_variational.rs:250-282):
// a d - c^2 with the rounding error of each product recovered by fma.
int32_t compensated_det(double a, double d, double c, double *out) {
    if (!fin(a) || !fin(d) || !fin(c)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    const double ad = a * d, cc = c * c;
    if (!fin(ad) || !fin(cc)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    const double ad_err = std::fma(a, d, -ad), cc_err = std::fma(c, c, -cc);
    const double leading = ad - cc, correction = ad_err - cc_err;
    const double det = leading + correction;
    if (!fin(ad_err) || !fin(cc_err) || !fin(leading) || !fin(correction) || !fin(det))
        return YM_ERR_NON_FINITE_ACCUMULATOR;
    *out = det;
    return YM_OK;
}

// solve_scaled_generalized_characteristic (glueball_scalar_variational.rs:284-378):
// the larger root of det(C1 - lambda C0) = 0 with C0 normalised to unit
// diagonal (off-diagonal r, determinant 1 - r^2), solved in the +/- basis
// that diagonalises C0.
int32_t characteristic_root(double ref_det, double ref_off, double d1, double d2, double off,
                            double *out) {
    if (!fin(ref_det) || ref_det <= 0.0 || !fin(ref_off) || !fin(d1) || !fin(d2) ||
        !fin(off))
        return YM_ERR_NON_FINITE_ACCUMULATOR;
    const double plus_den = 1.0 + ref_off, minus_den = 1.0 - ref_off;
    const double sqrt_det = std::sqrt(ref_det);
    if (!fin(plus_den) || !fin(minus_den) || !fin(sqrt_det) || plus_den <= 0.0 ||
        minus_den <= 0.0 || sqrt_det <= 0.0)
        return YM_ERR_REFERENCE_MATRIX_NOT_POSITIVE_DEFINITE;
    const double avg = 0.5 * d1 + 0.5 * d2;
    const double plus = avg + off, minus = avg - off;
    const double cross = 0.5 * d1 - 0.5 * d2;
    if (!fin(avg) || !fin(plus) || !fin(minus) || !fin(cross))
        return YM_ERR_NON_FINITE_ACCUMULATOR;
    const double t1 = plus / plus_den, t2 = minus / minus_den, toff = cross / sqrt_det;
    if (!fin(t1) || !fin(t2) || !fin(toff)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    if (toff == 0.0 && t1 == t2) return YM_ERR_DEGENERATE_PRINCIPAL_EIGENVECTOR;
    const double mid = 0.5 * t1 + 0.5 * t2;
    const double half = 0.5 * t1 - 0.5 * t2;
    const double radius = std::hypot(half, toff);
    if (!fin(mid) || !fin(half) || !fin(radius)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    if (radius == 0.0) return YM_ERR_DEGENERATE_PRINCIPAL_EIGENVECTOR;
    if (mid >= 0.0) {
        const double root = mid + radius;
        if (!fin(root)) return YM_ERR_NON_FINITE_ACCUMULATOR;
        *out = root;
        return YM_OK;
    }
    // negative midpoint: the principal root from the product of the roots,
    // det(C1)/det(C0) = lambda_small * lambda_principal
    const double smaller = mid - radius;
    if (!fin(smaller) || smaller == 0.0) return YM_ERR_NON_FINITE_ACCUMULATOR;
    double det1, root;
    if (int32_t st = compensated_det(d1, d2, off, &det1)) return st;
    if (int32_t st = divide_by_product(det1, ref_det, smaller, &root)) return st;
    if (!fin(root)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    *out = root;
    return YM_OK;
}

// stable_generalized_principal_eigenvalue (glueball_scalar_variational.rs:380-464)
int32_t principal_eigenvalue(const M2 &ref_in, const M2 &diag_in, double *out) {
    M2 ref, dg;
    if (int32_t st = symmetrized(ref_in, &ref)) return st;
    if (int32_t st = symmetrized(diag_in, &dg)) return st;
    const double r1 = ref.a[0][0], r2 = ref.a[1][1];
    if (!fin(r1) || !fin(r2) || r1 <= 0.0 || r2 <= 0.0)
        return YM_ERR_REFERENCE_MATRIX_NOT_POSITIVE_DEFINITE;
    const double rscale = std::sqrt(r1) * std::sqrt(r2);
    if (!fin(rscale) || rscale <= 0.0) return YM_ERR_REFERENCE_MATRIX_NOT_POSITIVE_DEFINITE;
    const double roff = ref.a[0][1] / rscale;
    const double rdet = 1.0 - roff * roff;
    if (!fin(roff) || !fin(rdet) || rdet <= kPdPivotTolerance)
        return YM_ERR_REFERENCE_MATRIX_NOT_POSITIVE_DEFINITE;
    const double d1 = dg.a[0][0] / r1, d2 = dg.a[1][1] / r2, off = dg.a[0][1] / rscale;
    if (!fin(d1) || !fin(d2) || !fin(off)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    if (roff == 0.0 && off == 0.0) {
        if (d1 == d2) return YM_ERR_DEGENERATE_PRINCIPAL_EIGENVECTOR;
        *out = std::fmax(d1, d2);
        return YM_OK;
    }
    const int32_t st = characteristic_root(rdet, roff, d1, d2, off, out);
    if (st != YM_ERR_NON_FINITE_ACCUMULATOR) return st;
    // the unscaled solve overflowed: solve at unit scale and scale back
    const double scale = std::fmax(std::fmax(std::fabs(d1), std::fabs(d2)), std::fabs(off));
    if (!fin(scale) || scale <= 0.0) return YM_ERR_NON_FINITE_ACCUMULATOR;
    double root;
    if (int32_t st2 = characteristic_root(rdet, roff, d1 / scale, d2 / scale, off / scale, &root))
        return st2;
    const double r = scale * root;
    if (!fin(r)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    *out = r;
    return YM_OK;
}

// The C0 normalisation every whitening step shares.
struct RefMetric {
    double first, second, scale, off, det;
};

// stable_cholesky_whitened (glueball_scalar_variational.rs:481-566): L^-1 M
// L^-T for C0 = L L^T, written through C0's unit-diagonal normalisation.
int32_t whiten(const M2 &m_in, const RefMetric &g, M2 *out) {
    M2 m;
    if (int32_t st = symmetrized(m_in, &m)) return st;
    if (!fin(g.first) || !fin(g.second) || !fin(g.scale) || !fin(g.off) ||
        !fin(g.det) || g.first <= 0.0 || g.second <= 0.0 || g.scale <= 0.0 || g.det <= 0.0)
        return YM_ERR_NON_FINITE_ACCUMULATOR;
    const double n1 = m.a[0][0] / g.first, n2 = m.a[1][1] / g.second, noff = m.a[0][1] / g.scale;
    if (!fin(n1) || !fin(n2) || !fin(noff)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    if (g.off == 0.0) {
        *out = M2{{{n1, noff}, {noff, n2}}};
        return YM_OK;
    }
    const double scale = std::fmax(std::fmax(std::fabs(n1), std::fabs(n2)), std::fabs(noff));
    if (!fin(scale)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    if (scale == 0.0) {
        *out = M2{{{0.0, 0.0}, {0.0, 0.0}}};
        return YM_OK;
    }
    const double f = n1 / scale, s = n2 / scale, o = noff / scale;
    const double sqrt_det = std::sqrt(g.det);
    if (!fin(sqrt_det) || sqrt_det <= 0.0) return YM_ERR_REFERENCE_MATRIX_NOT_POSITIVE_DEFINITE;
    const double w11 = f;
    const double w12 = std::fma(-g.off, f, o) / sqrt_det;
    const double lower = std::fma(g.off, g.off * f, std::fma(-2.0 * g.off, o, s));
    const double w22 = lower / g.det;
    if (!fin(w11) || !fin(w12) || !fin(w22)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    const M2 r{{{w11 * scale, w12 * scale}, {w12 * scale, w22 * scale}}};
    if (!m2_finite(r)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    *out = r;
    return YM_OK;
}

// stable_whitened_projection (glueball_scalar_variational.rs:568-603): v^T
// (whitened M) v for the metric-normalised principal vector v.
int32_t whitened_projection(const M2 &m_in, const M2 &c0, const RefMetric &g, const double v[2],
                            double *out) {
    M2 m;
    if (int32_t st = symmetrized(m_in, &m)) return st;
    if (m2_equal(m, c0)) {
        *out = 1.0;   // the normalisation v^T C0 v = 1, replayed exactly at equal lags
        return YM_OK;
    }
    M2 w;
    if (int32_t st = whiten(m, g, &w)) return st;
    const double row0 = std::fma(w.a[0][0], v[0], w.a[0][1] * v[1]);
    const double row1 = std::fma(w.a[1][0], v[0], w.a[1][1] * v[1]);
    const double value = std::fma(v[0], row0, v[1] * row1);
    if (!fin(value)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    *out = value;
    return YM_OK;
}

// principal_generalized_projection (glueball_scalar_variational.rs:746-925)
int32_t principal_projection(const double *mats, int64_t nt, int64_t t0, int64_t t1,
                             ym_principal_projection *res, double *projected) {
    if (int32_t st = validate_series(mats, nt)) return st;
    if (t0 != 1 || t1 != 2 || t1 >= nt) return YM_ERR_INVALID_REFERENCE_TIMES;
    M2 c0, c1;
    if (int32_t st = symmetrized(load_m2(mats + 4 * t0), &c0)) return st;
    if (int32_t st = symmetrized(load_m2(mats + 4 * t1), &c1)) return st;
    const double a = c0.a[0][0], d = c0.a[1][1];
    if (!fin(a) || !fin(d) || a <= 0.0 || d <= 0.0)
        return YM_ERR_REFERENCE_MATRIX_NOT_POSITIVE_DEFINITE;
    const double dscale = std::sqrt(a) * std::sqrt(d);
    if (!fin(dscale) || dscale <= 0.0) return YM_ERR_REFERENCE_MATRIX_NOT_POSITIVE_DEFINITE;
    const double noff = c0.a[0][1] / dscale;
    if (!fin(noff)) return YM_ERR_REFERENCE_MATRIX_NOT_POSITIVE_DEFINITE;
    const double ndet = 1.0 - noff * noff;
    if (!fin(ndet) || ndet <= kPdPivotTolerance) return YM_ERR_REFERENCE_MATRIX_NOT_POSITIVE_DEFINITE;
    // C0 = L L^T
    const double l00 = std::sqrt(a), l10 = c0.a[1][0] / l00, l11 = std::sqrt(d) * std::sqrt(ndet);
    if (!fin(l00) || !fin(l10) || !fin(l11) || l00 <= 0.0 || l11 <= 0.0)
        return YM_ERR_REFERENCE_MATRIX_NOT_POSITIVE_DEFINITE;
    double q;
    if (int32_t st = divide_by_product(l10, l00, l11, &q)) return st;
    const double inv_l[2][2] = {{1.0 / l00, 0.0}, {-q, 1.0 / l11}};
    const RefMetric g{a, d, dscale, noff, ndet};
    M2 w;
    if (int32_t st = whiten(c1, g, &w)) return st;
    const double wa = w.a[0][0], wd = w.a[1][1], woff = w.a[0][1];
    if (!fin(wa) || !fin(wd) || !fin(woff)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    double lambda;
    if (int32_t st = principal_eigenvalue(c0, c1, &lambda)) return st;
    if (!fin(lambda) || lambda <= 0.0) return YM_ERR_NON_POSITIVE_PRINCIPAL_EIGENVALUE;
    // principal direction of the whitened matrix from its 2x2 radius
    double e[2];
    if (woff != 0.0) {
        const double half = 0.5 * wa - 0.5 * wd;
        const double radius = std::hypot(half, woff);
        if (!fin(half) || !fin(radius) || radius == 0.0)
            return YM_ERR_DEGENERATE_PRINCIPAL_EIGENVECTOR;
        const double cs = std::fmax(std::fmax(std::fabs(radius), std::fabs(half)), std::fabs(woff));
        if (!fin(cs) || cs <= 0.0) return YM_ERR_DEGENERATE_PRINCIPAL_EIGENVECTOR;
        if (half >= 0.0) {
            e[0] = radius / cs + half / cs;
            e[1] = woff / cs;
        } else {
            e[0] = woff / cs;
            e[1] = radius / cs - half / cs;
        }
    } else if (wa > wd) {
        e[0] = 1.0;
        e[1] = 0.0;
    } else if (wd > wa) {
        e[0] = 0.0;
        e[1] = 1.0;
    } else {
        return YM_ERR_DEGENERATE_PRINCIPAL_EIGENVECTOR;
    }
    const double en = std::hypot(e[0], e[1]);
    if (!fin(en) || en <= 0.0) return YM_ERR_DEGENERATE_PRINCIPAL_EIGENVECTOR;
    e[0] /= en;
    e[1] /= en;
    // coefficients = L^-T e, normalised so that |L^T c| = 1
    double c[2] = {inv_l[0][0] * e[0] + inv_l[1][0] * e[1], inv_l[0][1] * e[0] + inv_l[1][1] * e[1]};
    {
        const double first = l00 * c[0] + l10 * c[1], second = l11 * c[1];
        const double norm = std::hypot(first, second);
        if (!fin(first) || !fin(second) || !fin(norm) || norm <= 0.0)
            return YM_ERR_PROJECTION_NORMALIZATION_FAILURE;
        c[0] /= norm;
        c[1] /= norm;
    }
    // sign: first coefficient positive, or the second when the first is ~0
    if (std::fabs(c[0]) > kPdPivotTolerance) {
        if (c[0] < 0.0) {
            c[0] = -c[0];
            c[1] = -c[1];
        }
    } else if (c[1] < 0.0) {
        c[0] = -c[0];
        c[1] = -c[1];
    }
    const double mv[2] = {l00 * c[0] + l10 * c[1], l11 * c[1]};
    if (!fin(mv[0]) || !fin(mv[1])) return YM_ERR_PROJECTION_NORMALIZATION_FAILURE;
    const double mn = std::hypot(mv[0], mv[1]);
    const double refproj = mn * mn;
    if (!fin(refproj) || std::fabs(refproj - 1.0) > kNormalizationTolerance)
        return YM_ERR_PROJECTION_NORMALIZATION_FAILURE;
    for (int64_t t = 0; t < nt; ++t) {
        if (t == t0) {
            projected[t] = 1.0;
        } else if (t == t1) {
            projected[t] = lambda;
        } else {
            double v;
            if (int32_t st = whitened_projection(load_m2(mats + 4 * t), c0, g, mv, &v)) return st;
            projected[t] = v;
        }
    }
    res->reference_time = t0;
    res->diagonalization_time = t1;
    res->principal_eigenvalue = lambda;
    res->coefficients[0] = c[0];
    res->coefficients[1] = c[1];
    return YM_OK;
}

// Same as ym_periodic_connected_estimator's connected part, over one
// operator of the interleaved [cfg][t][2] samples (glueball_correlators.rs:111-172).
int32_t operator_connected(const double *samples, int64_t ncfg, int64_t nt, int op,
                           std::vector<double> *connected) {
    const int64_t len = ncfg * nt;
    if (len == 0) return YM_ERR_CORRELATOR_SHAPE_MISMATCH;
    double ms = 0.0;
    for (int64_t i = 0; i < len; ++i) {
        const double v = samples[2 * i + op];
        if (!fin(v)) return YM_ERR_NON_FINITE_OBSERVABLE;
        ms += v;
        if (!fin(ms)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    }
    const double mean = ms / (double)len;
    if (!fin(mean)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    const double msq = mean * mean;
    if (!fin(msq)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    connected->assign((size_t)nt, 0.0);
    for (int64_t tau = 0; tau < nt; ++tau) {
        double s = 0.0;
        for (int64_t c = 0; c < ncfg; ++c)
            for (int64_t t = 0; t < nt; ++t) {
                const double p = samples[2 * (c * nt + t) + op] * samples[2 * (c * nt + (t + tau) % nt) + op];
                if (!fin(p)) return YM_ERR_NON_FINITE_ACCUMULATOR;
                s += p;
                if (!fin(s)) return YM_ERR_NON_FINITE_ACCUMULATOR;
            }
        const double raw = s / (double)len;
        const double cv = raw - msq;
        if (!fin(raw) || !fin(cv)) return YM_ERR_NON_FINITE_ACCUMULATOR;
        (*connected)[(size_t)tau] = cv;
    }
    return YM_OK;
}

// scalar_variational_connected_correlator (glueball_scalar_variational.rs:628-744)
// from the per-slice operator samples (plaquette, rectangle) of every
// configuration.
int32_t variational_correlator(const double *samples, int64_t ncfg, int64_t nt, double *means,
                               double *mats) {
    if (ncfg <= 0) return YM_ERR_EMPTY_CONFIGURATION_SET;
    if (ncfg > kMaxConfigurations) return YM_ERR_TOO_MANY_CONFIGURATIONS;
    if (nt < 3) return YM_ERR_TIME_EXTENT_TOO_SMALL;
    if (nt > kVarMaxTimeExtent) return YM_ERR_TIME_EXTENT_TOO_LARGE;
    const int64_t count = ncfg * nt;
    double sums[2] = {0.0, 0.0};
    for (int64_t i = 0; i < count; ++i) {
        const double p = samples[2 * i], r = samples[2 * i + 1];
        if (!fin(p) || !fin(r)) return YM_ERR_NON_FINITE_OBSERVABLE;
        sums[0] += p;
        if (!fin(sums[0])) return YM_ERR_NON_FINITE_ACCUMULATOR;
        sums[1] += r;
        if (!fin(sums[1])) return YM_ERR_NON_FINITE_ACCUMULATOR;
    }
    const double norm = (double)count;
    const double vm[2] = {sums[0] / norm, sums[1] / norm};
    if (!fin(vm[0]) || !fin(vm[1])) return YM_ERR_NON_FINITE_ACCUMULATOR;
    for (int64_t tau = 0; tau < nt; ++tau) {
        double pp = 0.0, rr = 0.0, pr = 0.0, rp = 0.0;
        for (int64_t c = 0; c < ncfg; ++c)
            for (int64_t t = 0; t < nt; ++t) {
                const double *x = samples + 2 * (c * nt + t);
                const double *y = samples + 2 * (c * nt + (t + tau) % nt);
                pp += x[0] * y[0];
                rr += x[1] * y[1];
                pr += x[0] * y[1];
                rp += x[1] * y[0];
                if (!fin(pp) || !fin(rr) || !fin(pr) || !fin(rp))
                    return YM_ERR_NON_FINITE_ACCUMULATOR;
            }
        const double cross = 0.5 * (pr / norm + rp / norm) - vm[0] * vm[1];
        double *m = mats + 4 * tau;
        m[0] = pp / norm - vm[0] * vm[0];
        m[1] = cross;
        m[2] = cross;
        m[3] = rr / norm - vm[1] * vm[1];
        if (!fin(m[0]) || !fin(m[1]) || !fin(m[3])) return YM_ERR_NON_FINITE_ACCUMULATOR;
    }
    // the diagonal must replay the frozen single-operator correlators
    std::vector<double> cp, cr;
    if (int32_t st = operator_connected(samples, ncfg, nt, 0, &cp)) return st;
    if (int32_t st = operator_connected(samples, ncfg, nt, 1, &cr)) return st;
    for (int64_t tau = 0; tau < nt; ++tau)
        if (std::fabs(mats[4 * tau] - cp[(size_t)tau]) > kSymmetryTolerance ||
            std::fabs(mats[4 * tau + 3] - cr[(size_t)tau]) > kSymmetryTolerance)
            return YM_ERR_CORRELATOR_SHAPE_MISMATCH;
    means[0] = vm[0];
    means[1] = vm[1];
    return YM_OK;
}

double periodic_weight(double mass, int64_t t, int64_t nt) {   // glueball_scalar_variational.rs:927-929
    return std::exp(-mass * (double)t) + std::exp(-mass * (double)(nt - t));
}

}  // namespace

extern "C" {

int32_t ym_cosh_effective_mass_with_jackknife(const double *full, int64_t time_extent,
                                              const double *const *jackknife,
                                              const int64_t *jackknife_lengths, int64_t n_replicas,
                                              const uint64_t *lags, int64_t n_lags,
                                              ym_effective_mass_point *points) {
    if (!full || (n_replicas > 0 && (!jackknife || !jackknife_lengths)) || (n_lags > 0 && !lags) ||
        !points)
        return YM_ERR_NULL_ARGUMENT;
    for (int64_t r = 0; r < n_replicas; ++r)
        if (!jackknife[r] && jackknife_lengths[r] > 0) return YM_ERR_NULL_ARGUMENT;
    return effective_mass_series(full, time_extent, Replicas{jackknife, jackknife_lengths, n_replicas},
                                 lags, n_lags, points);
}

int32_t ym_analytic_periodic_single_state(int64_t time_extent, double mass, double amplitude,
                                          double *correlator) {
    if (!correlator) return YM_ERR_NULL_ARGUMENT;
    return single_state(time_extent, mass, amplitude, correlator);
}

int32_t ym_correlated_scalar_fit(const double *full, int64_t time_extent,
                                 const double *const *jackknife, const int64_t *jackknife_lengths,
                                 int64_t n_replicas, const ym_fit_window *candidates,
                                 int64_t n_candidates, ym_scalar_fit_result *result) {
    if (!full || (n_replicas > 0 && (!jackknife || !jackknife_lengths)) ||
        (n_candidates > 0 && !candidates) || !result)
        return YM_ERR_NULL_ARGUMENT;
    for (int64_t r = 0; r < n_replicas; ++r)
        if (!jackknife[r] && jackknife_lengths[r] > 0) return YM_ERR_NULL_ARGUMENT;
    return scalar_fit(full, time_extent, Replicas{jackknife, jackknife_lengths, n_replicas}, candidates,
                      n_candidates, result);
}

int32_t ym_scalar_fit_window_covariance(const double *const *jackknife,
                                        const int64_t *jackknife_lengths, int64_t n_replicas,
                                        ym_fit_window window, double *covariance) {
    if ((n_replicas > 0 && (!jackknife || !jackknife_lengths)) || !covariance)
        return YM_ERR_NULL_ARGUMENT;
    Dense cov(0);
    if (int32_t st = window_covariance(Replicas{jackknife, jackknife_lengths, n_replicas}, window, &cov))
        return st;
    for (size_t i = 0; i < cov.v.size(); ++i) covariance[i] = cov.v[i];
    return YM_OK;
}

int32_t ym_scalar_fit_invert_covariance(const double *matrix, int64_t n, double *inverse) {
    if (!matrix || !inverse) return YM_ERR_NULL_ARGUMENT;
    if (n < 0 || n > 64) return YM_ERR_INVALID_ARGUMENT;
    Dense m(n), inv(0);
    for (int64_t i = 0; i < n * n; ++i) m.v[(size_t)i] = matrix[i];
    if (int32_t st = invert(m, &inv)) return st;
    for (int64_t i = 0; i < n * n; ++i) inverse[i] = inv.v[(size_t)i];
    return YM_OK;
}

int32_t ym_maximum_off_diagonal_correlation(const double *covariance, int64_t n, double *out) {
    if (!covariance || !out) return YM_ERR_NULL_ARGUMENT;
    if (n < 0) return YM_ERR_INVALID_ARGUMENT;
    Dense m(n);
    for (int64_t i = 0; i < n * n; ++i) m.v[(size_t)i] = covariance[i];
    return max_off_diagonal(m, out);
}

// canonical_scalar_fit_fixture (glueball_scalar_fit.rs:652-690)
int32_t ym_canonical_scalar_fit_fixture(double *full, double *jackknife, ym_fit_window *candidates) {
    if (!full || !jackknife || !candidates) return YM_ERR_NULL_ARGUMENT;
    if (int32_t st = single_state(16, 0.5, 1.0, full)) return st;
    const double perturbation = 0.005, shared = 0.25;   // glueball_scalar_fit.rs:25-26
    for (int r = 0; r < 8; ++r) {
        // row r of the order-8 Sylvester Hadamard matrix: (-1)^popcount(r & c)
        double h[8];
        for (int c = 0; c < 8; ++c) h[c] = (__builtin_popcount((unsigned)(r & c)) & 1) ? -1.0 : 1.0;
        double *rep = jackknife + 16 * r;
        for (int t = 0; t < 16; ++t) rep[t] = full[t];
        for (int t = 1; t <= 7; ++t) {
            const double pattern = t == 1 ? h[1] : h[t] + shared * h[1];
            rep[t] = full[t] * (1.0 + perturbation * pattern);
        }
    }
    candidates[0] = ym_fit_window{1, 3};
    candidates[1] = ym_fit_window{2, 5};
    candidates[2] = ym_fit_window{3, 6};
    return YM_OK;
}

int32_t ym_scalar_variational_connected_correlator(const double *samples, int64_t n_configurations,
                                                   int64_t time_extent, double *vacuum_means,
                                                   double *matrices) {
    if (!samples || !vacuum_means || !matrices) return YM_ERR_NULL_ARGUMENT;
    if (n_configurations > 0 && time_extent > 0 && n_configurations > INT64_MAX / time_extent)
        return YM_ERR_SAMPLE_COUNT_OVERFLOW;
    return variational_correlator(samples, n_configurations, time_extent, vacuum_means, matrices);
}

int32_t ym_principal_generalized_projection(const double *matrices, int64_t time_extent,
                                            int64_t reference_time, int64_t diagonalization_time,
                                            ym_principal_projection *result, double *projected) {
    if (!matrices || !result || !projected) return YM_ERR_NULL_ARGUMENT;
    return principal_projection(matrices, time_extent, reference_time, diagonalization_time, result,
                                projected);
}

// canonical_two_state_matrices (glueball_scalar_variational.rs:931-951)
int32_t ym_canonical_two_state_matrices(double *matrices) {
    if (!matrices) return YM_ERR_NULL_ARGUMENT;
    const int64_t nt = 16;
    const double gm = 0.4, em = 0.9, ga = 1.2, ea = 0.8;   // glueball_scalar_variational.rs:30-36
    const double gc[2] = {1.0, 0.5}, ec[2] = {0.25, 1.0};
    for (int64_t t = 0; t < nt; ++t) {
        const double g = ga * periodic_weight(gm, t, nt), e = ea * periodic_weight(em, t, nt);
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 2; ++c) matrices[4 * t + 2 * r + c] = g * gc[r] * gc[c] + e * ec[r] * ec[c];
    }
    return YM_OK;
}

// max_matrix_series_residual (glueball_scalar_variational.rs:953-975)
int32_t ym_max_matrix_series_residual(const double *first, int64_t n_first, const double *second,
                                      int64_t n_second, double *out) {
    if (!first || !second || !out) return YM_ERR_NULL_ARGUMENT;
    if (int32_t st = validate_series(first, n_first)) return st;
    if (int32_t st = validate_series(second, n_second)) return st;
    if (n_first != n_second) return YM_ERR_CORRELATOR_SHAPE_MISMATCH;
    double mx = 0.0;
    for (int64_t i = 0; i < 4 * n_first; ++i) {
        const double r = std::fabs(first[i] - second[i]);
        if (!fin(r)) return YM_ERR_NON_FINITE_ACCUMULATOR;
        mx = std::fmax(mx, r);
    }
    *out = mx;
    return YM_OK;
}

}  // extern "C"

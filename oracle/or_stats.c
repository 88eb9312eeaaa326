/* or_stats.c -- CPU oracle: chain diagnostics, sampling efficiency, connected
 * correlators, delete-one jackknife and jackknife covariance, restated from
 * the reference crate.  TEST INFRASTRUCTURE ONLY (see or_internal.h).
 *
 *   diagnostics                 reference/rust/src/su2_ensemble.rs:375-463
 *   evaluate                    reference/rust/src/sampling_efficiency.rs:57-135
 *   periodic estimator          reference/rust/src/glueball_correlators.rs:111-172
 *   connected_from_samples      reference/rust/src/glueball_scalar_production.rs:383-443
 *   jackknife_covariance        reference/rust/src/glueball_scalar_fit.rs:276-322
 */
#include <stdlib.h>

#include "oracle.h"
#include "or_internal.h"

/* autocorrelation must hold max_lag+1 doubles. */
int or_diagnostics(const double *v, int64_t n, int64_t max_lag, or_diagnostics_out *o,
                   double *autocorrelation) {
    if (n < 2) return YM_ERR_TOO_FEW_MEASUREMENTS;
    if (max_lag >= n) return YM_ERR_AUTOCORRELATION_LAG_OUT_OF_RANGE;
    for (int64_t i = 0; i < n; ++i) if (!isfinite(v[i])) return YM_ERR_NON_FINITE_STATISTIC;
    double nf = (double)n;
    double s = -0.0;
    for (int64_t i = 0; i < n; ++i) s += v[i];
    double mean = s / nf;
    double q = -0.0;
    for (int64_t i = 0; i < n; ++i) { double d = v[i] - mean; q += d * d; }
    double var = q / nf;
    if (!isfinite(mean) || !isfinite(var)) return YM_ERR_NON_FINITE_STATISTIC;
    autocorrelation[0] = 1.0;
    o->mean = mean;
    o->variance = var;
    if (var == 0.0) {
        for (int64_t k = 1; k <= max_lag; ++k) autocorrelation[k] = 0.0;
        o->positive_window_lag = 0;
        o->integrated_autocorrelation_time = 0.5;
        o->effective_sample_size = nf;
        o->standard_error = 0.0;
        return YM_OK;
    }
    double tau = 0.5;
    int64_t window_lag = 0;
    int open = 1;
    for (int64_t lag = 1; lag <= max_lag; ++lag) {
        int64_t pairs = n - lag;
        double c = -0.0;
        for (int64_t i = 0; i < pairs; ++i) c += (v[i] - mean) * (v[i + lag] - mean);
        c = c / (double)pairs;
        double rho = c / var;
        if (!isfinite(rho)) return YM_ERR_NON_FINITE_STATISTIC;
        autocorrelation[lag] = rho;
        if (open && rho > 0.0) {
            tau += rho;
            window_lag = lag;
        } else {
            open = 0;
        }
    }
    if (!isfinite(tau) || tau < 0.5) return YM_ERR_NON_FINITE_STATISTIC;
    double ess = fmin(nf / (2.0 * tau), nf);
    double se = sqrt(var / ess);
    if (!isfinite(ess) || !isfinite(se)) return YM_ERR_NON_FINITE_STATISTIC;
    o->positive_window_lag = window_lag;
    o->integrated_autocorrelation_time = tau;
    o->effective_sample_size = ess;
    o->standard_error = se;
    return YM_OK;
}

/* sampling_efficiency.rs:57-135.  log_weights may be NULL (unit weights). */
int or_sampling_efficiency(const double *v, int64_t n, const double *log_weights, int64_t max_lag,
                           double setup, double thermalization, double sampling,
                           or_efficiency_out *o, double *autocorrelation) {
    if (n < 2 || n > 4096) return YM_ERR_INVALID_LENGTH;
    if (max_lag == 0 || max_lag >= n || max_lag > 256) return YM_ERR_INVALID_LAG;
    double costs[3] = {setup, thermalization, sampling};
    for (int i = 0; i < 3; ++i)
        if (!isfinite(costs[i]) || costs[i] < 0.0) return YM_ERR_INVALID_COST;
    if (sampling == 0.0) return YM_ERR_INVALID_COST;
    double total = setup + thermalization + sampling;
    if (!isfinite(total)) return YM_ERR_INVALID_COST;
    double eff = 1.0;
    if (log_weights) {
        double mx = -INFINITY;
        for (int64_t i = 0; i < n; ++i) {
            if (!isfinite(log_weights[i])) return YM_ERR_INVALID_WEIGHT;
            mx = fmax(mx, log_weights[i]);
        }
        double sum = 0.0, sq = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            double w = exp(log_weights[i] - mx);
            sum += w;
            sq += w * w;
        }
        eff = fmin((sum / (double)n) * (sum / sq), 1.0);
    }
    int constant = 1;
    for (int64_t i = 1; i < n; ++i) if (v[i] != v[0]) { constant = 0; break; }
    if (constant) return YM_ERR_DEGENERATE_OBSERVABLE;
    int st = or_diagnostics(v, n, max_lag, &o->diagnostics, autocorrelation);
    if (st) return YM_ERR_INVALID_DIAGNOSTIC;
    if (o->diagnostics.variance <= 0.0) return YM_ERR_DEGENERATE_OBSERVABLE;
    if (!isfinite(o->diagnostics.standard_error) || o->diagnostics.standard_error <= 0.0)
        return YM_ERR_NON_FINITE_RESULT;
    o->reweighting_efficiency = eff;
    o->weight_only_ess = (double)n * eff;
    o->combined_ess_proxy = o->diagnostics.effective_sample_size * eff;
    o->total_cost = total;
    o->sampling_cost_per_effective_sample_proxy = sampling / o->combined_ess_proxy;
    o->total_cost_per_effective_sample_proxy = total / o->combined_ess_proxy;
    double chk[5] = {eff, o->weight_only_ess, o->combined_ess_proxy,
                     o->sampling_cost_per_effective_sample_proxy,
                     o->total_cost_per_effective_sample_proxy};
    for (int i = 0; i < 5; ++i) if (!isfinite(chk[i]) || chk[i] <= 0.0) return YM_ERR_NON_FINITE_RESULT;
    return YM_OK;
}

/* glueball_correlators.rs:111-172: samples laid out [configuration][time]. */
int or_periodic_connected_estimator(const double *samples, int64_t ncfg, int64_t nt,
                                    double *vacuum_mean, double *raw, double *connected) {
    int64_t len = ncfg * nt;
    if (len == 0) return YM_ERR_CORRELATOR_SHAPE_MISMATCH;
    double ms = 0.0;
    for (int64_t i = 0; i < len; ++i) {
        if (!isfinite(samples[i])) return YM_ERR_NON_FINITE_OBSERVABLE;
        ms += samples[i];
        if (!isfinite(ms)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    }
    double mean = ms / (double)len;
    if (!isfinite(mean)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    double msq = mean * mean;
    if (!isfinite(msq)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    for (int64_t tau = 0; tau < nt; ++tau) {
        double s = 0.0;
        for (int64_t c = 0; c < ncfg; ++c) {
            const double *row = samples + c * nt;
            for (int64_t t = 0; t < nt; ++t) {
                double p = row[t] * row[(t + tau) % nt];
                if (!isfinite(p)) return YM_ERR_NON_FINITE_ACCUMULATOR;
                s += p;
                if (!isfinite(s)) return YM_ERR_NON_FINITE_ACCUMULATOR;
            }
        }
        double r = s / (double)len;
        double cval = r - msq;
        if (!isfinite(r) || !isfinite(cval)) return YM_ERR_NON_FINITE_ACCUMULATOR;
        raw[tau] = r;
        connected[tau] = cval;
    }
    *vacuum_mean = mean;
    return YM_OK;
}

/* glueball_scalar_production.rs:383-443: omitted < 0 means keep every row. */
int or_connected_from_samples(const double *samples, int64_t ncfg, int64_t nt, int64_t omitted,
                              double *connected) {
    if (ncfg == 0) return YM_ERR_EMPTY_CONFIGURATION_SET;
    if (nt == 0) return YM_ERR_CONFIGURATION_SHAPE_MISMATCH;
    int64_t kept;
    if (omitted >= 0) {
        if (omitted >= ncfg) return YM_ERR_CONFIGURATION_SHAPE_MISMATCH;
        kept = ncfg - 1;
    } else {
        kept = ncfg;
    }
    if (kept == 0) return YM_ERR_EMPTY_CONFIGURATION_SET;
    int64_t count = kept * nt;
    double ms = 0.0;
    for (int64_t c = 0; c < ncfg; ++c) {
        if (c == omitted) continue;
        for (int64_t t = 0; t < nt; ++t) {
            double v = samples[c * nt + t];
            if (!isfinite(v)) return YM_ERR_NON_FINITE_STATISTIC;
            ms += v;
        }
    }
    double mean = ms / (double)count;
    double msq = mean * mean;
    if (!isfinite(mean) || !isfinite(msq)) return YM_ERR_NON_FINITE_STATISTIC;
    for (int64_t tau = 0; tau < nt; ++tau) {
        double s = 0.0;
        for (int64_t c = 0; c < ncfg; ++c) {
            if (c == omitted) continue;
            const double *row = samples + c * nt;
            for (int64_t t = 0; t < nt; ++t) s += row[t] * row[(t + tau) % nt];
        }
        double v = s / (double)count - msq;
        if (!isfinite(v)) return YM_ERR_NON_FINITE_STATISTIC;
        connected[tau] = v;
    }
    return YM_OK;
}

/* glueball_scalar_fit.rs:276-322: replicas laid out [replica][tau]; the
 * window is [start, end] inclusive; out is points x points row-major. */
int or_jackknife_covariance(const double *replicas, int64_t nrep, int64_t nt, int64_t start,
                            int64_t end, double *out) {
    if (end < start || start < 0) return YM_ERR_INVALID_CANDIDATE_WINDOW;
    int64_t points = end - start + 1;
    if (nrep <= points) return YM_ERR_INSUFFICIENT_REPLICATES_FOR_COVARIANCE;
    if (end >= nt) return YM_ERR_INVALID_CANDIDATE_WINDOW;
    double *means = calloc((size_t)points, sizeof(double));
    if (!means) return YM_ERR_ALLOCATION_FAILED;
    for (int64_t r = 0; r < nrep; ++r)
        for (int64_t c = 0; c < points; ++c) {
            double v = replicas[r * nt + start + c];
            if (!isfinite(v)) { free(means); return YM_ERR_NON_FINITE_STATISTIC; }
            means[c] += v;
        }
    double n = (double)nrep;
    for (int64_t c = 0; c < points; ++c) means[c] /= n;
    for (int64_t i = 0; i < points * points; ++i) out[i] = 0.0;
    for (int64_t r = 0; r < nrep; ++r)
        for (int64_t a = 0; a < points; ++a) {
            double left = replicas[r * nt + start + a] - means[a];
            for (int64_t b = 0; b < points; ++b) {
                double right = replicas[r * nt + start + b] - means[b];
                out[a * points + b] += left * right;
            }
        }
    double factor = (n - 1.0) / n;
    for (int64_t i = 0; i < points * points; ++i) {
        out[i] *= factor;
        if (!isfinite(out[i])) { free(means); return YM_ERR_NON_FINITE_STATISTIC; }
    }
    free(means);
    return YM_OK;
}

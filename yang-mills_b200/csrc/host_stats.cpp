// host_stats.cpp -- host-side FP64 analysis of the drop-in boundary: stream
// seeds, the paired proposal-angle grid, chain diagnostics and the sampling
// efficiency report.  These are the reference's own host computations on
// measurement series (tiny, sequential FP64); they sit beside the device
// kernels so that run_chain-style callers get the reference's numbers.
// Compiled with -ffp-contract=off: every sum is left to right as in the
// reference's iterator chains.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "../../include/ymgpu.h"

namespace {

constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ULL;
constexpr uint64_t kStreamDomain = 0x535533454e535631ULL;   // su3_ensemble.rs:23

uint64_t mix64(uint64_t v) {   // su2_ensemble.rs:46-50
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
    return v ^ (v >> 31);
}

}  // namespace

extern "C" {

uint64_t ym_derive_chain_seed(uint64_t master_seed, uint64_t chain_id) {   // su2_ensemble.rs:52-55
    return mix64(master_seed ^ ((chain_id + 1) * kGolden));
}

uint64_t ym_derive_su3_chain_seed(uint64_t master_seed, uint64_t chain_id) {   // su3_ensemble.rs:189-192
    return mix64(master_seed ^ kStreamDomain ^ ((chain_id + 1) * kGolden));
}

uint64_t ym_splitmix64_at(uint64_t seed, uint64_t n) { return mix64(seed + (n + 1) * kGolden); }

int32_t ym_proposal_angle_from_u64(uint64_t raw, double proposal_angle, double *out) {
    if (!out) return YM_ERR_NULL_ARGUMENT;               // su3_ensemble.rs:199-213
    if (!std::isfinite(proposal_angle) || proposal_angle < 1.0e-8 || proposal_angle > 1.0)
        return YM_ERR_PROPOSAL_ANGLE_OUTSIDE_REFERENCE_RANGE;
    const uint64_t m = raw & ((uint64_t(1) << 52) - 1);
    const double magnitude = proposal_angle * (double)(m * 2 + 1) * (1.0 / 9007199254740992.0);
    const double sign = (raw >> 63) == 0 ? -1.0 : 1.0;
    const double a = sign * magnitude;
    if (!std::isfinite(a) || a == 0.0 || std::fabs(a) >= proposal_angle)
        return YM_ERR_NON_FINITE_STATISTIC;
    *out = a;
    return YM_OK;
}

// su2_ensemble.rs:375-463: mean, variance, autocorrelation up to max_lag,
// integrated time over the initial positive window, ESS = min(n/(2 tau), n).
int32_t ym_diagnostics(const double *v, int64_t n, int64_t max_lag, ym_chain_diagnostics *o,
                       double *autocorrelation) {
    if (!v || !o || !autocorrelation) return YM_ERR_NULL_ARGUMENT;
    if (n < 2) return YM_ERR_TOO_FEW_MEASUREMENTS;
    if (max_lag >= n || max_lag < 0) return YM_ERR_AUTOCORRELATION_LAG_OUT_OF_RANGE;
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(v[i])) return YM_ERR_NON_FINITE_STATISTIC;
    const double nf = (double)n;
    double s = -0.0;
    for (int64_t i = 0; i < n; ++i) s += v[i];
    const double mean = s / nf;
    double q = -0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double d = v[i] - mean;
        q += d * d;
    }
    const double var = q / nf;
    if (!std::isfinite(mean) || !std::isfinite(var)) return YM_ERR_NON_FINITE_STATISTIC;
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
    int64_t window = 0;
    bool open = true;
    for (int64_t lag = 1; lag <= max_lag; ++lag) {
        const int64_t pairs = n - lag;
        double c = -0.0;
        for (int64_t i = 0; i < pairs; ++i) c += (v[i] - mean) * (v[i + lag] - mean);
        c = c / (double)pairs;
        const double rho = c / var;
        if (!std::isfinite(rho)) return YM_ERR_NON_FINITE_STATISTIC;
        autocorrelation[lag] = rho;
        if (open && rho > 0.0) {
            tau += rho;
            window = lag;
        } else {
            open = false;
        }
    }
    if (!std::isfinite(tau) || tau < 0.5) return YM_ERR_NON_FINITE_STATISTIC;
    const double ess = std::fmin(nf / (2.0 * tau), nf);
    const double se = std::sqrt(var / ess);
    if (!std::isfinite(ess) || !std::isfinite(se)) return YM_ERR_NON_FINITE_STATISTIC;
    o->positive_window_lag = window;
    o->integrated_autocorrelation_time = tau;
    o->effective_sample_size = ess;
    o->standard_error = se;
    return YM_OK;
}

// sampling_efficiency.rs:57-135; log_weights may be NULL (unit weights).
int32_t ym_sampling_efficiency(const double *v, int64_t n, const double *log_weights,
                               int64_t max_lag, double setup, double thermalization,
                               double sampling, ym_efficiency_report *o,
                               double *autocorrelation) {
    if (!v || !o || !autocorrelation) return YM_ERR_NULL_ARGUMENT;
    if (n < 2 || n > 4096) return YM_ERR_INVALID_LENGTH;
    if (max_lag == 0 || max_lag >= n || max_lag > 256) return YM_ERR_INVALID_LAG;
    const double costs[3] = {setup, thermalization, sampling};
    for (double c : costs)
        if (!std::isfinite(c) || c < 0.0) return YM_ERR_INVALID_COST;
    if (sampling == 0.0) return YM_ERR_INVALID_COST;
    const double total = setup + thermalization + sampling;
    if (!std::isfinite(total)) return YM_ERR_INVALID_COST;
    double eff = 1.0;
    if (log_weights) {
        double mx = -INFINITY;
        for (int64_t i = 0; i < n; ++i) {
            if (!std::isfinite(log_weights[i])) return YM_ERR_INVALID_WEIGHT;
            mx = std::fmax(mx, log_weights[i]);
        }
        double sum = 0.0, sq = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            const double w = std::exp(log_weights[i] - mx);
            sum += w;
            sq += w * w;
        }
        eff = std::fmin((sum / (double)n) * (sum / sq), 1.0);
    }
    bool constant = true;
    for (int64_t i = 1; i < n; ++i)
        if (v[i] != v[0]) { constant = false; break; }
    if (constant) return YM_ERR_DEGENERATE_OBSERVABLE;
    if (ym_diagnostics(v, n, max_lag, &o->diagnostics, autocorrelation)) return YM_ERR_INVALID_DIAGNOSTIC;
    if (o->diagnostics.variance <= 0.0) return YM_ERR_DEGENERATE_OBSERVABLE;
    if (!std::isfinite(o->diagnostics.standard_error) || o->diagnostics.standard_error <= 0.0)
        return YM_ERR_NON_FINITE_RESULT;
    o->reweighting_efficiency = eff;
    o->weight_only_ess = (double)n * eff;
    o->combined_ess_proxy = o->diagnostics.effective_sample_size * eff;
    o->total_cost = total;
    o->sampling_cost_per_effective_sample_proxy = sampling / o->combined_ess_proxy;
    o->total_cost_per_effective_sample_proxy = total / o->combined_ess_proxy;
    const double chk[5] = {eff, o->weight_only_ess, o->combined_ess_proxy,
                           o->sampling_cost_per_effective_sample_proxy,
                           o->total_cost_per_effective_sample_proxy};
    for (double c : chk)
        if (!std::isfinite(c) || c <= 0.0) return YM_ERR_NON_FINITE_RESULT;
    return YM_OK;
}

}  // extern "C"

// ---- connected correlators, jackknife, covariance (host FP64) ----

extern "C" {

// glueball_correlators.rs:111-172
int32_t ym_periodic_connected_estimator(const double *samples, int64_t ncfg, int64_t nt,
                                        double *vacuum_mean, double *raw, double *connected) {
    if (!samples || !vacuum_mean || !raw || !connected) return YM_ERR_NULL_ARGUMENT;
    if (ncfg < 0 || nt < 0 || (nt > 0 && ncfg > INT64_MAX / nt)) return YM_ERR_SAMPLE_COUNT_OVERFLOW;
    const int64_t len = ncfg * nt;
    if (len == 0) return YM_ERR_CORRELATOR_SHAPE_MISMATCH;
    double ms = 0.0;
    for (int64_t i = 0; i < len; ++i) {
        if (!std::isfinite(samples[i])) return YM_ERR_NON_FINITE_OBSERVABLE;
        ms += samples[i];
        if (!std::isfinite(ms)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    }
    const double mean = ms / (double)len;
    if (!std::isfinite(mean)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    const double msq = mean * mean;
    if (!std::isfinite(msq)) return YM_ERR_NON_FINITE_ACCUMULATOR;
    for (int64_t tau = 0; tau < nt; ++tau) {
        double s = 0.0;
        for (int64_t c = 0; c < ncfg; ++c) {
            const double *row = samples + c * nt;
            for (int64_t t = 0; t < nt; ++t) {
                const double p = row[t] * row[(t + tau) % nt];
                if (!std::isfinite(p)) return YM_ERR_NON_FINITE_ACCUMULATOR;
                s += p;
                if (!std::isfinite(s)) return YM_ERR_NON_FINITE_ACCUMULATOR;
            }
        }
        const double r = s / (double)len;
        const double cv = r - msq;
        if (!std::isfinite(r) || !std::isfinite(cv)) return YM_ERR_NON_FINITE_ACCUMULATOR;
        raw[tau] = r;
        connected[tau] = cv;
    }
    *vacuum_mean = mean;
    return YM_OK;
}

// glueball_scalar_production.rs:383-443
int32_t ym_connected_from_samples(const double *samples, int64_t ncfg, int64_t nt, int64_t omitted,
                                  double *connected) {
    if (!samples || !connected) return YM_ERR_NULL_ARGUMENT;
    if (ncfg <= 0) return YM_ERR_EMPTY_CONFIGURATION_SET;
    if (nt <= 0) return YM_ERR_CONFIGURATION_SHAPE_MISMATCH;
    int64_t kept = ncfg;
    if (omitted >= 0) {
        if (omitted >= ncfg) return YM_ERR_CONFIGURATION_SHAPE_MISMATCH;
        kept = ncfg - 1;
    }
    if (kept == 0) return YM_ERR_EMPTY_CONFIGURATION_SET;
    const int64_t count = kept * nt;
    double ms = 0.0;
    for (int64_t c = 0; c < ncfg; ++c) {
        if (c == omitted) continue;
        for (int64_t t = 0; t < nt; ++t) {
            const double v = samples[c * nt + t];
            if (!std::isfinite(v)) return YM_ERR_NON_FINITE_STATISTIC;
            ms += v;
        }
    }
    const double mean = ms / (double)count;
    const double msq = mean * mean;
    if (!std::isfinite(mean) || !std::isfinite(msq)) return YM_ERR_NON_FINITE_STATISTIC;
    for (int64_t tau = 0; tau < nt; ++tau) {
        double s = 0.0;
        for (int64_t c = 0; c < ncfg; ++c) {
            if (c == omitted) continue;
            const double *row = samples + c * nt;
            for (int64_t t = 0; t < nt; ++t) s += row[t] * row[(t + tau) % nt];
        }
        const double v = s / (double)count - msq;
        if (!std::isfinite(v)) return YM_ERR_NON_FINITE_STATISTIC;
        connected[tau] = v;
    }
    return YM_OK;
}

// Every delete-one replica of ym_connected_from_samples.  Each replica's
// sums run in that function's order (configurations ascending, t ascending,
// the omitted one skipped) over the same rounded products, so every value is
// its bits; the products row[t] * row[(t + tau) % nt] are formed once for all
// replicas and the replicas are spread over the host's threads.  Inputs that
// the function would reject (a non-finite sample, fewer than two
// configurations) take the one-replica-at-a-time path, which returns the
// first failing replica's status exactly as before.
int32_t ym_jackknife_replicas(const double *samples, int64_t ncfg, int64_t nt, double *replicas) {
    if (!samples || !replicas) return YM_ERR_NULL_ARGUMENT;
    bool plain = ncfg < 2 || nt <= 0 || ncfg > (((int64_t)1 << 40) / std::max<int64_t>(nt, 1));
    for (int64_t i = 0; !plain && i < ncfg * nt; ++i)
        if (!std::isfinite(samples[i])) plain = true;
    if (plain) {
        for (int64_t k = 0; k < ncfg; ++k) {
            const int32_t st = ym_connected_from_samples(samples, ncfg, nt, k, replicas + k * nt);
            if (st) return st;
        }
        return ncfg > 0 ? YM_OK : YM_ERR_EMPTY_CONFIGURATION_SET;
    }
    // products[(c * nt + tau) * nt + t], kept while they fit in 256 MB
    std::vector<double> products;
    if (ncfg * nt * nt <= ((int64_t)1 << 25)) {
        products.resize((size_t)(ncfg * nt * nt));
        for (int64_t c = 0; c < ncfg; ++c) {
            const double *row = samples + c * nt;
            for (int64_t tau = 0; tau < nt; ++tau)
                for (int64_t t = 0; t < nt; ++t)
                    products[(size_t)((c * nt + tau) * nt + t)] = row[t] * row[(t + tau) % nt];
        }
    }
    std::vector<int32_t> status((size_t)ncfg, YM_OK);
    auto replica = [&](int64_t k) {
        const int64_t count = (ncfg - 1) * nt;
        double ms = 0.0;
        for (int64_t c = 0; c < ncfg; ++c) {
            if (c == k) continue;
            for (int64_t t = 0; t < nt; ++t) ms += samples[c * nt + t];
        }
        const double mean = ms / (double)count;
        const double msq = mean * mean;
        if (!std::isfinite(mean) || !std::isfinite(msq)) {
            status[(size_t)k] = YM_ERR_NON_FINITE_STATISTIC;
            return;
        }
        for (int64_t tau = 0; tau < nt; ++tau) {
            double s = 0.0;
            for (int64_t c = 0; c < ncfg; ++c) {
                if (c == k) continue;
                if (!products.empty()) {
                    const double *pr = products.data() + (c * nt + tau) * nt;
                    for (int64_t t = 0; t < nt; ++t) s += pr[t];
                } else {
                    const double *row = samples + c * nt;
                    for (int64_t t = 0; t < nt; ++t) s += row[t] * row[(t + tau) % nt];
                }
            }
            const double v = s / (double)count - msq;
            if (!std::isfinite(v)) {
                status[(size_t)k] = YM_ERR_NON_FINITE_STATISTIC;
                return;
            }
            replicas[k * nt + tau] = v;
        }
    };
    const int64_t hw = std::max<int64_t>(1, (int64_t)std::thread::hardware_concurrency());
    const int64_t n_threads = std::min<int64_t>(hw, std::max<int64_t>(1, ncfg / 8));
    if (n_threads <= 1) {
        for (int64_t k = 0; k < ncfg; ++k) replica(k);
    } else {
        std::vector<std::thread> pool;
        for (int64_t w = 0; w < n_threads; ++w)
            pool.emplace_back([&, w] {
                for (int64_t k = w; k < ncfg; k += n_threads) replica(k);
            });
        for (std::thread &th : pool) th.join();
    }
    for (int64_t k = 0; k < ncfg; ++k)
        if (status[(size_t)k] != YM_OK) return status[(size_t)k];
    return YM_OK;
}

// glueball_scalar_fit.rs:276-322
int32_t ym_jackknife_covariance(const double *replicas, int64_t nrep, int64_t nt, int64_t start,
                                int64_t end, double *out) {
    if (!replicas || !out) return YM_ERR_NULL_ARGUMENT;
    if (start < 0 || end < start) return YM_ERR_INVALID_CANDIDATE_WINDOW;
    const int64_t points = end - start + 1;
    if (nrep <= points) return YM_ERR_INSUFFICIENT_REPLICATES_FOR_COVARIANCE;
    if (end >= nt) return YM_ERR_INVALID_CANDIDATE_WINDOW;
    std::vector<double> means((size_t)points, 0.0);
    for (int64_t r = 0; r < nrep; ++r)
        for (int64_t c = 0; c < points; ++c) {
            const double v = replicas[r * nt + start + c];
            if (!std::isfinite(v)) return YM_ERR_NON_FINITE_STATISTIC;
            means[(size_t)c] += v;
        }
    const double n = (double)nrep;
    for (double &m : means) m /= n;
    for (int64_t i = 0; i < points * points; ++i) out[i] = 0.0;
    for (int64_t r = 0; r < nrep; ++r)
        for (int64_t a = 0; a < points; ++a) {
            const double left = replicas[r * nt + start + a] - means[(size_t)a];
            for (int64_t b = 0; b < points; ++b) {
                const double right = replicas[r * nt + start + b] - means[(size_t)b];
                out[a * points + b] += left * right;
            }
        }
    const double factor = (n - 1.0) / n;
    for (int64_t i = 0; i < points * points; ++i) {
        out[i] *= factor;
        if (!std::isfinite(out[i])) return YM_ERR_NON_FINITE_STATISTIC;
    }
    return YM_OK;
}

}  // extern "C"

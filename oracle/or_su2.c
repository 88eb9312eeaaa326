/* or_su2.c -- CPU oracle: SU(2) core and the SU(2) heat-bath ensemble,
 * restated from the reference crate.  TEST INFRASTRUCTURE ONLY (see
 * or_internal.h).
 *
 *   Su2 / Lattice4          reference/rust/src/lib.rs:106-782
 *   SU(2) ensemble          reference/rust/src/su2_ensemble.rs:24-552
 *
 * SU(2) links are unit quaternions (a0,a1,a2,a3), U = a0 I - i a.sigma,
 * stored 4 doubles per link at link = site*4+mu.
 */
#include <stdlib.h>

#include "oracle.h"
#include "or_internal.h"

#define MAX_SU2_LINKS ((int64_t)1 << 20)      /* lib.rs:21 */
#define SU2_MAX_BETA 8.0                       /* su2_ensemble.rs:18 */
#define SU2_MAX_SWEEPS ((int64_t)1 << 20)      /* su2_ensemble.rs:19 */
#define SU2_MAX_MEASUREMENTS ((int64_t)1 << 20)
#define SU2_MAX_OR 16                          /* su2_ensemble.rs:21 */
#define ALPHA_ZERO_LIMIT 1.0e-300              /* su2_ensemble.rs:22 */
#define TAU_2PI 6.283185307179586

typedef struct { double c[4]; } q4;

/* lib.rs:106-130: divide by the largest magnitude, then by the Euclidean norm. */
static int normalize_scaled(const double *v, int n, double *out) {
    double scale = 0.0;
    for (int i = 0; i < n; ++i) scale = rmax(scale, fabs(v[i]));
    if (scale == 0.0 || !isfinite(scale)) return 0;
    double s[4];
    for (int i = 0; i < n; ++i) s[i] = v[i] / scale;
    double ss = 0.0;
    for (int i = 0; i < n; ++i) ss += s[i] * s[i];
    double norm = sqrt(ss);
    if (norm == 0.0 || !isfinite(norm)) return 0;
    for (int i = 0; i < n; ++i) out[i] = s[i] / norm;
    return 1;
}

static int q_from_normalized(const double c[4], q4 *out) {   /* lib.rs:155-161 */
    for (int i = 0; i < 4; ++i) if (!isfinite(c[i])) return YM_ERR_NON_FINITE_SU2_COMPONENT;
    if (!normalize_scaled(c, 4, out->c)) return YM_ERR_ZERO_SU2_NORM;
    return YM_OK;
}

static q4 q_dagger(q4 a) { q4 o = {{a.c[0], -a.c[1], -a.c[2], -a.c[3]}}; return o; }

/* lib.rs:212-224.  A failed normalisation is a panic in the reference; it
 * cannot happen for finite unit inputs, so the raw product is kept then. */
static q4 q_mul(q4 a, q4 b) {
    double a0 = a.c[0], a1 = a.c[1], a2 = a.c[2], a3 = a.c[3];
    double b0 = b.c[0], b1 = b.c[1], b2 = b.c[2], b3 = b.c[3];
    double raw[4] = {
        a0 * b0 - a1 * b1 - a2 * b2 - a3 * b3,
        a0 * b1 + a1 * b0 + a2 * b3 - a3 * b2,
        a0 * b2 - a1 * b3 + a2 * b0 + a3 * b1,
        a0 * b3 + a1 * b2 - a2 * b1 + a3 * b0,
    };
    q4 o;
    if (!normalize_scaled(raw, 4, o.c)) memcpy(o.c, raw, sizeof raw);
    return o;
}

int or_su2_mul(const double *a, const double *b, double *out) {
    q4 x, y;
    memcpy(x.c, a, 32);
    memcpy(y.c, b, 32);
    q4 p = q_mul(x, y);
    memcpy(out, p.c, 32);
    return YM_OK;
}

int or_su2_from_axis_angle(const double *axis, double angle, double *out) {   /* lib.rs:179-189 */
    if (!isfinite(angle) || !isfinite(axis[0]) || !isfinite(axis[1]) || !isfinite(axis[2]))
        return YM_ERR_INVALID_AXIS;
    double n[3];
    if (!normalize_scaled(axis, 3, n)) return YM_ERR_INVALID_AXIS;
    double half = 0.5 * angle;
    double s = sin(half);
    out[0] = cos(half);
    out[1] = s * n[0];
    out[2] = s * n[1];
    out[3] = s * n[2];
    return YM_OK;
}

int or_su2_from_normalized(const double *c, double *out) {
    q4 q;
    int st = q_from_normalized(c, &q);
    if (st) return st;
    memcpy(out, q.c, 32);
    return YM_OK;
}

static q4 q_load(const double *links, int64_t l) { q4 q; memcpy(q.c, links + 4 * l, 32); return q; }
static void q_store(double *links, int64_t l, q4 q) { memcpy(links + 4 * l, q.c, 32); }
static q4 q_link(const extents4 *e, const double *links, const int64_t x[4], int mu) {
    return q_load(links, site_index(e, x) * 4 + mu);
}

int or_su2_identity(const int64_t *ext, double *links) {
    extents4 e; int64_t nl;
    int st = extents_from(ext, &e, MAX_SU2_LINKS, &nl);
    if (st) return st;
    q4 id = {{1.0, 0.0, 0.0, 0.0}};
    for (int64_t l = 0; l < nl; ++l) q_store(links, l, id);
    return YM_OK;
}

static q4 su2_plaquette(const extents4 *e, const double *links, const int64_t x[4], int mu, int nu) {
    int64_t xm[4], xn[4];                     /* lib.rs:348-361 */
    nb_plus(e, x, mu, xm);
    nb_plus(e, x, nu, xn);
    q4 p = q_mul(q_link(e, links, x, mu), q_link(e, links, xm, nu));
    p = q_mul(p, q_dagger(q_link(e, links, xn, mu)));
    return q_mul(p, q_dagger(q_link(e, links, x, nu)));
}

int or_su2_plaquette(const int64_t *ext, const double *links, const int64_t *x, int mu, int nu,
                     double *out4) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    if (mu < 0 || mu >= 4 || nu < 0 || nu >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    if (mu == nu) return YM_ERR_DIRECTIONS_MUST_DIFFER;
    if (!coord_ok(&e, x)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    q4 p = su2_plaquette(&e, links, x, mu, nu);
    memcpy(out4, p.c, 32);
    return YM_OK;
}

int or_su2_wilson_action(const int64_t *ext, const double *links, double beta, double *out) {
    extents4 e;                               /* lib.rs:363-382 */
    int64_t x[4];
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    if (!isfinite(beta)) return YM_ERR_NON_FINITE_BETA;
    if (beta < 0.0) return YM_ERR_NEGATIVE_BETA;
    double sum = 0.0;
    for (x[0] = 0; x[0] < e.n[0]; ++x[0])
        for (x[1] = 0; x[1] < e.n[1]; ++x[1])
            for (x[2] = 0; x[2] < e.n[2]; ++x[2])
                for (x[3] = 0; x[3] < e.n[3]; ++x[3])
                    for (int mu = 0; mu < 4; ++mu)
                        for (int nu = mu + 1; nu < 4; ++nu)
                            sum += 1.0 - su2_plaquette(&e, links, x, mu, nu).c[0];
    if (!isfinite(sum)) return YM_ERR_NON_FINITE_ACTION;
    double a = beta * sum;
    if (!isfinite(a)) return YM_ERR_NON_FINITE_ACTION;
    *out = a;
    return YM_OK;
}

/* lib.rs:384-436: steps[i] = +(mu+1) forward, -(mu+1) backward; returns the
 * half real trace of a closed path. */
int or_su2_wilson_loop(const int64_t *ext, const double *links, const int64_t *start,
                       const int32_t *steps, int64_t nsteps, double *out) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    if (!coord_ok(&e, start)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    if (nsteps <= 0) return YM_ERR_EMPTY_PATH;
    if (nsteps > ((int64_t)1 << 20)) return YM_ERR_PATH_TOO_LONG;
    int64_t x[4];
    memcpy(x, start, sizeof x);
    q4 h = {{1.0, 0.0, 0.0, 0.0}};
    for (int64_t i = 0; i < nsteps; ++i) {
        int d = steps[i] > 0 ? steps[i] - 1 : -steps[i] - 1;
        if (steps[i] == 0 || d >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
        int64_t y[4];
        q4 seg;
        if (steps[i] > 0) {
            seg = q_link(&e, links, x, d);
            nb_plus(&e, x, d, y);
        } else {
            nb_minus(&e, x, d, y);
            seg = q_dagger(q_link(&e, links, y, d));
        }
        memcpy(x, y, sizeof x);
        h = q_mul(h, seg);
    }
    for (int i = 0; i < 4; ++i) if (x[i] != start[i]) return YM_ERR_PATH_NOT_CLOSED;
    *out = h.c[0];
    return YM_OK;
}

int or_su2_polyakov_loop(const int64_t *ext, const double *links, const int64_t *start, int dir,
                         double *out) {                      /* lib.rs:483-505 */
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    if (dir < 0 || dir >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    if (!coord_ok(&e, start)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    int64_t x[4];
    memcpy(x, start, sizeof x);
    q4 h = {{1.0, 0.0, 0.0, 0.0}};
    for (int64_t k = 0; k < e.n[dir]; ++k) {
        h = q_mul(h, q_link(&e, links, x, dir));
        int64_t y[4];
        nb_plus(&e, x, dir, y);
        memcpy(x, y, sizeof x);
    }
    *out = h.c[0];
    return YM_OK;
}

/* lib.rs:507-546: unnormalised sum of the six staple products. */
static void su2_staple(const extents4 *e, const double *links, const int64_t x[4], int mu,
                       double comp[4]) {
    comp[0] = comp[1] = comp[2] = comp[3] = 0.0;
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        int64_t xpm[4], xpn[4], xmn[4], xmnpm[4];
        nb_plus(e, x, mu, xpm);
        nb_plus(e, x, nu, xpn);
        q4 fwd = q_mul(q_mul(q_link(e, links, xpm, nu), q_dagger(q_link(e, links, xpn, mu))),
                       q_dagger(q_link(e, links, x, nu)));
        nb_minus(e, x, nu, xmn);
        nb_plus(e, xmn, mu, xmnpm);
        q4 bwd = q_mul(q_mul(q_dagger(q_link(e, links, xmnpm, nu)),
                             q_dagger(q_link(e, links, xmn, mu))),
                       q_link(e, links, xmn, nu));
        for (int i = 0; i < 4; ++i) comp[i] += fwd.c[i];
        for (int i = 0; i < 4; ++i) comp[i] += bwd.c[i];
    }
}

int or_su2_staple(const int64_t *ext, const double *links, const int64_t *x, int mu, double *out4) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    if (mu < 0 || mu >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    if (!coord_ok(&e, x)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    su2_staple(&e, links, x, mu, out4);
    return YM_OK;
}

int or_su2_max_unit_residual(const int64_t *ext, const double *links, double *out) {
    extents4 e; int64_t nl;                   /* lib.rs:726-740 */
    int st = extents_from(ext, &e, 0, &nl);
    if (st) return st;
    double m = 0.0;
    for (int64_t l = 0; l < nl; ++l) {
        const double *c = links + 4 * l;
        double n2 = 0.0;
        for (int i = 0; i < 4; ++i) n2 += c[i] * c[i];
        if (!isfinite(n2)) { *out = INFINITY; return YM_OK; }
        double r = fabs(n2 - 1.0);
        if (!isfinite(r)) { *out = INFINITY; return YM_OK; }
        m = rmax(m, r);
    }
    *out = m;
    return YM_OK;
}

/* ---------------------------------------------------------------- ensemble */

uint64_t or_derive_chain_seed(uint64_t master, uint64_t chain) {   /* su2_ensemble.rs:52-55 */
    return or_mix64(master ^ ((chain + 1) * 0x9E3779B97F4A7C15ULL));
}

uint64_t or_splitmix_next(uint64_t *state) { return sm_next(state); }
double or_splitmix_unit(uint64_t *state) { return sm_unit(state); }

/* su2_ensemble.rs:204-209 */
static void sphere_direction(uint64_t *rng, double d[3]) {
    double z = 2.0 * sm_unit(rng) - 1.0;
    double phi = TAU_2PI * sm_unit(rng);
    double planar = sqrt(rmax(1.0 - z * z, 0.0));
    d[0] = planar * cos(phi);
    d[1] = planar * sin(phi);
    d[2] = z;
}

/* su2_ensemble.rs:220-254: truncated-exponential proposal for r0, Haar
 * Jacobian by rejection, uniform direction on S^2. */
int or_su2_sample_heatbath(double alpha, uint64_t *rng, int64_t max_attempts, double *out4,
                           uint64_t *attempts) {
    if (!isfinite(alpha) || alpha < 0.0) return YM_ERR_NON_FINITE_STATISTIC;
    for (int64_t a = 1; a <= max_attempts; ++a) {
        double pu = sm_unit(rng);
        double r0;
        if (alpha <= ALPHA_ZERO_LIMIT) {
            r0 = 2.0 * pu - 1.0;
        } else {
            double mass = -expm1(-2.0 * alpha);
            double y = -log1p(-pu * mass) / alpha;
            r0 = 1.0 - y;
            if (r0 < -1.0) r0 = -1.0;
            if (r0 > 1.0) r0 = 1.0;
        }
        double radial = sqrt(rmax(1.0 - r0 * r0, 0.0));
        if (sm_unit(rng) <= radial) {
            double d[3];
            sphere_direction(rng, d);
            double c[4] = {r0, radial * d[0], radial * d[1], radial * d[2]};
            q4 s;
            int st = q_from_normalized(c, &s);
            if (st) return st;
            memcpy(out4, s.c, 32);
            *attempts = (uint64_t)a;
            return YM_OK;
        }
    }
    return YM_ERR_HEATBATH_ATTEMPT_LIMIT_EXCEEDED;
}

static int staple_norm(const double c[4], double *norm) {
    double s = 0.0;
    for (int i = 0; i < 4; ++i) s += c[i] * c[i];
    *norm = sqrt(s);
    return isfinite(*norm) ? YM_OK : YM_ERR_NON_FINITE_STATISTIC;
}

/* su2_ensemble.rs:256-281 */
static int heatbath_link(const extents4 *e, double *links, const int64_t x[4], int mu, double beta,
                         uint64_t *rng, int64_t max_attempts, uint64_t *attempts) {
    double comp[4], norm;
    su2_staple(e, links, x, mu, comp);
    int st = staple_norm(comp, &norm);
    if (st) return st;
    double alpha = beta * norm;
    if (!isfinite(alpha)) return YM_ERR_NON_FINITE_STATISTIC;
    q4 r;
    st = or_su2_sample_heatbath(alpha, rng, max_attempts, r.c, attempts);
    if (st) return st;
    q4 next = r;
    if (norm != 0.0) {
        q4 ns;
        st = q_from_normalized(comp, &ns);
        if (st) return st;
        next = q_mul(r, q_dagger(ns));
    }
    q_store(links, site_index(e, x) * 4 + mu, next);
    return YM_OK;
}

/* su2_ensemble.rs:283-299 */
static int overrelax_link(const extents4 *e, double *links, const int64_t x[4], int mu) {
    double comp[4], norm;
    su2_staple(e, links, x, mu, comp);
    int st = staple_norm(comp, &norm);
    if (st) return st;
    if (norm == 0.0) return YM_OK;
    q4 ns;
    st = q_from_normalized(comp, &ns);
    if (st) return st;
    int64_t l = site_index(e, x) * 4 + mu;
    q4 nd = q_dagger(ns);
    q_store(links, l, q_mul(q_mul(nd, q_dagger(q_load(links, l))), nd));
    return YM_OK;
}

/* su2_ensemble.rs:321-342 */
int or_su2_heatbath_sweep(const int64_t *ext, double *links, double beta, uint64_t *rng,
                          int64_t max_attempts, uint64_t *proposals, uint64_t *updates) {
    extents4 e;
    int64_t x[4];
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    if (!isfinite(beta) || beta < 0.0 || beta > SU2_MAX_BETA)
        return YM_ERR_BETA_OUTSIDE_REFERENCE_RANGE;
    if (max_attempts == 0) return YM_ERR_ZERO_HEATBATH_ATTEMPT_LIMIT;
    uint64_t np = 0, nu = 0;
    for (x[0] = 0; x[0] < e.n[0]; ++x[0])
        for (x[1] = 0; x[1] < e.n[1]; ++x[1])
            for (x[2] = 0; x[2] < e.n[2]; ++x[2])
                for (x[3] = 0; x[3] < e.n[3]; ++x[3])
                    for (int mu = 0; mu < 4; ++mu) {
                        uint64_t att;
                        st = heatbath_link(&e, links, x, mu, beta, rng, max_attempts, &att);
                        if (st) return st;
                        np += att;
                        nu += 1;
                    }
    *proposals = np;
    *updates = nu;
    return YM_OK;
}

int or_su2_overrelaxation_sweep(const int64_t *ext, double *links) {   /* :344-346 */
    extents4 e;
    int64_t x[4];
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    for (x[0] = 0; x[0] < e.n[0]; ++x[0])
        for (x[1] = 0; x[1] < e.n[1]; ++x[1])
            for (x[2] = 0; x[2] < e.n[2]; ++x[2])
                for (x[3] = 0; x[3] < e.n[3]; ++x[3])
                    for (int mu = 0; mu < 4; ++mu) {
                        st = overrelax_link(&e, links, x, mu);
                        if (st) return st;
                    }
    return YM_OK;
}

int or_su2_average_plaquette(const int64_t *ext, const double *links, double *out) {
    extents4 e;                               /* su2_ensemble.rs:348-373 */
    int64_t x[4];
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    double sum = 0.0;
    int64_t count = 0;
    for (x[0] = 0; x[0] < e.n[0]; ++x[0])
        for (x[1] = 0; x[1] < e.n[1]; ++x[1])
            for (x[2] = 0; x[2] < e.n[2]; ++x[2])
                for (x[3] = 0; x[3] < e.n[3]; ++x[3])
                    for (int mu = 0; mu < 4; ++mu)
                        for (int nu = mu + 1; nu < 4; ++nu) {
                            sum += su2_plaquette(&e, links, x, mu, nu).c[0];
                            count += 1;
                        }
    double v = sum / (double)count;
    if (!isfinite(v)) return YM_ERR_NON_FINITE_STATISTIC;
    *out = v;
    return YM_OK;
}

/* su2_ensemble.rs:488-552 (diagnostics left to the caller, as for SU(3)). */
int or_su2_run_chain(const or_su2_config *cfg, double *links_out, double *measurements,
                     or_su2_chain_scalars *out) {
    if (!isfinite(cfg->beta) || cfg->beta < 0.0 || cfg->beta > SU2_MAX_BETA)
        return YM_ERR_BETA_OUTSIDE_REFERENCE_RANGE;
    if (cfg->measurements > SU2_MAX_MEASUREMENTS) return YM_ERR_SCHEDULE_OUTSIDE_REFERENCE_RANGE;
    int64_t total = cfg->thermalization_sweeps +
                    cfg->measurements * cfg->sweeps_between_measurements;
    if (total > SU2_MAX_SWEEPS || total < 0) return YM_ERR_SCHEDULE_OUTSIDE_REFERENCE_RANGE;
    if (cfg->measurements < 2) return YM_ERR_TOO_FEW_MEASUREMENTS;
    if (cfg->sweeps_between_measurements == 0) return YM_ERR_ZERO_MEASUREMENT_STRIDE;
    if (cfg->overrelaxation_sweeps_per_heatbath > SU2_MAX_OR)
        return YM_ERR_TOO_MANY_OVERRELAXATION_SWEEPS;
    if (cfg->max_heatbath_attempts_per_link == 0) return YM_ERR_ZERO_HEATBATH_ATTEMPT_LIMIT;
    if (cfg->autocorrelation_max_lag >= cfg->measurements)
        return YM_ERR_AUTOCORRELATION_LAG_OUT_OF_RANGE;
    int st = or_su2_identity(cfg->extents, links_out);
    if (st) return st;
    uint64_t seed = or_derive_chain_seed(cfg->master_seed, cfg->chain_id);
    uint64_t rng = seed, hp = 0, hu = 0, p, u;
    int64_t ors = 0;
    int64_t nsweeps = cfg->thermalization_sweeps;
    for (int64_t m = -1; m < cfg->measurements; ++m) {
        for (int64_t s = 0; s < nsweeps; ++s) {
            st = or_su2_heatbath_sweep(cfg->extents, links_out, cfg->beta, &rng,
                                       cfg->max_heatbath_attempts_per_link, &p, &u);
            if (st) return st;
            hp += p;
            hu += u;
            for (int64_t k = 0; k < cfg->overrelaxation_sweeps_per_heatbath; ++k) {
                st = or_su2_overrelaxation_sweep(cfg->extents, links_out);
                if (st) return st;
                ors += 1;
            }
        }
        if (m >= 0) {
            st = or_su2_average_plaquette(cfg->extents, links_out, &measurements[m]);
            if (st) return st;
        }
        nsweeps = cfg->sweeps_between_measurements;
    }
    out->derived_seed = seed;
    out->total_heatbath_sweeps = total;
    out->total_overrelaxation_sweeps = ors;
    out->heatbath_proposals = hp;
    out->heatbath_updates = hu;
    out->mean_heatbath_acceptance = (double)hu / (double)hp;
    or_su2_max_unit_residual(cfg->extents, links_out, &out->final_link_unit_residual);
    if (!isfinite(out->mean_heatbath_acceptance) || !isfinite(out->final_link_unit_residual))
        return YM_ERR_NON_FINITE_STATISTIC;
    return YM_OK;
}

/* ------------------------------------------------------ engine order */

/* The engine's SU(2) sweep restated on the CPU (see or_b200.c for the
 * rationale): checkerboard order, one counter-based SplitMix64 stream per
 * link visit keyed S(S(seed, sweep), 4*site+mu), S(k, n) = mix64(k+(n+1)g),
 * with the reference sampler drawing stream words 0, 1, 2, ... in the order
 * sample_local_heatbath consumes them (su2_ensemble.rs:220-254). */
static inline uint64_t sm_at(uint64_t seed, uint64_t n) {
    return or_mix64(seed + (n + 1) * 0x9E3779B97F4A7C15ULL);
}
static inline double unit_of(uint64_t w) { return (double)(w >> 11) * (1.0 / 9007199254740992.0); }

static int sample_from_stream(double alpha, uint64_t key, int64_t max_attempts, q4 *out,
                              uint64_t *attempts) {
    uint64_t j = 0;
    double mass = alpha <= ALPHA_ZERO_LIMIT ? 0.0 : -expm1(-2.0 * alpha);
    for (int64_t a = 1; a <= max_attempts; ++a) {
        double pu = unit_of(sm_at(key, j++));
        double r0;
        if (alpha <= ALPHA_ZERO_LIMIT) {
            r0 = 2.0 * pu - 1.0;
        } else {
            double y = -log1p(-pu * mass) / alpha;
            r0 = 1.0 - y;
            if (r0 < -1.0) r0 = -1.0;
            if (r0 > 1.0) r0 = 1.0;
        }
        double radial = sqrt(rmax(1.0 - r0 * r0, 0.0));
        if (unit_of(sm_at(key, j++)) <= radial) {
            double z = 2.0 * unit_of(sm_at(key, j++)) - 1.0;
            double phi = TAU_2PI * unit_of(sm_at(key, j++));
            double planar = sqrt(rmax(1.0 - z * z, 0.0));
            double c[4] = {r0, radial * (planar * cos(phi)), radial * (planar * sin(phi)), radial * z};
            int st = q_from_normalized(c, out);
            if (st) return st;
            *attempts = (uint64_t)a;
            return YM_OK;
        }
    }
    *attempts = (uint64_t)max_attempts;
    return YM_ERR_HEATBATH_ATTEMPT_LIMIT_EXCEEDED;
}

int or_su2_cb_sweep(const int64_t *ext, double *links, double beta, uint64_t chain_seed,
                    uint64_t sweep, int64_t overrelaxation_sweeps, int64_t max_attempts,
                    uint64_t *proposals) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    for (int i = 0; i < 4; ++i) if (e.n[i] % 2) return YM_ERR_NOT_CHECKERBOARDABLE;
    uint64_t np = 0;
    int failed = 0;
    for (int p = 0; p < 2; ++p)
        for (int mu = 0; mu < 4; ++mu) {
            int64_t x[4];
            for (x[0] = 0; x[0] < e.n[0]; ++x[0])
                for (x[1] = 0; x[1] < e.n[1]; ++x[1])
                    for (x[2] = 0; x[2] < e.n[2]; ++x[2])
                        for (x[3] = 0; x[3] < e.n[3]; ++x[3]) {
                            if (((x[0] + x[1] + x[2] + x[3]) & 1) != p) continue;
                            int64_t lex = site_index(&e, x);
                            double comp[4], norm;
                            su2_staple(&e, links, x, mu, comp);
                            st = staple_norm(comp, &norm);
                            if (st) return st;
                            q4 r;
                            uint64_t att = 0;
                            uint64_t key = sm_at(sm_at(chain_seed, sweep), (uint64_t)(4 * lex + mu));
                            st = sample_from_stream(beta * norm, key, max_attempts, &r, &att);
                            np += att;
                            if (st == YM_ERR_HEATBATH_ATTEMPT_LIMIT_EXCEEDED) { failed = 1; continue; }
                            if (st) return st;
                            q4 next = r;
                            if (norm != 0.0) {
                                q4 ns;
                                q_from_normalized(comp, &ns);
                                next = q_mul(r, q_dagger(ns));
                            }
                            q_store(links, lex * 4 + mu, next);
                        }
        }
    for (int64_t k = 0; k < overrelaxation_sweeps; ++k)
        for (int p = 0; p < 2; ++p)
            for (int mu = 0; mu < 4; ++mu) {
                int64_t x[4];
                for (x[0] = 0; x[0] < e.n[0]; ++x[0])
                    for (x[1] = 0; x[1] < e.n[1]; ++x[1])
                        for (x[2] = 0; x[2] < e.n[2]; ++x[2])
                            for (x[3] = 0; x[3] < e.n[3]; ++x[3]) {
                                if (((x[0] + x[1] + x[2] + x[3]) & 1) != p) continue;
                                st = overrelax_link(&e, links, x, mu);
                                if (st) return st;
                            }
            }
    *proposals = np;
    return failed ? YM_ERR_HEATBATH_ATTEMPT_LIMIT_EXCEEDED : YM_OK;
}

/* Overrelaxation only, engine (checkerboard) order. */
int or_su2_cb_overrelax(const int64_t *ext, double *links) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    for (int i = 0; i < 4; ++i) if (e.n[i] % 2) return YM_ERR_NOT_CHECKERBOARDABLE;
    for (int p = 0; p < 2; ++p)
        for (int mu = 0; mu < 4; ++mu) {
            int64_t x[4];
            for (x[0] = 0; x[0] < e.n[0]; ++x[0])
                for (x[1] = 0; x[1] < e.n[1]; ++x[1])
                    for (x[2] = 0; x[2] < e.n[2]; ++x[2])
                        for (x[3] = 0; x[3] < e.n[3]; ++x[3]) {
                            if (((x[0] + x[1] + x[2] + x[3]) & 1) != p) continue;
                            st = overrelax_link(&e, links, x, mu);
                            if (st) return st;
                        }
        }
    return YM_OK;
}

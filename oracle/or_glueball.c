/* or_glueball.c -- CPU oracle: scalar (A1++) glueball operator basis,
 * spatial stout smearing, stride-2 spatial blocking and the configuration
 * correlator entry point, restated from the reference crate.  TEST
 * INFRASTRUCTURE ONLY (see or_internal.h).
 *
 *   operator basis     reference/rust/src/glueball_operators.rs:72-160
 *   stout smearing     reference/rust/src/glueball_smearing.rs:83-301
 *   stride-2 blocking  reference/rust/src/glueball_blocking.rs:71-175
 *   correlators        reference/rust/src/glueball_correlators.rs:179-235
 */
#include <stdlib.h>

#include "oracle.h"
#include "or_internal.h"

#define TIME_DIR 3
#define MIN_SPATIAL 3
#define STOUT_MAX_RHO 0.25
#define STOUT_MAX_LEVELS 8
#define ALGEBRA_RESIDUAL_TOL 2.0e-12
#define SU3_TOL 5.0e-12

static const int PLAQ_OR[3][2] = {{0, 1}, {0, 2}, {1, 2}};
static const int RECT_OR[6][2] = {{0, 1}, {0, 2}, {1, 0}, {1, 2}, {2, 0}, {2, 1}};

/* glueball_operators.rs:93-139: mean of Re W over orientations x spatial
 * starts, orientation outermost, then x0, x1, x2. */
static int average_orbit(const int64_t *ext, const double *links, int64_t t, const int (*ori)[2],
                         int nori, int64_t r, int64_t tt, double *mean, int64_t *count) {
    double sum = 0.0;
    int64_t cnt = 0;
    int32_t steps[64];
    for (int o = 0; o < nori; ++o) {
        int64_t ns;
        int st = or_rectangular_path(ori[o][0], ori[o][1], r, tt, steps, 64, &ns);
        if (st) return st;
        int64_t x[4];
        x[3] = t;
        for (x[0] = 0; x[0] < ext[0]; ++x[0])
            for (x[1] = 0; x[1] < ext[1]; ++x[1])
                for (x[2] = 0; x[2] < ext[2]; ++x[2]) {
                    double re, im;
                    st = or_su3_wilson_loop(ext, links, x, steps, ns, &re, &im);
                    if (st) return st;
                    if (!isfinite(re)) return YM_ERR_NON_FINITE_OBSERVABLE;
                    sum += re;
                    if (!isfinite(sum)) return YM_ERR_NON_FINITE_OBSERVABLE;
                    cnt += 1;
                }
    }
    if (cnt == 0) return YM_ERR_COUNT_OVERFLOW;
    double m = sum / (double)cnt;
    if (!isfinite(m)) return YM_ERR_NON_FINITE_OBSERVABLE;
    *mean = m;
    *count = cnt;
    return YM_OK;
}

static int operator_geometry(const int64_t *ext, int64_t t) {   /* :72-91 */
    if (t < 0 || t >= ext[TIME_DIR]) return YM_ERR_TIME_SLICE_OUT_OF_RANGE;
    for (int d = 0; d < 3; ++d) if (ext[d] < MIN_SPATIAL) return YM_ERR_SPATIAL_EXTENT_TOO_SMALL;
    if (ext[0] != ext[1] || ext[1] != ext[2]) return YM_ERR_SPATIAL_EXTENTS_NOT_CUBIC;
    return YM_OK;
}

int or_scalar_a1pp_operator_basis(const int64_t *ext, const double *links, int64_t t,
                                  double *plaq, double *rect, int64_t *plaq_count,
                                  int64_t *rect_count) {
    int st = operator_geometry(ext, t);
    if (st) return st;
    st = average_orbit(ext, links, t, PLAQ_OR, 3, 1, 1, plaq, plaq_count);
    if (st) return st;
    return average_orbit(ext, links, t, RECT_OR, 6, 2, 1, rect, rect_count);
}

/* ----------------------------------------------------------------- stout */

static int stout_parameters(const int64_t *ext, double rho, int64_t levels) {   /* :83-108 */
    if (!isfinite(rho)) return YM_ERR_NON_FINITE_RHO;
    if (rho <= 0.0 || rho > STOUT_MAX_RHO) return YM_ERR_RHO_OUT_OF_RANGE;
    if (levels > STOUT_MAX_LEVELS || levels < 0) return YM_ERR_TOO_MANY_LEVELS;
    for (int d = 0; d < 3; ++d) if (ext[d] < MIN_SPATIAL) return YM_ERR_SPATIAL_EXTENT_TOO_SMALL;
    if (ext[0] != ext[1] || ext[1] != ext[2]) return YM_ERR_SPATIAL_EXTENTS_NOT_CUBIC;
    return YM_OK;
}

/* glueball_smearing.rs:137-172: rho * sum over spatial nu != mu of
 * U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag + U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu). */
static int spatial_staple_sum(const extents4 *e, const double *links, const int64_t x[4], int mu,
                              double rho, mat3 *out) {
    mat3 sum = m3_zero();
    int st;
    for (int nu = 0; nu < 3; ++nu) {
        if (nu == mu) continue;
        int64_t xpm[4], xpn[4], xmn[4], xmnpm[4];
        nb_plus(e, x, mu, xpm);
        nb_plus(e, x, nu, xpn);
        mat3 f;
        st = su3_mul_checked(su3_link(e, links, x, nu), su3_link(e, links, xpn, mu), &f);
        if (!st) st = su3_mul_checked(f, m3_dagger(su3_link(e, links, xpm, nu)), &f);
        if (st) return st;
        sum = m3_add(sum, f);
        nb_minus(e, x, nu, xmn);
        nb_plus(e, xmn, mu, xmnpm);
        mat3 b;
        st = su3_mul_checked(m3_dagger(su3_link(e, links, xmn, nu)), su3_link(e, links, xmn, mu), &b);
        if (!st) st = su3_mul_checked(b, su3_link(e, links, xmnpm, nu), &b);
        if (st) return st;
        sum = m3_add(sum, b);
    }
    mat3 w = m3_scale_real(sum, rho);
    if (!m3_finite(w)) return YM_ERR_NON_FINITE_STAPLE;
    *out = w;
    return YM_OK;
}

/* glueball_smearing.rs:174-193 */
static int stout_q(mat3 staple, mat3 link, mat3 *q) {
    mat3 omega = m3_mul(staple, m3_dagger(link));
    if (!m3_finite(omega)) return YM_ERR_NON_FINITE_STAPLE;
    mat3 anti = m3_sub(m3_dagger(omega), omega);
    mat3 first = m3_scale_complex(anti, c_make(0.0, 0.5));
    c64 tc = c_scale(c_mul(m3_trace(anti), c_make(0.0, 1.0)), 1.0 / 6.0);
    mat3 r = m3_sub(first, m3_scale_complex(m3_identity(), tc));
    if (!m3_finite(r)) return YM_ERR_NON_FINITE_STAPLE;
    if (m3_hermiticity_residual(r) > ALGEBRA_RESIDUAL_TOL || c_abs(m3_trace(r)) > ALGEBRA_RESIDUAL_TOL)
        return YM_ERR_ALGEBRA_PROJECTION_RESIDUAL;
    *q = r;
    return YM_OK;
}

/* glueball_smearing.rs:195-205 */
static int q_coefficients(mat3 q, double coef[8]) {
    for (int i = 0; i < 8; ++i) {
        mat3 g;
        su3_gell_mann(i, &g);
        c64 p = m3_trace(m3_mul(q, g));
        if (!c_finite(p) || fabs(p.im) > ALGEBRA_RESIDUAL_TOL) return YM_ERR_ALGEBRA_PROJECTION_RESIDUAL;
        coef[i] = p.re;
    }
    return YM_OK;
}

/* glueball_smearing.rs:225-251: one synchronous level from `in` into `out`
 * (out starts as a copy; temporal links untouched). */
static int smear_one_level(const extents4 *e, const double *in, double *out, double rho,
                           int64_t nlinks) {
    memcpy(out, in, (size_t)nlinks * 18 * sizeof(double));
    int64_t x[4];
    for (x[0] = 0; x[0] < e->n[0]; ++x[0])
        for (x[1] = 0; x[1] < e->n[1]; ++x[1])
            for (x[2] = 0; x[2] < e->n[2]; ++x[2])
                for (x[3] = 0; x[3] < e->n[3]; ++x[3])
                    for (int mu = 0; mu < 3; ++mu) {
                        mat3 old = su3_link(e, in, x, mu), staple, q, rot, upd;
                        double coef[8];
                        int st = spatial_staple_sum(e, in, x, mu, rho, &staple);
                        if (!st) st = stout_q(staple, old, &q);
                        if (!st) st = q_coefficients(q, coef);
                        if (!st) st = su3_from_algebra(coef, &rot);
                        if (!st) st = su3_mul_checked(rot, old, &upd);
                        if (st) return st;
                        if (m3_unitarity_residual(upd) > SU3_TOL ||
                            m3_determinant_residual(upd) > SU3_TOL)
                            return YM_ERR_NON_UNITARY_MATRIX;
                        su3_store(out, site_index(e, x) * 4 + mu, upd);
                    }
    return YM_OK;
}

/* glueball_smearing.rs:257-268.  `lift_level_cap` admits more than 8
 * levels; the reference composes such runs from capped calls, and because
 * levels are sequential the result is identical. */
int or_spatial_stout_smear(const int64_t *ext, const double *links, double rho, int64_t levels,
                           int lift_level_cap, double *out) {
    int st = stout_parameters(ext, rho, lift_level_cap ? (levels < 0 ? -1 : 0) : levels);
    if (st) return st;
    extents4 e; int64_t nl;
    st = extents_from(ext, &e, 0, &nl);
    if (st) return st;
    memcpy(out, links, (size_t)nl * 18 * sizeof(double));
    if (levels == 0) return YM_OK;
    double *tmp = malloc((size_t)nl * 18 * sizeof(double));
    if (!tmp) return YM_ERR_ALLOCATION_FAILED;
    for (int64_t l = 0; l < levels; ++l) {
        memcpy(tmp, out, (size_t)nl * 18 * sizeof(double));
        st = smear_one_level(&e, tmp, out, rho, nl);
        if (st) break;
    }
    free(tmp);
    return st;
}

/* glueball_smearing.rs:270-301 and glueball_blocking.rs:138-169 */
int or_max_link_residual(const int64_t *ext, const double *a, const double *b, double *out) {
    extents4 e; int64_t nl;
    int st = extents_from(ext, &e, 0, &nl);
    if (st) return st;
    double m = 0.0;
    for (int64_t l = 0; l < nl; ++l) {
        double r = m3_max_residual(su3_load(a, l), su3_load(b, l));
        if (!isfinite(r)) return YM_ERR_NON_FINITE_STAPLE;
        m = rmax(m, r);
    }
    *out = m;
    return YM_OK;
}

/* --------------------------------------------------------------- blocking */

int or_blocked_extents(const int64_t *ext, int64_t *out) {     /* glueball_blocking.rs:71-94 */
    if (ext[0] != ext[1] || ext[1] != ext[2]) return YM_ERR_SPATIAL_EXTENTS_NOT_CUBIC;
    if (ext[0] < 2 * MIN_SPATIAL) return YM_ERR_SPATIAL_EXTENT_TOO_SMALL;
    if (ext[0] % 2 != 0) return YM_ERR_SPATIAL_EXTENT_NOT_EVEN;
    out[0] = ext[0] / 2;
    out[1] = ext[1] / 2;
    out[2] = ext[2] / 2;
    out[3] = ext[3];
    return YM_OK;
}

/* glueball_blocking.rs:105-136 */
int or_spatial_stride2_block(const int64_t *ext, const double *links, double *coarse) {
    int64_t cext[4];
    int st = or_blocked_extents(ext, cext);
    if (st) return st;
    extents4 e, c;
    st = extents_from(ext, &e, 0, NULL);
    if (!st) st = extents_from(cext, &c, 0, NULL);
    if (st) return st;
    int64_t y[4];
    for (y[0] = 0; y[0] < c.n[0]; ++y[0])
        for (y[1] = 0; y[1] < c.n[1]; ++y[1])
            for (y[2] = 0; y[2] < c.n[2]; ++y[2])
                for (y[3] = 0; y[3] < c.n[3]; ++y[3]) {
                    int64_t x[4] = {2 * y[0], 2 * y[1], 2 * y[2], y[3]};
                    int64_t cs = site_index(&c, y);
                    for (int mu = 0; mu < 3; ++mu) {
                        int64_t xp[4];
                        nb_plus(&e, x, mu, xp);
                        mat3 b;
                        st = su3_mul_checked(su3_link(&e, links, x, mu), su3_link(&e, links, xp, mu), &b);
                        if (st) return st;
                        if (m3_unitarity_residual(b) > SU3_TOL || m3_determinant_residual(b) > SU3_TOL)
                            return YM_ERR_NON_UNITARY_MATRIX;
                        su3_store(coarse, cs * 4 + mu, b);
                    }
                    su3_store(coarse, cs * 4 + 3, su3_link(&e, links, x, 3));
                }
    return YM_OK;
}

/* ------------------------------------------------------------ correlators */

/* glueball_correlators.rs:179-235.  `configs` holds ncfg lattices of equal
 * extents back to back; outputs: vac[2], raw/connected [2][nt]
 * (index 0 = plaquette basis element, 1 = rectangle). */
int or_scalar_connected_correlators(const int64_t *ext, const double *configs, int64_t ncfg,
                                    double *vac, double *raw, double *connected) {
    if (ncfg == 0) return YM_ERR_EMPTY_CONFIGURATION_SET;
    if (ncfg > 64) return YM_ERR_TOO_MANY_CONFIGURATIONS;
    int64_t nt = ext[3];
    if (nt > 64) return YM_ERR_TIME_EXTENT_TOO_LARGE;
    extents4 e; int64_t nl;
    int st = extents_from(ext, &e, 0, &nl);
    if (st) return st;
    double *ps = malloc((size_t)(ncfg * nt) * sizeof(double));
    double *rs = malloc((size_t)(ncfg * nt) * sizeof(double));
    if (!ps || !rs) { free(ps); free(rs); return YM_ERR_ALLOCATION_FAILED; }
    for (int64_t c = 0; c < ncfg && !st; ++c)
        for (int64_t t = 0; t < nt && !st; ++t) {
            int64_t pc, rc;
            st = or_scalar_a1pp_operator_basis(ext, configs + c * nl * 18, t, &ps[c * nt + t],
                                               &rs[c * nt + t], &pc, &rc);
        }
    if (!st) st = or_periodic_connected_estimator(ps, ncfg, nt, &vac[0], raw, connected);
    if (!st) st = or_periodic_connected_estimator(rs, ncfg, nt, &vac[1], raw + nt, connected + nt);
    free(ps);
    free(rs);
    return st;
}

/* or_su3.c -- CPU oracle: SU(3) algebra, lattice, paths and the Metropolis
 * ensemble, restated from the reference crate.  TEST INFRASTRUCTURE ONLY
 * (see or_internal.h).
 *
 *   Mat3 / Su3 / exp        reference/rust/src/su3.rs:77-450
 *   Su3Lattice4             reference/rust/src/su3_lattice.rs:85-346
 *   path holonomy / loops   reference/rust/src/path_holonomy.rs:132-260
 *   Metropolis ensemble     reference/rust/src/su3_ensemble.rs:183-480
 */
#include <stdlib.h>

#include "oracle.h"
#include "or_internal.h"

#define SU3_TOL 5.0e-12                 /* SU3_ACCEPTANCE_TOLERANCE su3.rs:20 */
#define EXP_MAX_COEF 64.0               /* su3.rs:21 */
#define INV_SQRT_3 0.5773502691896258   /* su3.rs:22 */
#define EXP_TAYLOR_TERMS 64             /* su3.rs:23 */
#define EXP_SCALE_TARGET 0.5            /* su3.rs:24 */
#define EXP_TERM_CUTOFF 1.0e-18         /* su3.rs:25 */
#define MAX_SU3_LINKS ((int64_t)1 << 18) /* su3_lattice.rs:17 */

/* ------------------------------------------------------------------ Mat3 */

mat3 m3_zero(void) { mat3 z; memset(&z, 0, sizeof z); return z; }

mat3 m3_identity(void) {
    mat3 z = m3_zero();
    for (int i = 0; i < 3; ++i) z.m[i][i] = c_make(1.0, 0.0);
    return z;
}

mat3 m3_add(mat3 a, mat3 b) {
    mat3 o;
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) o.m[r][c] = c_add(a.m[r][c], b.m[r][c]);
    return o;
}

mat3 m3_sub(mat3 a, mat3 b) {
    mat3 o;
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) o.m[r][c] = c_sub(a.m[r][c], b.m[r][c]);
    return o;
}

mat3 m3_scale_real(mat3 a, double f) {
    mat3 o;
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) o.m[r][c] = c_scale(a.m[r][c], f);
    return o;
}

mat3 m3_scale_complex(mat3 a, c64 f) {
    mat3 o;
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) o.m[r][c] = c_mul(a.m[r][c], f);
    return o;
}

/* su3.rs:147-159: every entry accumulated from Complex64::ZERO over k = 0,1,2. */
mat3 m3_mul(mat3 a, mat3 b) {
    mat3 o;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            c64 v = c_make(0.0, 0.0);
            for (int k = 0; k < 3; ++k) v = c_add(v, c_mul(a.m[r][k], b.m[k][c]));
            o.m[r][c] = v;
        }
    return o;
}

mat3 m3_dagger(mat3 a) {
    mat3 o;
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) o.m[r][c] = c_conj(a.m[c][r]);
    return o;
}

c64 m3_trace(mat3 a) { return c_add(c_add(a.m[0][0], a.m[1][1]), a.m[2][2]); }

/* su3.rs:175-189 (cofactor expansion along the first row). */
c64 m3_det(mat3 a) {
    c64 A = a.m[0][0], B = a.m[0][1], C = a.m[0][2];
    c64 D = a.m[1][0], E = a.m[1][1], F = a.m[1][2];
    c64 G = a.m[2][0], H = a.m[2][1], I = a.m[2][2];
    c64 t1 = c_mul(A, c_sub(c_mul(E, I), c_mul(F, H)));
    c64 t2 = c_mul(B, c_sub(c_mul(D, I), c_mul(F, G)));
    c64 t3 = c_mul(C, c_sub(c_mul(D, H), c_mul(E, G)));
    return c_add(c_sub(t1, t2), t3);
}

double m3_max_abs(mat3 a) {
    double m = 0.0;
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) m = rmax(m, c_abs(a.m[r][c]));
    return m;
}

double m3_one_norm(mat3 a) {
    double best = 0.0;
    for (int c = 0; c < 3; ++c) {
        double s = 0.0;
        for (int r = 0; r < 3; ++r) s += c_abs(a.m[r][c]);
        best = rmax(best, s);
    }
    return best;
}

double m3_max_residual(mat3 a, mat3 b) { return m3_max_abs(m3_sub(a, b)); }
double m3_hermiticity_residual(mat3 a) { return m3_max_residual(a, m3_dagger(a)); }

double m3_unitarity_residual(mat3 a) {
    double left = m3_max_residual(m3_mul(m3_dagger(a), a), m3_identity());
    double right = m3_max_residual(m3_mul(a, m3_dagger(a)), m3_identity());
    return rmax(left, right);
}

double m3_determinant_residual(mat3 a) {
    double direct = c_abs(c_sub(m3_det(a), c_make(1.0, 0.0)));
    double dag = c_abs(c_sub(m3_det(m3_dagger(a)), c_make(1.0, 0.0)));
    return rmax(direct, dag);
}

int m3_finite(mat3 a) {
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) if (!c_finite(a.m[r][c])) return 0;
    return 1;
}

/* ------------------------------------------------------------------ Su3 */

int su3_checked(mat3 a, mat3 *out) {          /* su3.rs:242-253 */
    if (!m3_finite(a)) return YM_ERR_NON_FINITE_MATRIX;
    if (m3_unitarity_residual(a) > SU3_TOL) return YM_ERR_NON_UNITARY_MATRIX;
    if (m3_determinant_residual(a) > SU3_TOL) return YM_ERR_DETERMINANT_NOT_ONE;
    *out = a;
    return YM_OK;
}

int su3_mul_checked(mat3 a, mat3 b, mat3 *out) { return su3_checked(m3_mul(a, b), out); }

int su3_gell_mann(int index, mat3 *out) {     /* su3.rs:325-348 */
    mat3 g = m3_zero();
    switch (index) {
    case 0: g.m[0][1] = c_make(1, 0); g.m[1][0] = c_make(1, 0); break;
    case 1: g.m[0][1] = c_make(0, -1); g.m[1][0] = c_make(0, 1); break;
    case 2: g.m[0][0] = c_make(1, 0); g.m[1][1] = c_make(-1, 0); break;
    case 3: g.m[0][2] = c_make(1, 0); g.m[2][0] = c_make(1, 0); break;
    case 4: g.m[0][2] = c_make(0, -1); g.m[2][0] = c_make(0, 1); break;
    case 5: g.m[1][2] = c_make(1, 0); g.m[2][1] = c_make(1, 0); break;
    case 6: g.m[1][2] = c_make(0, -1); g.m[2][1] = c_make(0, 1); break;
    case 7:
        g.m[0][0] = c_make(INV_SQRT_3, 0);
        g.m[1][1] = c_make(INV_SQRT_3, 0);
        g.m[2][2] = c_make(-2.0 * INV_SQRT_3, 0);
        break;
    default: return YM_ERR_GENERATOR_INDEX_OUT_OF_RANGE;
    }
    *out = g;
    return YM_OK;
}

int su3_generator(int index, mat3 *out) {
    mat3 g;
    int st = su3_gell_mann(index, &g);
    if (st) return st;
    *out = m3_scale_real(g, 0.5);
    return YM_OK;
}

/* su3.rs:409-450: scale-and-square to 1-norm <= 0.5, Taylor until the last
 * term's largest entry is <= 1e-18 (at most 64 terms), square back. */
int su3_matrix_exponential(mat3 a, mat3 *out) {
    if (!m3_finite(a)) return YM_ERR_NON_FINITE_MATRIX;
    double norm = m3_one_norm(a);
    if (!isfinite(norm)) return YM_ERR_NON_FINITE_MATRIX;
    int squarings = 0;
    double scaled_norm = norm;
    while (scaled_norm > EXP_SCALE_TARGET) {
        squarings += 1;
        if (squarings > 32) return YM_ERR_EXPONENTIAL_SCALING_OVERFLOW;
        scaled_norm *= 0.5;
    }
    double scale = ldexp(1.0, -squarings);
    mat3 scaled = m3_scale_real(a, scale);
    mat3 sum = m3_identity(), term = m3_identity();
    for (int order = 1; order <= EXP_TAYLOR_TERMS; ++order) {
        term = m3_scale_real(m3_mul(term, scaled), 1.0 / (double)order);
        sum = m3_add(sum, term);
        if (m3_max_abs(term) <= EXP_TERM_CUTOFF) break;
    }
    for (int s = 0; s < squarings; ++s) sum = m3_mul(sum, sum);
    if (!m3_finite(sum)) return YM_ERR_NON_FINITE_MATRIX;
    *out = sum;
    return YM_OK;
}

int su3_from_algebra(const double coef[8], mat3 *out) {   /* su3.rs:255-262,395-407 */
    mat3 h = m3_zero();
    for (int i = 0; i < 8; ++i) {
        if (!isfinite(coef[i])) return YM_ERR_NON_FINITE_COEFFICIENT;
        if (fabs(coef[i]) > EXP_MAX_COEF) return YM_ERR_ALGEBRA_COEFFICIENT_TOO_LARGE;
        mat3 g;
        su3_generator(i, &g);
        h = m3_add(h, m3_scale_real(g, coef[i]));
    }
    mat3 e;
    int st = su3_matrix_exponential(m3_scale_complex(h, c_make(0.0, 1.0)), &e);
    if (st) return st;
    return su3_checked(e, out);
}

/* ---------------------------------------------------------------- lattice */

int extents_from(const int64_t *ext, extents4 *e, int64_t max_links, int64_t *links_out) {
    int64_t sites = 1;
    for (int i = 0; i < 4; ++i) {
        if (ext[i] < 2) return YM_ERR_INVALID_LATTICE_EXTENT;
        e->n[i] = ext[i];
    }
    for (int i = 0; i < 4; ++i) {
        if (sites > INT64_MAX / ext[i]) return YM_ERR_LATTICE_SIZE_OVERFLOW;
        sites *= ext[i];
    }
    if (sites > INT64_MAX / 4) return YM_ERR_LATTICE_SIZE_OVERFLOW;
    if (max_links > 0 && sites * 4 > max_links) return YM_ERR_LATTICE_TOO_LARGE;
    if (links_out) *links_out = sites * 4;
    return YM_OK;
}

static int64_t su3_cap(int lift_cap) { return lift_cap ? 0 : MAX_SU3_LINKS; }

int or_su3_identity(const int64_t *ext, int lift_cap, double *links) {
    extents4 e; int64_t nl;
    int st = extents_from(ext, &e, su3_cap(lift_cap), &nl);
    if (st) return st;
    mat3 id = m3_identity();
    for (int64_t l = 0; l < nl; ++l) su3_store(links, l, id);
    return YM_OK;
}

/* su3_lattice.rs:168-181: U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag, each
 * product checked. */
int su3_plaquette(const extents4 *e, const double *links, const int64_t x[4], int mu, int nu,
                  mat3 *out) {
    if (mu < 0 || mu >= 4 || nu < 0 || nu >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    if (mu == nu) return YM_ERR_DIRECTIONS_MUST_DIFFER;
    if (!coord_ok(e, x)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    int64_t xm[4], xn[4];
    nb_plus(e, x, mu, xm);
    nb_plus(e, x, nu, xn);
    mat3 p;
    int st = su3_mul_checked(su3_link(e, links, x, mu), su3_link(e, links, xm, nu), &p);
    if (st) return st;
    st = su3_mul_checked(p, m3_dagger(su3_link(e, links, xn, mu)), &p);
    if (st) return st;
    st = su3_mul_checked(p, m3_dagger(su3_link(e, links, x, nu)), &p);
    if (st) return st;
    *out = p;
    return YM_OK;
}

int or_su3_plaquette_matrix(const int64_t *ext, const double *links, const int64_t *x, int mu,
                            int nu, double *out18) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    mat3 p;
    st = su3_plaquette(&e, links, x, mu, nu, &p);
    if (st) return st;
    memcpy(out18, &p, sizeof p);
    return YM_OK;
}

int or_su3_wilson_action(const int64_t *ext, const double *links, double beta, double *out) {
    extents4 e;
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
                        for (int nu = mu + 1; nu < 4; ++nu) {
                            mat3 p;
                            st = su3_plaquette(&e, links, x, mu, nu, &p);
                            if (st) return st;
                            sum += 1.0 - m3_trace(p).re / 3.0;
                            if (!isfinite(sum)) return YM_ERR_NON_FINITE_ACTION;
                        }
    double action = beta * sum;
    if (!isfinite(action)) return YM_ERR_NON_FINITE_ACTION;
    *out = action;
    return YM_OK;
}

/* su3_lattice.rs:185-212 */
int or_su3_polyakov_loop(const int64_t *ext, const double *links, const int64_t *start, int dir,
                         double *out_re, double *out_im) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    if (dir < 0 || dir >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    if (!coord_ok(&e, start)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    int64_t x[4];
    memcpy(x, start, sizeof x);
    mat3 h = m3_identity();
    for (int64_t k = 0; k < e.n[dir]; ++k) {
        st = su3_mul_checked(h, su3_link(&e, links, x, dir), &h);
        if (st) return st;
        int64_t y[4];
        nb_plus(&e, x, dir, y);
        memcpy(x, y, sizeof x);
    }
    c64 t = c_scale(m3_trace(h), 1.0 / 3.0);
    *out_re = t.re;
    *out_im = t.im;
    return YM_OK;
}

/* su3_lattice.rs:244-283; omega is given per site (lexicographic site order). */
int or_su3_gauge_transform(const int64_t *ext, const double *links, const double *site_gauges,
                           double *out_links) {
    extents4 e;
    int64_t x[4];
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    for (x[0] = 0; x[0] < e.n[0]; ++x[0])
        for (x[1] = 0; x[1] < e.n[1]; ++x[1])
            for (x[2] = 0; x[2] < e.n[2]; ++x[2])
                for (x[3] = 0; x[3] < e.n[3]; ++x[3]) {
                    int64_t s = site_index(&e, x);
                    mat3 gx = su3_load(site_gauges, s);
                    for (int mu = 0; mu < 4; ++mu) {
                        int64_t xp[4];
                        nb_plus(&e, x, mu, xp);
                        mat3 gxp = su3_load(site_gauges, site_index(&e, xp));
                        mat3 v;
                        st = su3_mul_checked(gx, su3_load(links, s * 4 + mu), &v);
                        if (st) return st;
                        st = su3_mul_checked(v, m3_dagger(gxp), &v);
                        if (st) return st;
                        su3_store(out_links, s * 4 + mu, v);
                    }
                }
    return YM_OK;
}

/* su3_lattice.rs:285-297 */
int or_su3_max_residuals(const int64_t *ext, const double *links, double *unitarity,
                         double *determinant) {
    extents4 e; int64_t nl;
    int st = extents_from(ext, &e, 0, &nl);
    if (st) return st;
    double u = 0.0, d = 0.0;
    for (int64_t l = 0; l < nl; ++l) {
        mat3 m = su3_load(links, l);
        u = rmax(u, m3_unitarity_residual(m));
        d = rmax(d, m3_determinant_residual(m));
    }
    *unitarity = u;
    *determinant = d;
    return YM_OK;
}

/* Fixtures: traceless_cycle_link (su3_lattice.rs:318-325) and
 * deterministic_su3_site_gauge (su3_lattice.rs:327-340). */
int or_su3_traceless_cycle_link(double *out18) {
    mat3 m = m3_zero();
    m.m[0][1] = c_make(1, 0);
    m.m[1][2] = c_make(1, 0);
    m.m[2][0] = c_make(1, 0);
    mat3 c;
    int st = su3_checked(m, &c);
    if (st) return st;
    memcpy(out18, &c, sizeof c);
    return YM_OK;
}

int or_su3_deterministic_site_gauge(const int64_t *x, double *out18) {
    const int64_t mod = 1024;
    int64_t code = ((x[0] % mod) + 3 * (x[1] % mod) + 7 * (x[2] % mod) + 11 * (x[3] % mod)) % mod;
    double coef[8] = {0};
    coef[2] = 0.031 * ((double)code + 1.0);
    mat3 g;
    int st = su3_from_algebra(coef, &g);
    if (st) return st;
    memcpy(out18, &g, sizeof g);
    return YM_OK;
}

int or_su3_from_algebra(const double *coef, double *out18) {
    mat3 g;
    int st = su3_from_algebra(coef, &g);
    if (st) return st;
    memcpy(out18, &g, sizeof g);
    return YM_OK;
}

int or_su3_matrix_residuals(const double *m18, double *unitarity, double *determinant) {
    mat3 m;
    memcpy(&m, m18, sizeof m);
    *unitarity = m3_unitarity_residual(m);
    *determinant = m3_determinant_residual(m);
    return YM_OK;
}

int or_su3_mul(const double *a18, const double *b18, double *out18) {
    mat3 a, b;
    memcpy(&a, a18, sizeof a);
    memcpy(&b, b18, sizeof b);
    mat3 p = m3_mul(a, b);
    memcpy(out18, &p, sizeof p);
    return YM_OK;
}

/* su3.rs:354-368: structure constants through commutator/anticommutator traces. */
int or_su3_structure(int a, int b, int c, double *f, double *d) {
    mat3 ta, tb, tc;
    int st = su3_generator(a, &ta);
    if (!st) st = su3_generator(b, &tb);
    if (!st) st = su3_generator(c, &tc);
    if (st) return st;
    mat3 ab = m3_mul(ta, tb), ba = m3_mul(tb, ta);
    *f = 2.0 * m3_trace(m3_mul(m3_sub(ab, ba), tc)).im;
    *d = 2.0 * m3_trace(m3_mul(m3_add(ab, ba), tc)).re;
    return YM_OK;
}

/* ------------------------------------------------------------------ paths */

/* path_holonomy.rs:132-157.  steps[i] = +(mu+1) forward, -(mu+1) backward. */
int or_su3_path_holonomy(const int64_t *ext, const double *links, const int64_t *start,
                         const int32_t *steps, int64_t nsteps, double *out18, int64_t *end) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    if (nsteps <= 0) return YM_ERR_EMPTY_PATH;
    if (nsteps > ((int64_t)1 << 20)) return YM_ERR_PATH_TOO_LONG;
    for (int64_t i = 0; i < nsteps; ++i) {
        int d = steps[i] > 0 ? steps[i] - 1 : -steps[i] - 1;
        if (steps[i] == 0 || d >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    }
    if (!coord_ok(&e, start)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    int64_t x[4];
    memcpy(x, start, sizeof x);
    mat3 h = m3_identity();
    for (int64_t i = 0; i < nsteps; ++i) {
        mat3 seg;
        int64_t y[4];
        if (steps[i] > 0) {
            int d = steps[i] - 1;
            seg = su3_link(&e, links, x, d);
            nb_plus(&e, x, d, y);
        } else {
            int d = -steps[i] - 1;
            nb_minus(&e, x, d, y);
            seg = m3_dagger(su3_link(&e, links, y, d));
        }
        memcpy(x, y, sizeof x);
        st = su3_mul_checked(h, seg, &h);
        if (st) return st;
    }
    memcpy(out18, &h, sizeof h);
    memcpy(end, x, sizeof x);
    return YM_OK;
}

/* path_holonomy.rs:219-260 */
int or_rectangular_path(int mu, int nu, int64_t r, int64_t t, int32_t *steps, int64_t cap,
                        int64_t *n) {
    if (mu < 0 || mu >= 4 || nu < 0 || nu >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    if (mu == nu) return YM_ERR_DIRECTIONS_MUST_DIFFER;
    if (r == 0 || t == 0) return YM_ERR_ZERO_RECTANGLE_EXTENT;
    int64_t per = 2 * (r + t);
    if (per > ((int64_t)1 << 20)) return YM_ERR_PATH_TOO_LONG;
    if (per > cap) return YM_ERR_INVALID_ARGUMENT;
    int64_t k = 0;
    for (int64_t i = 0; i < r; ++i) steps[k++] = mu + 1;
    for (int64_t i = 0; i < t; ++i) steps[k++] = nu + 1;
    for (int64_t i = 0; i < r; ++i) steps[k++] = -(mu + 1);
    for (int64_t i = 0; i < t; ++i) steps[k++] = -(nu + 1);
    *n = per;
    return YM_OK;
}

/* wilson_loop (path_holonomy.rs:172-181): (1/3) Tr of a closed holonomy. */
int or_su3_wilson_loop(const int64_t *ext, const double *links, const int64_t *start,
                       const int32_t *steps, int64_t nsteps, double *re, double *im) {
    double h[18];
    int64_t end[4];
    int st = or_su3_path_holonomy(ext, links, start, steps, nsteps, h, end);
    if (st) return st;
    for (int i = 0; i < 4; ++i) if (end[i] != start[i]) return YM_ERR_PATH_NOT_CLOSED;
    mat3 m;
    memcpy(&m, h, sizeof m);
    c64 t = c_scale(m3_trace(m), 1.0 / 3.0);
    *re = t.re;
    *im = t.im;
    return YM_OK;
}

/* --------------------------------------------------------------- ensemble */

#define SU3_MAX_BETA 12.0          /* su3_ensemble.rs:24 */
#define SU3_MAX_SWEEPS 512         /* su3_ensemble.rs:25 */
#define SU3_MAX_MEASUREMENTS 512   /* su3_ensemble.rs:26 */
#define MIN_ANGLE 1.0e-8           /* su3_ensemble.rs:27 */
#define MAX_ANGLE 1.0              /* su3_ensemble.rs:28 */
#define PLAQ_TOL 1.0e-12           /* su3_ensemble.rs:29 */
#define LINK_RESIDUAL_LIMIT 5.0e-12 /* su3_ensemble.rs:30 */
#define STREAM_DOMAIN 0x535533454e535631ULL /* su3_ensemble.rs:23 */

uint64_t or_mix64_pub(uint64_t v) { return or_mix64(v); }

uint64_t or_derive_su3_chain_seed(uint64_t master, uint64_t chain) {   /* :189-192 */
    uint64_t lane = (chain + 1) * 0x9E3779B97F4A7C15ULL;
    return or_mix64(master ^ STREAM_DOMAIN ^ lane);
}

static int angle_ok(double a) { return isfinite(a) && a >= MIN_ANGLE && a <= MAX_ANGLE; }

/* su3_ensemble.rs:199-213 */
int or_proposal_angle_from_u64(uint64_t raw, double angle, double *out) {
    if (!angle_ok(angle)) return YM_ERR_PROPOSAL_ANGLE_OUTSIDE_REFERENCE_RANGE;
    uint64_t m = raw & ((1ULL << 52) - 1);
    uint64_t odd = m * 2 + 1;
    double magnitude = angle * (double)odd * (1.0 / 9007199254740992.0);
    double sign = (raw >> 63) == 0 ? -1.0 : 1.0;
    double a = sign * magnitude;
    if (!isfinite(a) || a == 0.0 || fabs(a) >= angle) return YM_ERR_NON_FINITE_STATISTIC;
    *out = a;
    return YM_OK;
}

/* su3_ensemble.rs:228-259 */
int or_su3_average_plaquette(const int64_t *ext, const double *links, double *out) {
    extents4 e;
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
                            mat3 p;
                            st = su3_plaquette(&e, links, x, mu, nu, &p);
                            if (st) return st;
                            double v = m3_trace(p).re / 3.0;
                            if (!isfinite(v)) return YM_ERR_NON_FINITE_STATISTIC;
                            sum += v;
                            count += 1;
                        }
    if (count == 0) return YM_ERR_NON_FINITE_STATISTIC;
    double mean = sum / (double)count;
    if (!isfinite(mean)) return YM_ERR_NON_FINITE_STATISTIC;
    *out = mean;
    return YM_OK;
}

/* su3_ensemble.rs:261-307: six forward and six backward plaquettes with the
 * candidate substituted, every product checked. */
static int local_action_with_value(const extents4 *e, const double *links, const int64_t x[4],
                                   int mu, mat3 u, double beta, double *out) {
    if (!isfinite(beta) || beta < 0.0 || beta > SU3_MAX_BETA)
        return YM_ERR_BETA_OUTSIDE_REFERENCE_RANGE;
    double sum = 0.0;
    int st;
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        int64_t xm[4], xn[4], bx[4], bxm[4];
        nb_plus(e, x, mu, xm);
        nb_plus(e, x, nu, xn);
        mat3 f;
        st = su3_mul_checked(u, su3_link(e, links, xm, nu), &f);
        if (!st) st = su3_mul_checked(f, m3_dagger(su3_link(e, links, xn, mu)), &f);
        if (!st) st = su3_mul_checked(f, m3_dagger(su3_link(e, links, x, nu)), &f);
        if (st) return st;
        nb_minus(e, x, nu, bx);
        nb_plus(e, bx, mu, bxm);
        mat3 b;
        st = su3_mul_checked(su3_link(e, links, bx, mu), su3_link(e, links, bxm, nu), &b);
        if (!st) st = su3_mul_checked(b, m3_dagger(u), &b);
        if (!st) st = su3_mul_checked(b, m3_dagger(su3_link(e, links, bx, nu)), &b);
        if (st) return st;
        sum += 1.0 - m3_trace(f).re / 3.0;
        sum += 1.0 - m3_trace(b).re / 3.0;
        if (!isfinite(sum)) return YM_ERR_NON_FINITE_STATISTIC;
    }
    double action = beta * sum;
    if (!isfinite(action)) return YM_ERR_NON_FINITE_STATISTIC;
    *out = action;
    return YM_OK;
}

/* su3_ensemble.rs:319-334 */
int or_su3_local_action_difference(const int64_t *ext, const double *links, const int64_t *x,
                                   int mu, const double *cand18, double beta, double *out) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    if (mu < 0 || mu >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    if (!coord_ok(&e, x)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    mat3 cand, old = su3_link(&e, links, x, mu);
    memcpy(&cand, cand18, sizeof cand);
    double a_old, a_new;
    st = local_action_with_value(&e, links, x, mu, old, beta, &a_old);
    if (st) return st;
    st = local_action_with_value(&e, links, x, mu, cand, beta, &a_new);
    if (st) return st;
    double d = a_new - a_old;
    if (!isfinite(d)) return YM_ERR_NON_FINITE_STATISTIC;
    *out = d;
    return YM_OK;
}

/* su3_ensemble.rs:336-340 */
static int generator_proposal(int g, double angle, mat3 *out) {
    double coef[8] = {0};
    coef[g] = angle;
    return su3_from_algebra(coef, out);
}

/* su3_ensemble.rs:342-391.  `lift_cap` only skips the 2^18-link guard so the
 * CPU baseline can run the reference algorithm on larger lattices. */
int or_su3_metropolis_sweep(const int64_t *ext, double *links, double beta, double angle,
                            uint64_t *rng, uint64_t *proposals, uint64_t *accepts) {
    extents4 e;
    int64_t x[4];
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    if (!isfinite(beta) || beta < 0.0 || beta > SU3_MAX_BETA)
        return YM_ERR_BETA_OUTSIDE_REFERENCE_RANGE;
    if (!angle_ok(angle)) return YM_ERR_PROPOSAL_ANGLE_OUTSIDE_REFERENCE_RANGE;
    uint64_t np = 0, na = 0;
    for (x[0] = 0; x[0] < e.n[0]; ++x[0])
        for (x[1] = 0; x[1] < e.n[1]; ++x[1])
            for (x[2] = 0; x[2] < e.n[2]; ++x[2])
                for (x[3] = 0; x[3] < e.n[3]; ++x[3])
                    for (int mu = 0; mu < 4; ++mu)
                        for (int g = 0; g < 8; ++g) {
                            double a;
                            st = or_proposal_angle_from_u64(sm_next(rng), angle, &a);
                            if (st) return st;
                            mat3 rot, cand;
                            st = generator_proposal(g, a, &rot);
                            if (st) return st;
                            int64_t l = site_index(&e, x) * 4 + mu;
                            st = su3_mul_checked(rot, su3_load(links, l), &cand);
                            if (st) return st;
                            double delta;
                            st = or_su3_local_action_difference(ext, links, x, mu,
                                                                (const double *)&cand, beta,
                                                                &delta);
                            if (st) return st;
                            double acc = exp(-rmax(delta, 0.0));
                            if (!isfinite(acc) || !(acc >= 0.0 && acc <= 1.0))
                                return YM_ERR_NON_FINITE_STATISTIC;
                            double u = sm_unit(rng);
                            np += 1;
                            if (u < acc) {
                                su3_store(links, l, cand);
                                na += 1;
                            }
                        }
    *proposals = np;
    *accepts = na;
    return YM_OK;
}

/* su3_ensemble.rs:408-480.  Output: measurements[measurements], report
 * scalars, final residuals.  Diagnostics are computed by the caller with
 * or_diagnostics (su2_ensemble.rs:375-463), as run_chain does. */
int or_su3_run_chain(const or_su3_config *cfg, double *links_out, double *measurements,
                     or_su3_chain_scalars *out) {
    if (!isfinite(cfg->beta) || cfg->beta < 0.0 || cfg->beta > SU3_MAX_BETA)
        return YM_ERR_BETA_OUTSIDE_REFERENCE_RANGE;
    if (!angle_ok(cfg->proposal_angle)) return YM_ERR_PROPOSAL_ANGLE_OUTSIDE_REFERENCE_RANGE;
    if (cfg->measurements < 2 || cfg->measurements > SU3_MAX_MEASUREMENTS)
        return YM_ERR_MEASUREMENT_COUNT_OUTSIDE_REFERENCE_RANGE;
    if (cfg->sweeps_between_measurements == 0) return YM_ERR_ZERO_MEASUREMENT_STRIDE;
    if (cfg->autocorrelation_max_lag >= cfg->measurements)
        return YM_ERR_AUTOCORRELATION_LAG_OUT_OF_RANGE;
    int64_t total = cfg->thermalization_sweeps +
                    cfg->measurements * cfg->sweeps_between_measurements;
    if (total > SU3_MAX_SWEEPS || total < 0) return YM_ERR_SCHEDULE_OUTSIDE_REFERENCE_RANGE;
    extents4 e;
    int64_t nl;
    for (int i = 0; i < 4; ++i)
        if (cfg->extents[i] < 2) return YM_ERR_LATTICE_OUTSIDE_REFERENCE_RANGE;
    if (extents_from(cfg->extents, &e, MAX_SU3_LINKS, &nl)) return YM_ERR_LATTICE_OUTSIDE_REFERENCE_RANGE;

    uint64_t seed = or_derive_su3_chain_seed(cfg->master_seed, cfg->chain_id);
    uint64_t rng = seed;
    or_su3_identity(cfg->extents, 0, links_out);
    uint64_t np = 0, na = 0, p, a;
    int st;
    for (int64_t s = 0; s < cfg->thermalization_sweeps; ++s) {
        st = or_su3_metropolis_sweep(cfg->extents, links_out, cfg->beta, cfg->proposal_angle,
                                     &rng, &p, &a);
        if (st) return st;
        np += p;
        na += a;
    }
    for (int64_t m = 0; m < cfg->measurements; ++m) {
        for (int64_t s = 0; s < cfg->sweeps_between_measurements; ++s) {
            st = or_su3_metropolis_sweep(cfg->extents, links_out, cfg->beta, cfg->proposal_angle,
                                         &rng, &p, &a);
            if (st) return st;
            np += p;
            na += a;
        }
        double v;
        st = or_su3_average_plaquette(cfg->extents, links_out, &v);
        if (st) return st;
        if (v < -0.5 - PLAQ_TOL || v > 1.0 + PLAQ_TOL) return YM_ERR_NON_FINITE_STATISTIC;
        measurements[m] = v;
    }
    if (np == 0) return YM_ERR_NON_FINITE_STATISTIC;
    out->derived_seed = seed;
    out->total_sweeps = total;
    out->proposals = np;
    out->accepts = na;
    out->mean_acceptance = (double)na / (double)np;
    or_su3_max_residuals(cfg->extents, links_out, &out->final_unitarity_residual,
                         &out->final_determinant_residual);
    if (!isfinite(out->mean_acceptance) || !isfinite(out->final_unitarity_residual) ||
        !isfinite(out->final_determinant_residual) ||
        out->final_unitarity_residual > LINK_RESIDUAL_LIMIT ||
        out->final_determinant_residual > LINK_RESIDUAL_LIMIT)
        return YM_ERR_NON_FINITE_STATISTIC;
    return YM_OK;
}

/* or_b200.c -- CPU oracle for the engine's own update order.
 *
 * TEST INFRASTRUCTURE ONLY (see or_internal.h).
 *
 * The CUDA engine updates links on an even/odd checkerboard with one
 * counter-based SplitMix64 stream per link visit, instead of the
 * reference's lexicographic single-stream sweep (su3_ensemble.rs:342-391,
 * su2_ensemble.rs:321-346).  The single-link update rule itself is the
 * reference's:
 *   SU(3): left-multiplicative proposal exp(i theta T^a) U, theta on the
 *          paired angle grid (su3_ensemble.rs:199-213), accept iff
 *          u < exp(-max(dS, 0)) (su3_ensemble.rs:368-377);
 *   SU(2): the reference heat-bath sampler (su2_ensemble.rs:220-281) and
 *          overrelaxation V^dag U^dag V^dag (su2_ensemble.rs:283-299).
 * This file restates the engine's order with the reference's arithmetic so
 * the device result can be compared bit for bit.  The only difference in the
 * SU(3) update is the action change: the engine contracts the candidate with
 * the staple sum, dS = (beta/3)*(ReTr(U A) - ReTr(U' A)), where the reference
 * multiplies out twelve plaquettes; the two agree to ~1e-15 and the tests
 * check that against or_su3_local_action_difference.
 *
 * Exponential: for a single generator the reference's dense Taylor series
 * (su3.rs:409-450) only ever multiplies a term by one non-zero entry per
 * column, so every non-zero entry of every term follows the scalar
 * recurrence t_k = (t_{k-1} * h) * fl(1/k) with h the (scaled) coefficient
 * entry; the zero entries only ever add exact zeros.  The functions below
 * evaluate that recurrence, which reproduces the reference rotation's
 * non-zero entries exactly (the tests check this against
 * or_su3_from_algebra for every generator).
 */
#include <stdlib.h>

#include "oracle.h"
#include "or_internal.h"

#define GOLDEN 0x9E3779B97F4A7C15ULL
#define INV_SQRT_3 0.5773502691896258

/* Output n (0-based) of the SplitMix64 stream seeded with `seed`. */
static inline uint64_t splitmix_at(uint64_t seed, uint64_t n) {
    return or_mix64(seed + (n + 1) * GOLDEN);
}

uint64_t or_cb_link_key(uint64_t chain_seed, uint64_t sweep, int64_t lex, int mu) {
    return splitmix_at(splitmix_at(chain_seed, sweep), (uint64_t)(4 * lex + mu));
}

uint64_t or_splitmix_at(uint64_t seed, uint64_t n) { return splitmix_at(seed, n); }

/* Scalar Taylor chain of the reference exponential: returns the number of
 * terms; c = 1 - t2 + t4 - ..., s = t1 - t3 + ... accumulated in order. */
static int taylor_chain(double h, double *c_out, double *s_out, double *tk_max_out, int nmax) {
    double t = 1.0, c = 1.0, s = 0.0;
    int k;
    for (k = 1; k <= nmax; ++k) {
        t = (t * h) * (1.0 / (double)k);
        switch (k & 3) {
        case 1: s = s + t; break;
        case 2: c = c - t; break;
        case 3: s = s - t; break;
        case 0: c = c + t; break;
        }
        if (fabs(t) <= 1.0e-18) break;
    }
    *c_out = c;
    *s_out = s;
    if (tk_max_out) *tk_max_out = t;
    return k > nmax ? nmax : k;
}

/* Two chains advanced in lock-step (generator 8): the series stops when the
 * larger term magnitude reaches the cutoff, as max_abs_entry does. */
static void taylor_chain2(double h1, double h2, double *c1, double *s1, double *c2, double *s2) {
    double t1 = 1.0, t2 = 1.0;
    double a1 = 1.0, b1 = 0.0, a2 = 1.0, b2 = 0.0;
    for (int k = 1; k <= 64; ++k) {
        double inv = 1.0 / (double)k;
        t1 = (t1 * h1) * inv;
        t2 = (t2 * h2) * inv;
        switch (k & 3) {
        case 1: b1 = b1 + t1; b2 = b2 + t2; break;
        case 2: a1 = a1 - t1; a2 = a2 - t2; break;
        case 3: b1 = b1 - t1; b2 = b2 - t2; break;
        case 0: a1 = a1 + t1; a2 = a2 + t2; break;
        }
        if (fmax(fabs(t1), fabs(t2)) <= 1.0e-18) break;
    }
    *c1 = a1; *s1 = b1; *c2 = a2; *s2 = b2;
}

static inline c64 cm(c64 a, c64 b) { return c_mul(a, b); }

/* exp(i theta T^g) with the reference's arithmetic, written into a dense
 * 3x3 (zero entries are +0). */
int or_su3_generator_rotation(int g, double theta, double *out18) {
    if (g < 0 || g > 7) return YM_ERR_GENERATOR_INDEX_OUT_OF_RANGE;
    if (!isfinite(theta)) return YM_ERR_NON_FINITE_COEFFICIENT;
    if (fabs(theta) > 64.0) return YM_ERR_ALGEBRA_COEFFICIENT_TOO_LARGE;
    mat3 r = m3_identity();
    if (g < 7) {
        /* block (i0, i1) of the SU(2) subgroup; h = fl(0.5*theta) */
        static const int blk[7][2] = {{0, 1}, {0, 1}, {0, 1}, {0, 2}, {0, 2}, {1, 2}, {1, 2}};
        int i0 = blk[g][0], i1 = blk[g][1];
        double h = 0.5 * theta;
        int sq = 0;
        double nrm = fabs(h);
        while (nrm > 0.5) { sq++; if (sq > 32) return YM_ERR_EXPONENTIAL_SCALING_OVERFLOW; nrm *= 0.5; }
        double hs = h * ldexp(1.0, -sq);
        double c, s;
        taylor_chain(hs, &c, &s, NULL, 64);
        c64 a, b, cc, d;   /* [[a, b], [cc, d]] */
        if (g == 0 || g == 3 || g == 5) {          /* lambda_1,4,6: i h sigma_x */
            a = c_make(c, 0); b = c_make(0, s); cc = c_make(0, s); d = c_make(c, 0);
        } else if (g == 1 || g == 4 || g == 6) {   /* lambda_2,5,7: i h sigma_y (real) */
            a = c_make(c, 0); b = c_make(s, 0); cc = c_make(-s, 0); d = c_make(c, 0);
        } else {                                   /* lambda_3: diag(i h, -i h) */
            a = c_make(c, s); b = c_make(0, 0); cc = c_make(0, 0); d = c_make(c, -s);
        }
        for (int k = 0; k < sq; ++k) {
            c64 na = c_add(cm(a, a), cm(b, cc));
            c64 nb = c_add(cm(a, b), cm(b, d));
            c64 nc = c_add(cm(cc, a), cm(d, cc));
            c64 nd = c_add(cm(cc, b), cm(d, d));
            a = na; b = nb; cc = nc; d = nd;
        }
        r.m[i0][i0] = a; r.m[i0][i1] = b; r.m[i1][i0] = cc; r.m[i1][i1] = d;
    } else {
        double d1 = (0.5 * INV_SQRT_3) * theta;
        double d2 = (-INV_SQRT_3) * theta;
        int sq = 0;
        double nrm = fmax(fabs(d1), fabs(d2));
        while (nrm > 0.5) { sq++; if (sq > 32) return YM_ERR_EXPONENTIAL_SCALING_OVERFLOW; nrm *= 0.5; }
        double sc = ldexp(1.0, -sq);
        double c1, s1, c2, s2;
        taylor_chain2(d1 * sc, d2 * sc, &c1, &s1, &c2, &s2);
        c64 e1 = c_make(c1, s1), e2 = c_make(c2, s2);
        for (int k = 0; k < sq; ++k) { e1 = cm(e1, e1); e2 = cm(e2, e2); }
        r.m[0][0] = e1; r.m[1][1] = e1; r.m[2][2] = e2;
    }
    memcpy(out18, &r, sizeof r);
    return YM_OK;
}

/* acc += a*b as four fused multiply-adds in a fixed order (the engine's
 * staple and trace formulation; C99 fma() rounds exactly like the device). */
static inline void c_fma_acc(c64 *acc, c64 a, c64 b) {
    acc->re = fma(a.re, b.re, acc->re);
    acc->re = fma(-a.im, b.im, acc->re);
    acc->im = fma(a.re, b.im, acc->im);
    acc->im = fma(a.im, b.re, acc->im);
}

/* Staple sum A = sum_{nu != mu} [U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
 *                              + U_nu(x-nu+mu)^dag U_mu(x-nu)^dag U_nu(x-nu)],
 * nu ascending, forward then backward.  Each term: P = product of the first
 * two factors as fma chains from zero (j = 0,1,2), then A[r][c] += P[r][k] *
 * third[k][c] as fma chains over k = 0,1,2 into the running sum. */
static mat3 su3_staple(const extents4 *e, const double *links, const int64_t x[4], int mu) {
    mat3 a = m3_zero();
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        int64_t xpm[4], xpn[4], xmn[4], xmnpm[4];
        nb_plus(e, x, mu, xpm);
        nb_plus(e, x, nu, xpn);
        nb_minus(e, x, nu, xmn);
        nb_plus(e, xmn, mu, xmnpm);
        mat3 l1 = su3_link(e, links, xpm, nu), l2 = su3_link(e, links, xpn, mu);
        mat3 l3 = su3_link(e, links, x, nu), p;
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k) {
                c64 v = c_make(0.0, 0.0);
                for (int j = 0; j < 3; ++j) c_fma_acc(&v, l1.m[r][j], c_conj(l2.m[k][j]));
                p.m[r][k] = v;
            }
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                for (int k = 0; k < 3; ++k) c_fma_acc(&a.m[r][c], p.m[r][k], c_conj(l3.m[c][k]));
        l1 = su3_link(e, links, xmnpm, nu);
        l2 = su3_link(e, links, xmn, mu);
        l3 = su3_link(e, links, xmn, nu);
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k) {
                c64 v = c_make(0.0, 0.0);
                for (int j = 0; j < 3; ++j) c_fma_acc(&v, c_conj(l1.m[j][r]), c_conj(l2.m[k][j]));
                p.m[r][k] = v;
            }
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                for (int k = 0; k < 3; ++k) c_fma_acc(&a.m[r][c], p.m[r][k], l3.m[k][c]);
    }
    return a;
}

int or_su3_staple(const int64_t *ext, const double *links, const int64_t *x, int mu, double *out18) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    mat3 a = su3_staple(&e, links, x, mu);
    memcpy(out18, &a, sizeof a);
    return YM_OK;
}

/* ReTr(X A) = (r0 + r1) + r2 with row i a fused chain:
 * r = x0.re*a0.re; r = fma(-x0.im, a0.im, r); r = fma(x1.re, a1.re, r);
 * r = fma(-x1.im, a1.im, r); r = fma(x2.re, a2.re, r); r = fma(-x2.im, a2.im, r)
 * where a_k = A[k][i]. */
static double retr_product(const mat3 *x, const mat3 *a) {
    double r[3];
    for (int i = 0; i < 3; ++i) {
        double acc = x->m[i][0].re * a->m[0][i].re;
        acc = fma(-x->m[i][0].im, a->m[0][i].im, acc);
        acc = fma(x->m[i][1].re, a->m[1][i].re, acc);
        acc = fma(-x->m[i][1].im, a->m[1][i].im, acc);
        acc = fma(x->m[i][2].re, a->m[2][i].re, acc);
        acc = fma(-x->m[i][2].im, a->m[2][i].im, acc);
        r[i] = acc;
    }
    return (r[0] + r[1]) + r[2];
}

/* Rows of R*U for the rows the rotation touches, accumulated in ascending
 * index order (the order of Mat3::mul); untouched rows stay bitwise equal. */
static mat3 rotate_rows(int g, const mat3 *r, const mat3 *u) {
    static const int blk[8][2] = {{0, 1}, {0, 1}, {0, 1}, {0, 2}, {0, 2}, {1, 2}, {1, 2}, {0, 1}};
    mat3 o = *u;
    if (g < 7) {
        int i0 = blk[g][0], i1 = blk[g][1];
        for (int c = 0; c < 3; ++c) {
            o.m[i0][c] = c_add(cm(r->m[i0][i0], u->m[i0][c]), cm(r->m[i0][i1], u->m[i1][c]));
            o.m[i1][c] = c_add(cm(r->m[i1][i0], u->m[i0][c]), cm(r->m[i1][i1], u->m[i1][c]));
        }
    } else {
        for (int i = 0; i < 3; ++i)
            for (int c = 0; c < 3; ++c) o.m[i][c] = cm(r->m[i][i], u->m[i][c]);
    }
    return o;
}

/* One link visit: 8 hits, generator h (ordered) or bits 52..54 of the angle
 * word (uniform), two stream words per hit as in the reference. */
static void su3_visit(mat3 *u, const mat3 *a, double beta, double angle, uint64_t key,
                      int uniform_generator, uint64_t *np, uint64_t *na) {
    double old_tr = retr_product(u, a);
    for (int h = 0; h < 8; ++h) {
        uint64_t w_angle = splitmix_at(key, (uint64_t)(2 * h));
        uint64_t w_acc = splitmix_at(key, (uint64_t)(2 * h + 1));
        int g = uniform_generator ? (int)((w_angle >> 52) & 7) : h;
        double theta;
        or_proposal_angle_from_u64(w_angle, angle, &theta);
        mat3 r, cand;
        or_su3_generator_rotation(g, theta, (double *)&r);
        cand = rotate_rows(g, &r, u);
        double new_tr = retr_product(&cand, a);
        double ds = (beta / 3.0) * (old_tr - new_tr);
        double acc = exp(-fmax(ds, 0.0));
        double uu = (double)(w_acc >> 11) * (1.0 / 9007199254740992.0);
        *np += 1;
        if (uu < acc) {
            *u = cand;
            old_tr = new_tr;
            *na += 1;
        }
    }
}

/* One hit with a given generator: the paired-grid angle of w_angle at half
 * width `angle` (any positive width; the learned proposal goes beyond the
 * reference's admissible 1.0), the exact rotation, the binary64 accept test
 * on the uniform of w_acc. */
int or_su3_hit(double *u18, const double *a18, double beta, double angle, uint64_t w_angle,
               uint64_t w_acc, int g, uint64_t *accepted) {
    if (!(angle > 0.0) || g < 0 || g > 7) return YM_ERR_INVALID_ARGUMENT;
    mat3 u, a, r, cand;
    memcpy(&u, u18, sizeof u);
    memcpy(&a, a18, sizeof a);
    uint64_t m = w_angle & ((1ULL << 52) - 1);
    double theta = ((w_angle >> 63) == 0 ? -1.0 : 1.0) * (angle * (double)(2 * m + 1) *
                                                          (1.0 / 9007199254740992.0));
    double old_tr = retr_product(&u, &a);
    or_su3_generator_rotation(g, theta, (double *)&r);
    cand = rotate_rows(g, &r, &u);
    double new_tr = retr_product(&cand, &a);
    double ds = (beta / 3.0) * (old_tr - new_tr);
    double acc = exp(-fmax(ds, 0.0));
    double uu = (double)(w_acc >> 11) * (1.0 / 9007199254740992.0);
    *accepted = 0;
    if (uu < acc) {
        memcpy(u18, &cand, sizeof cand);
        *accepted = 1;
    }
    return YM_OK;
}

/* One checkerboard sweep: parity 0 then 1, direction 0..3 within each. */
int or_su3_cb_sweep(const int64_t *ext, double *links, double beta, double angle,
                    uint64_t chain_seed, uint64_t sweep, int uniform_generator,
                    uint64_t *proposals, uint64_t *accepts) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    for (int i = 0; i < 4; ++i) if (e.n[i] % 2) return YM_ERR_NOT_CHECKERBOARDABLE;
    uint64_t np = 0, na = 0;
    for (int p = 0; p < 2; ++p)
        for (int mu = 0; mu < 4; ++mu) {
            int64_t x[4];
            for (x[0] = 0; x[0] < e.n[0]; ++x[0])
                for (x[1] = 0; x[1] < e.n[1]; ++x[1])
                    for (x[2] = 0; x[2] < e.n[2]; ++x[2])
                        for (x[3] = 0; x[3] < e.n[3]; ++x[3]) {
                            if (((x[0] + x[1] + x[2] + x[3]) & 1) != p) continue;
                            int64_t lex = site_index(&e, x);
                            mat3 a = su3_staple(&e, links, x, mu);
                            mat3 u = su3_load(links, lex * 4 + mu);
                            su3_visit(&u, &a, beta, angle,
                                      or_cb_link_key(chain_seed, sweep, lex, mu),
                                      uniform_generator, &np, &na);
                            su3_store(links, lex * 4 + mu, u);
                        }
        }
    *proposals = np;
    *accepts = na;
    return YM_OK;
}

/* Single visit for unit tests: U, A given, returns the updated U. */
int or_su3_visit(double *u18, const double *a18, double beta, double angle, uint64_t key,
                 int uniform_generator, uint64_t *accepts) {
    mat3 u, a;
    memcpy(&u, u18, sizeof u);
    memcpy(&a, a18, sizeof a);
    uint64_t np = 0, na = 0;
    su3_visit(&u, &a, beta, angle, key, uniform_generator, &np, &na);
    memcpy(u18, &u, sizeof u);
    *accepts = na;
    return YM_OK;
}

/* Engine-order per-plaquette value: ReTr of the product in reference order,
 * last factor contracted on the diagonal only, divided by 3. */
int or_su3_plaquette_value(const int64_t *ext, const double *links, const int64_t *x, int mu,
                           int nu, double *out) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    int64_t xm[4], xn[4];
    nb_plus(&e, x, mu, xm);
    nb_plus(&e, x, nu, xn);
    mat3 p = m3_mul(m3_mul(su3_link(&e, links, x, mu), su3_link(&e, links, xm, nu)),
                    m3_dagger(su3_link(&e, links, xn, mu)));
    mat3 q = m3_mul(p, m3_dagger(su3_link(&e, links, x, nu)));
    *out = m3_trace(q).re / 3.0;
    return YM_OK;
}

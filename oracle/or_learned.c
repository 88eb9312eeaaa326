/* or_learned.c -- CPU oracle of the learned SU(3) Metropolis proposal.
 *
 * TEST INFRASTRUCTURE ONLY.  The learned proposal has no reference
 * counterpart; its definition (features, network, objective, proposal) is
 * the one written in include/ym_learned.h, restated here in binary64 with
 * the BF16 roundings of the device network emulated exactly (round to
 * nearest even of the binary32 value).  The sampler around it is the
 * engine's checkerboard Metropolis (or_b200.c), whose update rule follows
 * su3_ensemble.rs:342-391; the accept test u < exp(-max(dS, 0)) is
 * su3_ensemble.rs:368,377.
 */
#include "oracle.h"
#include "or_internal.h"

#include "../include/ym_learned.h"

/* binary32 -> bfloat16 -> binary32, round to nearest even. */
static float bf16r(float x) {
    uint32_t b;
    memcpy(&b, &x, 4);
    if ((b & 0x7F800000u) == 0x7F800000u) return x;
    b += 0x7FFFu + ((b >> 16) & 1u);
    b &= 0xFFFF0000u;
    float r;
    memcpy(&r, &b, 4);
    return r;
}

float or_bf16_round(float x) { return bf16r(x); }

/* Features of a staple sum (a18: row-major re/im). */
static void features_of(const mat3 *a, double beta, double f[16]) {
    mat3 ah = m3_scale_real(*a, 1.0 / 6.0);
    mat3 b = m3_mul(ah, m3_dagger(ah));
    mat3 bb = m3_mul(b, b);
    double t1 = m3_trace(b).re / 3.0;
    double t2 = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t2 += b.m[i][j].re * b.m[i][j].re + b.m[i][j].im * b.m[i][j].im;
    t2 /= 3.0;
    double t3 = m3_trace(m3_mul(bb, b)).re / 3.0;
    c64 d = m3_det(ah);
    double d2 = d.re * d.re + d.im * d.im;
    double st1 = sqrt(fmax(t1, 0.0));
    double k = beta * st1, b6 = beta / 6.0, spread = t2 - t1 * t1;
    f[0] = t1;
    f[1] = t2;
    f[2] = t3;
    f[3] = st1;
    f[4] = d.re;
    f[5] = d.im;
    f[6] = d2;
    f[7] = spread;
    f[8] = b6;
    f[9] = k / 6.0;
    f[10] = (k / 6.0) * (k / 6.0);
    f[11] = 1.0 / (1.0 + k);
    f[12] = b6 * d.re;
    f[13] = b6 * t2;
    f[14] = b6 * d2;
    f[15] = b6 * spread;
}

int or_lp_features(const double *a18, double beta, double *f16) {
    mat3 a;
    memcpy(&a, a18, sizeof a);
    features_of(&a, beta, f16);
    return YM_OK;
}

static float keep(float x) { return x; }

/* Forward of one row with the device's roundings (rnd = bf16r) or without
 * any (rnd = keep); h1, h2 returned for the backward pass, already rounded. */
static void forward_row_r(float (*rnd)(float), const float *p, const float *x16, float xb[16],
                          float h1[64], float h2[64], double y[16]) {
    for (int k = 0; k < 16; ++k) xb[k] = rnd(x16[k]);
    for (int o = 0; o < 64; ++o) {
        double z = 0.0;
        for (int k = 0; k < 16; ++k) z += (double)rnd(p[YM_LP_OFF_W1 + o * 16 + k]) * xb[k];
        z += p[YM_LP_OFF_B1 + o];
        h1[o] = rnd((float)fmax(z, 0.0));
    }
    for (int o = 0; o < 64; ++o) {
        double z = 0.0;
        for (int k = 0; k < 64; ++k) z += (double)rnd(p[YM_LP_OFF_W2 + o * 64 + k]) * h1[k];
        z += p[YM_LP_OFF_B2 + o];
        h2[o] = rnd((float)fmax(z, 0.0));
    }
    for (int o = 0; o < 16; ++o) {
        double z = 0.0;
        for (int k = 0; k < 64; ++k) z += (double)rnd(p[YM_LP_OFF_W3 + o * 64 + k]) * h2[k];
        y[o] = z + p[YM_LP_OFF_B3 + o];
    }
}

static void forward_row(const float *p, const float *x16, float xb[16], float h1[64], float h2[64],
                        double y[16]) {
    forward_row_r(bf16r, p, x16, xb, h1, h2, y);
}

int or_lp_forward(const float *params, const float *x, int64_t n, double *y) {
    float xb[16], h1[64], h2[64];
    for (int64_t r = 0; r < n; ++r) forward_row(params, x + r * 16, xb, h1, h2, y + r * 16);
    return YM_OK;
}

/* Softmax of the logits (q), generator probabilities p = F/8 + (1-F) q and
 * angle half width from the outputs. */
static void proposal_q(const double y[16], double q[8], double p[8], double *s, double *sig) {
    double mx = y[0];
    for (int a = 1; a < 8; ++a) mx = fmax(mx, y[a]);
    double z = 0.0;
    for (int a = 0; a < 8; ++a) {
        q[a] = exp(y[a] - mx);
        z += q[a];
    }
    for (int a = 0; a < 8; ++a) {
        q[a] /= z;
        p[a] = YM_LP_GENERATOR_FLOOR / 8.0 + (1.0 - YM_LP_GENERATOR_FLOOR) * q[a];
    }
    *sig = 1.0 / (1.0 + exp(-y[8]));
    *s = YM_LP_SCALE_MIN + (YM_LP_SCALE_MAX - YM_LP_SCALE_MIN) * *sig;
}

static void proposal_of(const double y[16], double p[8], double *s, double *sig) {
    double q[8];
    proposal_q(y, q, p, s, sig);
}

int or_lp_proposal(const double *y16, double *p8, double *scale) {
    double sig;
    proposal_of(y16, p8, scale, &sig);
    return YM_OK;
}

/* ReTr(R_a(theta) M) and its theta-derivative in closed form.  SU(2)
 * subgroup generators act on rows (i, j) as cos(theta/2) + i sin(theta/2)
 * sigma_k; lambda_8 multiplies rows 0, 1 by e^{i phi} and row 2 by
 * e^{-2 i phi}, phi = theta / (2 sqrt 3). */
static void retr_rotated(int g, const mat3 *mm, double theta, double *f, double *df) {
    static const int blk[7][3] = {{0, 1, 0}, {0, 1, 1}, {0, 1, 2}, {0, 2, 0}, {0, 2, 1}, {1, 2, 0}, {1, 2, 1}};
    const c64 (*m)[3] = mm->m;
    double tr = m[0][0].re + m[1][1].re + m[2][2].re;
    if (g < 7) {
        int i = blk[g][0], j = blk[g][1], kind = blk[g][2];
        double c1 = m[i][i].re + m[j][j].re, c2;
        if (kind == 0) c2 = -(m[i][j].im + m[j][i].im);
        else if (kind == 1) c2 = m[j][i].re - m[i][j].re;
        else c2 = m[j][j].im - m[i][i].im;
        double c = cos(0.5 * theta), s = sin(0.5 * theta);
        *f = (tr - c1) + c1 * c + c2 * s;
        *df = 0.5 * (-c1 * s + c2 * c);
    } else {
        const double k = 0.28867513459481287; /* 1/(2 sqrt 3) */
        double phi = k * theta;
        double mr = m[0][0].re + m[1][1].re, mi = m[0][0].im + m[1][1].im;
        double c = cos(phi), s = sin(phi), c2 = cos(2.0 * phi), s2 = sin(2.0 * phi);
        *f = c * mr - s * mi + c2 * m[2][2].re + s2 * m[2][2].im;
        *df = k * (-s * mr - c * mi) + 2.0 * k * (-s2 * m[2][2].re + c2 * m[2][2].im);
    }
}

/* Objective O = E + w H(q) of one record and dO/dy for outputs 0..8. */
static double objective_row(const double y[16], const mat3 *m, double beta, double dy[9]) {
    double p[8], q[8], s, sig;
    proposal_q(y, q, p, &s, &sig);
    const double b3 = beta / 3.0;
    const double tr = m->m[0][0].re + m->m[1][1].re + m->m[2][2].re;
    const int K = YM_LP_QUADRATURE;
    double J[8], dJ[8], E = 0.0, dEs = 0.0;
    for (int a = 0; a < 8; ++a) {
        double j = 0.0, dj = 0.0;
        for (int q = 0; q < K; ++q) {
            double gk = (q + 0.5) / K;
            for (int sg = -1; sg <= 1; sg += 2) {
                double dth = sg * gk, th = s * dth, f, df;
                retr_rotated(a, m, th, &f, &df);
                double ds = b3 * (tr - f), dds = -b3 * df; /* dS and d dS / d theta */
                double al = ds > 0.0 ? exp(-ds) : 1.0;
                double dal = ds > 0.0 ? -al * dds : 0.0;   /* d alpha / d theta */
                j += al * ds * ds;
                dj += (dal * ds * ds + 2.0 * al * ds * dds) * dth;
            }
        }
        J[a] = j / (2.0 * K);
        dJ[a] = dj / (2.0 * K);
        E += p[a] * J[a];
        dEs += p[a] * dJ[a];
    }
    double Eq = 0.0, H = 0.0;
    for (int a = 0; a < 8; ++a) {
        Eq += q[a] * J[a];
        H -= q[a] * log(q[a]);
    }
    for (int a = 0; a < 8; ++a)
        dy[a] = (1.0 - YM_LP_GENERATOR_FLOOR) * q[a] * (J[a] - Eq) -
                YM_LP_ENTROPY_WEIGHT * q[a] * (log(q[a]) + H);
    dy[8] = dEs * (YM_LP_SCALE_MAX - YM_LP_SCALE_MIN) * sig * (1.0 - sig);
    return E + YM_LP_ENTROPY_WEIGHT * H;
}

int or_lp_retr_rotated(int g, const float *m18, double theta, double *f, double *df) {
    if (g < 0 || g > 7) return YM_ERR_INVALID_ARGUMENT;
    mat3 m;
    for (int i = 0; i < 9; ++i) m.m[i / 3][i % 3] = c_make(m18[2 * i], m18[2 * i + 1]);
    retr_rotated(g, &m, theta, f, df);
    return YM_OK;
}

int or_lp_objective(const double *y16, const float *m18, double beta, double *e_out,
                    double *dy9) {
    mat3 m;
    for (int i = 0; i < 9; ++i) m.m[i / 3][i % 3] = c_make(m18[2 * i], m18[2 * i + 1]);
    *e_out = objective_row(y16, &m, beta, dy9);
    return YM_OK;
}

/* Mean objective and gradient of -mean E with the device's roundings:
 * dY = bf16(-dE/dy), dZ2 = bf16((dY W3) * [h2 > 0]), dZ1 = bf16((dZ2 W2) * [h1 > 0]),
 * weight gradients as outer products of those with the BF16 activations. */
int or_lp_loss_grad_mode(const float *params, const float *x, const float *m18,
                         const double *beta, int64_t n, int exact, double *objective,
                         double *grad) {
    float (*rnd)(float) = exact ? keep : bf16r;
    if (n <= 0) return YM_ERR_INVALID_ARGUMENT;
    memset(grad, 0, sizeof(double) * YM_LP_PARAMS);
    double esum = 0.0;
    float xb[16], h1[64], h2[64];
    for (int64_t r = 0; r < n; ++r) {
        double y[16], dE[9];
        forward_row_r(rnd, params, x + r * 16, xb, h1, h2, y);
        mat3 m;
        for (int i = 0; i < 9; ++i)
            m.m[i / 3][i % 3] = c_make(m18[r * 18 + 2 * i], m18[r * 18 + 2 * i + 1]);
        esum += objective_row(y, &m, beta[r], dE);
        float dyb[16] = {0};
        for (int o = 0; o < 9; ++o) dyb[o] = rnd((float)(-dE[o]));
        float dz2[64], dz1[64];
        for (int j = 0; j < 64; ++j) {
            double acc = 0.0;
            for (int o = 0; o < 16; ++o) acc += (double)dyb[o] * rnd(params[YM_LP_OFF_W3 + o * 64 + j]);
            dz2[j] = rnd(h2[j] > 0.0f ? (float)acc : 0.0f);
        }
        for (int j = 0; j < 64; ++j) {
            double acc = 0.0;
            for (int o = 0; o < 64; ++o) acc += (double)dz2[o] * rnd(params[YM_LP_OFF_W2 + o * 64 + j]);
            dz1[j] = rnd(h1[j] > 0.0f ? (float)acc : 0.0f);
        }
        for (int o = 0; o < 9; ++o) {
            for (int j = 0; j < 64; ++j) grad[YM_LP_OFF_W3 + o * 64 + j] += (double)dyb[o] * h2[j];
            grad[YM_LP_OFF_B3 + o] += dyb[o];
        }
        for (int o = 0; o < 64; ++o) {
            for (int j = 0; j < 64; ++j) grad[YM_LP_OFF_W2 + o * 64 + j] += (double)dz2[o] * h1[j];
            grad[YM_LP_OFF_B2 + o] += dz2[o];
            for (int k = 0; k < 16; ++k) grad[YM_LP_OFF_W1 + o * 16 + k] += (double)dz1[o] * xb[k];
            grad[YM_LP_OFF_B1 + o] += dz1[o];
        }
    }
    for (int i = 0; i < YM_LP_PARAMS; ++i) grad[i] /= (double)n;
    *objective = esum / (double)n;
    return YM_OK;
}

int or_lp_loss_grad(const float *params, const float *x, const float *m18, const double *beta,
                    int64_t n, double *objective, double *grad) {
    return or_lp_loss_grad_mode(params, x, m18, beta, n, 0, objective, grad);
}

/* The same objective in plain binary64 (no BF16 roundings anywhere): the
 * quantity whose finite differences check the analytic gradient. */
int or_lp_objective_exact(const double *params, const double *x, const float *m18,
                          const double *beta, int64_t n, double *objective) {
    double esum = 0.0;
    for (int64_t r = 0; r < n; ++r) {
        double h1[64], h2[64], y[16], dE[9];
        for (int o = 0; o < 64; ++o) {
            double z = params[YM_LP_OFF_B1 + o];
            for (int k = 0; k < 16; ++k) z += params[YM_LP_OFF_W1 + o * 16 + k] * x[r * 16 + k];
            h1[o] = fmax(z, 0.0);
        }
        for (int o = 0; o < 64; ++o) {
            double z = params[YM_LP_OFF_B2 + o];
            for (int k = 0; k < 64; ++k) z += params[YM_LP_OFF_W2 + o * 64 + k] * h1[k];
            h2[o] = fmax(z, 0.0);
        }
        for (int o = 0; o < 16; ++o) {
            double z = params[YM_LP_OFF_B3 + o];
            for (int k = 0; k < 64; ++k) z += params[YM_LP_OFF_W3 + o * 64 + k] * h2[k];
            y[o] = z;
        }
        mat3 m;
        for (int i = 0; i < 9; ++i)
            m.m[i / 3][i % 3] = c_make(m18[r * 18 + 2 * i], m18[r * 18 + 2 * i + 1]);
        esum += objective_row(y, &m, beta[r], dE);
    }
    *objective = esum / (double)n;
    return YM_OK;
}

/* Generator index from the 11 bits 52..62 of the angle word. */
static int pick_generator(uint64_t w, const double p[8]) {
    double u = ((double)((w >> 52) & 0x7FF) + 0.5) * (1.0 / 2048.0), c = 0.0;
    for (int a = 0; a < 7; ++a) {
        c += p[a];
        if (u < c) return a;
    }
    return 7;
}

int or_lp_pick_generator(uint64_t w, const double *p8) { return pick_generator(w, p8); }

/* One learned checkerboard sweep in binary64: features and network from
 * the staple, then the eight hits with the exact (Taylor) rotation. */
int or_lp_cb_sweep(const int64_t *ext, double *links, double beta, const float *params,
                   uint64_t chain_seed, uint64_t sweep, uint64_t *proposals, uint64_t *accepts) {
    extents4 e;
    int st = extents_from(ext, &e, 0, NULL);
    if (st) return st;
    for (int i = 0; i < 4; ++i) if (e.n[i] % 2) return YM_ERR_NOT_CHECKERBOARDABLE;
    uint64_t np = 0, na = 0;
    for (int par = 0; par < 2; ++par)
        for (int mu = 0; mu < 4; ++mu) {
            int64_t x[4];
            for (x[0] = 0; x[0] < e.n[0]; ++x[0])
                for (x[1] = 0; x[1] < e.n[1]; ++x[1])
                    for (x[2] = 0; x[2] < e.n[2]; ++x[2])
                        for (x[3] = 0; x[3] < e.n[3]; ++x[3]) {
                            if (((x[0] + x[1] + x[2] + x[3]) & 1) != par) continue;
                            int64_t lex = site_index(&e, x);
                            double a18[18], u18[18], f[16], y[16], p[8], s;
                            or_su3_staple(ext, links, x, mu, a18);
                            features_of((const mat3 *)a18, beta, f);
                            float fx[16], xb[16], h1[64], h2[64];
                            for (int k = 0; k < 16; ++k) fx[k] = (float)f[k];
                            forward_row(params, fx, xb, h1, h2, y);
                            or_lp_proposal(y, p, &s);
                            memcpy(u18, links + (lex * 4 + mu) * 18, sizeof u18);
                            uint64_t key = or_cb_link_key(chain_seed, sweep, lex, mu);
                            for (int h = 0; h < 8; ++h) {
                                uint64_t wa = or_splitmix_at(key, (uint64_t)(2 * h));
                                uint64_t wu = or_splitmix_at(key, (uint64_t)(2 * h + 1));
                                int g = pick_generator(wa, p);
                                uint64_t acc = 0;
                                st = or_su3_hit(u18, a18, beta, s, wa, wu, g, &acc);
                                if (st) return st;
                                np += 1;
                                na += acc;
                            }
                            memcpy(links + (lex * 4 + mu) * 18, u18, sizeof u18);
                        }
        }
    *proposals = np;
    *accepts = na;
    return YM_OK;
}

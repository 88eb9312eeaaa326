/* or_internal.h -- shared helpers of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a plain-C restatement of the
 * reference Rust crate (QSOLKCB/YANG-MILLS, the files under `reference/rust/src`) used
 * by the test-suite, by `__graft_entry__.smoke()` and by the CPU-baseline leg
 * of `bench.py` to check the CUDA engine.  No product code path may link or
 * call it.
 *
 * Arithmetic rules: binary64 throughout, compiled with -ffp-contract=off (no
 * fused multiply-add), every sum accumulated left to right from zero exactly
 * as the Rust iterator chains do, glibc libm for transcendentals (the same
 * libm Rust's `f64::{exp, exp_m1, ln_1p, sin, cos, hypot}` call on
 * x86_64-unknown-linux-gnu).
 */
#ifndef OR_INTERNAL_H
#define OR_INTERNAL_H

#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include "../include/ym_status.h"

#define OR_DIM 4

typedef struct { double re, im; } c64;
typedef struct { c64 m[3][3]; } mat3;

/* ---- Complex64 (reference/rust/src/su3.rs:27-75) ---- */
static inline c64 c_make(double re, double im) { c64 z; z.re = re; z.im = im; return z; }
static inline c64 c_add(c64 a, c64 b) { return c_make(a.re + b.re, a.im + b.im); }
static inline c64 c_sub(c64 a, c64 b) { return c_make(a.re - b.re, a.im - b.im); }
static inline c64 c_mul(c64 a, c64 b) {
    return c_make(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
static inline c64 c_scale(c64 a, double f) { return c_make(a.re * f, a.im * f); }
static inline c64 c_conj(c64 a) { return c_make(a.re, -a.im); }
static inline double c_abs(c64 a) { return hypot(a.re, a.im); }
static inline int c_finite(c64 a) { return isfinite(a.re) && isfinite(a.im); }

/* Rust's f64::max: returns the other operand when one is NaN (= C fmax). */
static inline double rmax(double a, double b) { return fmax(a, b); }

/* ---- Mat3 (reference/rust/src/su3.rs:77-230) ---- */
mat3 m3_zero(void);
mat3 m3_identity(void);
mat3 m3_add(mat3 a, mat3 b);
mat3 m3_sub(mat3 a, mat3 b);
mat3 m3_scale_real(mat3 a, double f);
mat3 m3_scale_complex(mat3 a, c64 f);
mat3 m3_mul(mat3 a, mat3 b);
mat3 m3_dagger(mat3 a);
c64 m3_trace(mat3 a);
c64 m3_det(mat3 a);
double m3_max_abs(mat3 a);
double m3_one_norm(mat3 a);
double m3_max_residual(mat3 a, mat3 b);
double m3_hermiticity_residual(mat3 a);
double m3_unitarity_residual(mat3 a);
double m3_determinant_residual(mat3 a);
int m3_finite(mat3 a);

/* Su3 checked constructors (su3.rs:242-288). */
int su3_checked(mat3 a, mat3 *out);
int su3_mul_checked(mat3 a, mat3 b, mat3 *out);
int su3_gell_mann(int index, mat3 *out);
int su3_generator(int index, mat3 *out);
int su3_matrix_exponential(mat3 a, mat3 *out);
int su3_from_algebra(const double coef[8], mat3 *out);

/* Lattice geometry shared by the SU(2) and SU(3) lattices
 * (lib.rs:242-320, su3_lattice.rs:85-151). */
typedef struct { int64_t n[4]; } extents4;

static inline int64_t site_index(const extents4 *e, const int64_t x[4]) {
    return ((x[0] * e->n[1] + x[1]) * e->n[2] + x[2]) * e->n[3] + x[3];
}
static inline void nb_plus(const extents4 *e, const int64_t x[4], int mu, int64_t y[4]) {
    memcpy(y, x, 4 * sizeof(int64_t));
    y[mu] = (x[mu] + 1) % e->n[mu];
}
static inline void nb_minus(const extents4 *e, const int64_t x[4], int mu, int64_t y[4]) {
    memcpy(y, x, 4 * sizeof(int64_t));
    y[mu] = x[mu] == 0 ? e->n[mu] - 1 : x[mu] - 1;
}
static inline int coord_ok(const extents4 *e, const int64_t x[4]) {
    for (int i = 0; i < 4; ++i) if (x[i] < 0 || x[i] >= e->n[i]) return 0;
    return 1;
}
int extents_from(const int64_t *ext, extents4 *e, int64_t max_links, int64_t *links_out);

/* SU(3) AoS lattice: 18 doubles per link, link = site*4+mu, row-major
 * complex entries (re, im) -- the in-memory order of `Vec<Su3>`. */
static inline mat3 su3_load(const double *links, int64_t link) {
    mat3 m; memcpy(&m, links + link * 18, sizeof(mat3)); return m;
}
static inline void su3_store(double *links, int64_t link, mat3 m) {
    memcpy(links + link * 18, &m, sizeof(mat3));
}
static inline mat3 su3_link(const extents4 *e, const double *links, const int64_t x[4], int mu) {
    return su3_load(links, site_index(e, x) * 4 + mu);
}

int su3_plaquette(const extents4 *e, const double *links, const int64_t x[4], int mu, int nu,
                  mat3 *out);

/* SplitMix64 (su2_ensemble.rs:24-50). */
static inline uint64_t or_mix64(uint64_t v) {
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
    return v ^ (v >> 31);
}
static inline uint64_t sm_next(uint64_t *state) {
    *state += 0x9E3779B97F4A7C15ULL;
    return or_mix64(*state);
}
static inline double sm_unit(uint64_t *state) {
    return (double)(sm_next(state) >> 11) * (1.0 / 9007199254740992.0);
}

#endif /* OR_INTERNAL_H */
